"""Batched exp(tA)p over many FSP instances in one persistent launch (cufsp_batch_* in cufsp.h).

The reference solves one instance per KryExpvFSP object (src/KryExpvFSP.cu:184-188); parameter
sweeps and likelihood evaluations there loop over objects.  BatchKrylov solves hundreds of instances
of one reaction network -- each with its own box, factor tables and rates -- to a common final
time with the whole adaptive Krylov solve on the device.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import BatchDesc, BatchStat
from .fsp import _ptr, _stream


class BatchKrylov:
    """Instances share `nu` ([n_reactions, n_species] net changes); instance i has bounds[i],
    factor tables tables[i] ([n_reactions, sum_s(b_s + 1)], the reference layout) and rate
    coefficients coefs[i].  m <= 32, tol as KryExpvFSP; iop / q_iop: incomplete orthogonalisation."""

    def __init__(self, nu, bounds, tables, coefs, m: int = 30, tol: float = 1e-8, iop: bool = False, q_iop: int = 2,
                 lib: C.CDLL | None = None):
        self._lib = lib or _lib.load()
        nu = np.asarray(nu, np.int32)
        self.nr, self.ns = nu.shape
        self.n_instances = len(bounds)
        vals, cols, rows = [], [], [0]
        for r in range(self.nr):
            for s in range(self.ns):
                if nu[r, s]:
                    vals.append(int(nu[r, s]))
                    cols.append(s)
            rows.append(len(vals))
        self._vals = np.asarray(vals or [0], np.int32)
        self._cols = np.asarray(cols or [0], np.int32)
        self._rows = np.asarray(rows, np.int32)
        self._bounds = np.ascontiguousarray(np.asarray(bounds, np.int32).reshape(self.n_instances, self.ns))
        self._tabs = [np.ascontiguousarray(np.asarray(t, np.float64)) for t in tables]
        self._coefs = np.ascontiguousarray(np.asarray(coefs, np.float64).reshape(self.n_instances, self.nr))
        tab_ptrs = (C.POINTER(C.c_double) * self.n_instances)(
            *[t.ctypes.data_as(C.POINTER(C.c_double)) for t in self._tabs])
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))  # noqa: E731
        d = BatchDesc(self.ns, self.nr, ip(self._vals), ip(self._cols), ip(self._rows), self.n_instances,
                      ip(self._bounds), tab_ptrs, self._coefs.ctypes.data_as(C.POINTER(C.c_double)))
        h = C.c_void_p()
        _lib.check(self._lib, self._lib.cufsp_batch_create(C.byref(d), int(m), float(tol), int(bool(iop)), int(q_iop),
                                                           C.byref(h)), "cufsp_batch_create")
        self._h = h
        off = np.zeros(self.n_instances + 1, np.int64)
        _lib.check(self._lib, self._lib.cufsp_batch_layout(self._h, off.ctypes.data_as(C.POINTER(C.c_int64))),
                   "cufsp_batch_layout")
        self.offsets = off
        self.sizes = np.prod(self._bounds + 1, axis=1).astype(np.int64)

    @classmethod
    def from_models(cls, models_, m: int = 30, tol: float = 1e-8, iop: bool = False, q_iop: int = 2):
        nu = models_[0].nu
        for mm in models_:
            if not np.array_equal(mm.nu, nu):
                raise ValueError("all instances of a batch share one stoichiometry")
        return cls(nu, [mm.bounds for mm in models_], [mm.tables for mm in models_],
                   np.stack([mm.coefs(0.0) for mm in models_]), m=m, tol=tol, iop=iop, q_iop=q_iop)

    @property
    def total(self) -> int:
        return int(self.offsets[-1])

    def pack(self, vectors):
        """Host vectors (one per instance) -> packed device tensor."""
        import torch
        buf = np.zeros(self.total)
        for i, v in enumerate(vectors):
            buf[self.offsets[i]:self.offsets[i] + self.sizes[i]] = v
        return torch.as_tensor(buf, device="cuda")

    def unpack(self, packed) -> list[np.ndarray]:
        a = packed.detach().cpu().numpy() if hasattr(packed, "detach") else np.asarray(packed)
        return [a[self.offsets[i]:self.offsets[i] + self.sizes[i]].copy() for i in range(self.n_instances)]

    def set_coefs(self, coefs) -> None:
        c = np.ascontiguousarray(np.asarray(coefs, np.float64).reshape(self.n_instances, self.nr))
        _lib.check(self._lib, self._lib.cufsp_batch_set_coefs(self._h, c.ctypes.data_as(C.POINTER(C.c_double))),
                   "cufsp_batch_set_coefs")

    def set_limits(self, max_steps: int, max_reject: int) -> None:
        _lib.check(self._lib, self._lib.cufsp_batch_set_limits(self._h, int(max_steps), int(max_reject)),
                   "cufsp_batch_set_limits")

    def set_shape(self, cluster_ctas: int = 0, threads: int = 0) -> None:
        """Fix the launch shape; (0, 0) lets the autotuner choose at the next solve."""
        _lib.check(self._lib, self._lib.cufsp_batch_set_shape(self._h, int(cluster_ctas), int(threads)),
                   "cufsp_batch_set_shape")

    def solve(self, t_final: float, packed, stream=None, check: bool = True) -> list[dict]:
        """packed (device, float64, length total): p(0) in, exp(t_final A_i) p_i(0) out."""
        st = (BatchStat * self.n_instances)()
        rc = self._lib.cufsp_batch_solve(self._h, float(t_final), _ptr(packed), _stream(stream), st)
        if check:
            _lib.check(self._lib, rc, "cufsp_batch_solve")
        return [s.as_dict() for s in st]

    def describe(self) -> str:
        buf = C.create_string_buffer(512)
        _lib.check(self._lib, self._lib.cufsp_batch_describe(self._h, buf, len(buf)), "cufsp_batch_describe")
        return buf.value.decode()

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.cufsp_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _main(argv=None) -> None:
    """Solve models.gene_batch(sets, lo..hi mRNA bounds) to t and print the launch shape and totals
    (used to reproduce the profiles of the batched kernel)."""
    import argparse
    import json
    import time

    import torch

    from . import models
    ap = argparse.ArgumentParser(prog="python -m cuda_fsp_b200.batch")
    ap.add_argument("--sets", type=int, default=16)
    ap.add_argument("--lo", type=int, default=40)
    ap.add_argument("--hi", type=int, default=60)
    ap.add_argument("--t", type=float, default=1.0)
    ap.add_argument("--m", type=int, default=30)
    ap.add_argument("--cluster", type=int, default=8)
    ap.add_argument("--threads", type=int, default=256)
    ap.add_argument("--repeat", type=int, default=2)
    a = ap.parse_args(argv)
    ms = models.gene_batch(a.sets, lo=a.lo, hi=a.hi)
    B = BatchKrylov.from_models(ms, m=a.m, tol=1e-8)
    if a.cluster > 0:
        B.set_shape(a.cluster, a.threads)
    p0 = B.pack([mm.p0() for mm in ms])
    dt, st = 0.0, []
    for _ in range(a.repeat):
        p = p0.clone()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = B.solve(a.t, p)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
    print(json.dumps({"launch": B.describe(), "states": int(B.sizes.sum()), "steps": sum(s["steps"] for s in st),
                      "matvecs": sum(s["matvecs"] for s in st), "s_last_solve": round(dt, 4)}))


if __name__ == "__main__":
    _main()


# ---- several GPUs: one rank per GPU, parameter sets partitioned, one final gather --------------

def partition_instances(sizes, world: int) -> list[list[int]]:
    """Split instance indices over `world` ranks so that the ranks' total state counts are as even as
    a largest-first greedy assignment makes them (the solve time of an instance grows with its size).
    Deterministic: every rank computes the same partition."""
    sizes = np.asarray(sizes, np.int64)
    load = np.zeros(world, np.int64)
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        r = int(np.argmin(load))
        parts[r].append(i)
        load[r] += sizes[i]
    return [sorted(p) for p in parts]


def _gather_flat(local: np.ndarray, counts: list[int], group=None) -> list[np.ndarray]:
    """all_gather of variable-length float64 vectors whose lengths every rank knows (`counts[r]`):
    padded to the longest, gathered as tensors (NCCL: device tensors, gloo: host tensors), trimmed."""
    import torch
    import torch.distributed as dist
    world = len(counts)
    width = max(1, max(counts))
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else torch.device("cpu")
    buf = torch.zeros(width, dtype=torch.float64, device=dev)
    if local.size:
        buf[: local.size] = torch.from_numpy(np.ascontiguousarray(local, np.float64)).to(dev)
    parts = [torch.empty(width, dtype=torch.float64, device=dev) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    return [parts[r][: counts[r]].cpu().numpy() for r in range(world)]


def solve_sharded(models_, t_final: float, rank: int, world: int, m: int = 30, tol: float = 1e-8,
                  solver=None, group=None, gather: str = "summary", reduce=None) -> list:
    """Solve this rank's share of the instances (exp(t_final A_i) p_i(0) from each model's p0) and
    gather the results on all ranks -- the only collective.  `gather`:
      "summary"  every instance's final mass, steps and status (a dict per instance);
      "vectors"  the solution vectors themselves (a float64 array per instance, one padded tensor
                 all_gather of each rank's packed vectors);
      "reduce"   reduce(model, vector, stat) computed on the owning rank, gathered as objects (for
                 caller-chosen reductions: marginals, moments, likelihood terms).
    `solver(models, t)` -> list of (vector, stat) may replace the GPU batch (host tests)."""
    import torch.distributed as dist

    parts = partition_instances([mm.n_states for mm in models_], world)
    mine = parts[rank]
    vecs, stats = [], []
    if mine:
        sub = [models_[i] for i in mine]
        if solver is None:
            B = BatchKrylov.from_models(sub, m=m, tol=tol)
            p = B.pack([mm.p0() for mm in sub])
            stats = B.solve(t_final, p)
            vecs = B.unpack(p)
        else:
            vecs, stats = zip(*solver(sub, t_final))
    if gather == "vectors":
        local = np.concatenate([np.asarray(v, np.float64) for v in vecs]) if mine else np.zeros(0)
        counts = [int(sum(models_[i].n_states for i in part)) for part in parts]
        flat = [local] if world == 1 else _gather_flat(local, counts, group)
        out: list = [None] * len(models_)
        for r, part in enumerate(parts):
            off = 0
            for i in part:
                n = models_[i].n_states
                out[i] = flat[r][off:off + n]
                off += n
        return out
    if gather == "reduce":
        if reduce is None:
            raise ValueError("gather='reduce' needs reduce(model, vector, stat)")
        local = [(i, reduce(models_[i], v, st)) for i, v, st in zip(mine, vecs, stats)]
    elif gather == "summary":
        local = [(i, {"mass": float(np.sum(v)), "steps": int(st["steps"]), "status": int(st["status"])})
                 for i, v, st in zip(mine, vecs, stats)]
    else:
        raise ValueError(f"unknown gather mode {gather!r}")
    if world == 1:
        gathered = [local]
    else:
        gathered = [None] * world
        dist.all_gather_object(gathered, local, group=group)
    out = [None] * len(models_)
    for part in gathered:
        for i, value in part:
            out[i] = value
    return out


def gradient_sharded(likelihood, coef_sets, rank: int, world: int, workers: int = 4, group=None, grad_fn=None):
    """d log L / d log c for many parameter sets over several GPUs: the sets are split into `world`
    contiguous blocks, each rank computes its block (Likelihood.gradient_batched, or grad_fn(sets) ->
    (logL [k], grad [k, nr]) in host tests), and one all_gather of the packed (log L, gradient) rows
    gives every rank all of them.  Returns (logL [n_sets], grad [n_sets, n_reactions])."""
    c = np.asarray(coef_sets, np.float64)
    n_sets, nr = c.shape
    bounds = [n_sets * r // world for r in range(world + 1)]
    lo, hi = bounds[rank], bounds[rank + 1]
    if hi > lo:
        ll, g = (grad_fn or (lambda s: likelihood.gradient_batched(s, workers=workers)))(c[lo:hi])
        local = np.concatenate([np.asarray(ll, np.float64)[:, None], np.asarray(g, np.float64)], axis=1).ravel()
    else:
        local = np.zeros(0)
    counts = [(bounds[r + 1] - bounds[r]) * (nr + 1) for r in range(world)]
    flat = [local] if world == 1 else _gather_flat(local, counts, group)
    rows = np.concatenate([f.reshape(-1, nr + 1) for f in flat], axis=0)
    return rows[:, 0].copy(), rows[:, 1:].copy()
