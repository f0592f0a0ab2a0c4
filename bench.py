#!/usr/bin/env python3
"""Benchmark of the FSP generator action y += A(t) x (the hot path) on B200.

Workload: mass_action_3 -- 3 species, 9 mass-action reactions, box 255^3 = 16,777,216 states,
KRONECKER (matrix-free, factorised) format, FP64.  One step = one application of the generator to
the full state vector through the C ABI (cufsp_mat_apply, accumulate form).

  value     algorithmic HBM GB/s = 24 B/state * states / time (x read once, y read + written),
            device-resident inputs, CUDA events on the launching stream, summed over ranks
  e2e       the same metric through cufsp_mat_action_host with pinned HOST x, y: H2D of x and y and
            D2H of y inside the timed region
  roofline  the kernel's achieved GB/s against the measured HBM copy bandwidth
  cpu_baseline  the FP64 host oracle (OpenMP CSR SpMV restating the reference's assembly) timed on
            the host cores on the same 255^3 workload (about 10 s of steps)
  secondary [expmv solves/s on birth_death_2 (32,768 states, t = 10, m = 30, tol 1e-8) with the
             oracle's host solve time beside it;
             batched expmv solves/s on 256 gene-expression parameter sets (one persistent launch) with
             the plain single-instance path timed on a sample of the same instances;
             grad logL grads/s on the 131,072-state gene-expression model (adjoint)]

--impl reference: the reference has no CPU implementation of this path; its CPU restatement (the
oracle, "port") is timed on the same metric and workload sample with all host threads.
Multi-GPU (--gpus N under torchrun): the action of one generator does not shard, so every rank
runs an independent replica (weak scaling); time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "matvec HBM GB/s; expmv solves/s & ∇logL grads/s at 1e-8 err vs plain FSP"
BYTES_PER_STATE = 24
WORKLOAD = ("mass_action_3 generator action y += A(t)x: 3 species, 9 reactions, box 255^3 = 16,777,216 states, "
            "KRONECKER matrix-free, FP64")
CPU_BOUNDS = (255, 255, 255)  # the CPU baseline runs the same workload as the GPU arm


def workload_config(world: int) -> dict:
    """The `config` of both arms' lines (identical, so that the two lines describe one workload)."""
    return {"workload": WORKLOAD, "n_states": 16777216, "format": "KRONECKER", "form": "y += A x",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "l2": "4 rotating (x, y) input pairs, 1.07 GB > 126 MB L2", "bytes_per_state": BYTES_PER_STATE}


def measured_peak_hbm() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def profile_traffic() -> float | None:
    """DRAM bytes per launch of the KRONECKER action from the committed ncu summary, if present."""
    p = ROOT / "profiles" / "kron_plane_mass_action_3.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """SM clock and clock-event reasons sampled through NVML every ~1 ms during the timed region
    (read-only queries; nothing is set)."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown", 0x4: "sw_power_cap"}

    def __init__(self, index: int):
        self.index = index
        self.samples: list[tuple[float, float]] = []  # (time, MHz)
        self.reasons: set[str] = set()
        self.marks: list[float] = []
        self.smax = None
        self._stop = threading.Event()
        self.nvml = None

    def mark(self):
        """Start / end of the timed window inside the sampled period."""
        self.marks.append(time.perf_counter())

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
        except Exception:
            self.nvml = None
            return
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def _run(self):
        pv = self.nvml
        while not self._stop.is_set():
            try:
                self.samples.append((time.perf_counter(), float(pv.nvmlDeviceGetClockInfo(self.h, pv.NVML_CLOCK_SM))))
                r = pv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for bit, name in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.0002)

    def stop(self) -> dict:
        if self.nvml is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"], "samples": 0}
        self._stop.set()
        self.t.join(timeout=2)
        mhz = [v for _, v in self.samples]
        out = {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": self.smax,
               "reasons": sorted(self.reasons), "samples": len(mhz)}
        if len(self.marks) >= 2:  # the samples inside the timed window, and the warm-up window before it
            a, b = self.marks[0], self.marks[1]
            inside = [v for t, v in self.samples if a <= t <= b]
            before = [v for t, v in self.samples if t < a]
            out["timed_window"] = {"sm_mhz": statistics.median(inside) if inside else None, "samples": len(inside),
                                   "ms": round((b - a) * 1e3, 3)}
            out["warmup_window"] = {"sm_mhz": statistics.median(before) if before else None, "samples": len(before)}
            if inside:
                out["sm_mhz"] = statistics.median(inside)
        return out


def nvml_index(dev) -> int:
    """NVML index of a CUDA device (NVML ignores CUDA_VISIBLE_DEVICES): match the PCI bus id."""
    try:
        import pynvml
        import torch
        p = torch.cuda.get_device_properties(dev)
        pynvml.nvmlInit()
        for i in range(pynvml.nvmlDeviceGetCount()):
            pci = pynvml.nvmlDeviceGetPciInfo(pynvml.nvmlDeviceGetHandleByIndex(i))
            if pci.bus == p.pci_bus_id and pci.device == p.pci_device_id and pci.domain == p.pci_domain_id:
                return i
    except Exception:
        pass
    return 0


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_oracle_gbs(min_steps: int, warmup: int = 3, bounds=CPU_BOUNDS, budget_s: float = 10.0) -> dict:
    """Time the oracle's OpenMP CSR SpMV (y += A x, restating the reference's per-reaction CSR
    assembly) on the workload itself: `warmup` untimed steps, then at least `min_steps` steps and
    about `budget_s` seconds of CPU work, all host threads."""
    import oracle
    from cuda_fsp_b200 import models
    m = models.mass_action_3(bounds=bounds)
    csr = oracle.assemble_model(m)
    rng = np.random.default_rng(0)
    x = rng.uniform(0, 1, m.n_states)
    y = np.zeros(m.n_states)
    c = m.coefs(0)
    for _ in range(max(1, warmup)):
        y = csr.spmv(c, x, y, beta=1.0)
    steps = 0
    t0 = time.perf_counter()
    while steps < min_steps or time.perf_counter() - t0 < budget_s:
        y = csr.spmv(c, x, y, beta=1.0)
        steps += 1
    dt = (time.perf_counter() - t0) / steps
    return {"value": BYTES_PER_STATE * m.n_states / dt / 1e9, "unit": "GB/s", "cores": oracle.num_threads(),
            "kind": "port", "sample": f"oracle CSR SpMV y += A x on box {bounds[0]}x{bounds[1]}x{bounds[2]} "
                                      f"({m.n_states} states, the 9-reaction workload), {steps} steps after "
                                      f"{max(1, warmup)} untimed",
            "ms_per_step": dt * 1e3}


def reference_gpu_kernel() -> dict | None:
    """The reference's own Kronecker action (fspmat_sdkron_mv through SDKronMatSet::action,
    src/fspmat_kron_kernels.cu:31-129, built unmodified for sm_100a into oracle/_ref) on the full
    255^3 workload: a reported baseline beside the CPU one, None without a GPU or the build."""
    try:
        import torch
        if not torch.cuda.is_available():
            return None
    except Exception:
        return None
    import oracle
    from cuda_fsp_b200 import models
    R = oracle.ref()
    if R is None:
        return None
    m = models.mass_action_3()
    b = np.asarray(m.bounds, np.int32)
    sv, sc, sr = m.stoich_csr()
    tab = np.ascontiguousarray(m.tables)
    c = np.ascontiguousarray(m.coefs(0))
    ms = R.ref_gpu_kron_time(m.ns, m.nr, b.ctypes.data, sv.ctypes.data, sc.ctypes.data, sr.ctypes.data,
                             tab.ctypes.data, c.ctypes.data, 100)
    if ms <= 0:
        return None
    out = {"value": round(BYTES_PER_STATE * m.n_states / (ms * 1e-3) / 1e9, 3), "unit": "GB/s",
           "ms_per_action": round(ms, 4),
           "kernel": "reference fspmat_sdkron_mv built for sm_100a, called through SDKronMatSet::action "
                     "(coefficient copy and device synchronisation per call, as the reference does); "
                     "100 actions (the count of the reference's benchmark_fsp_mat.cu:158), CUDA events, x and y resident"}
    # The reference's HYB format (src/fspmat_hyb_kernels.cu:66-106) on the same workload, built by its
    # own fill kernel from a factor-table PropFun; GB/s counted with the sparse format's algorithmic
    # bytes (x, y and one propensity table row per reaction: 24 + 8 nr B/state), as our sparse leg is.
    import ctypes as C
    hms = C.c_double(0.0)
    rc = R.ref_gpu_hyb_tables(m.ns, m.nr, b.ctypes.data, sv.ctypes.data, sc.ctypes.data, sr.ctypes.data,
                              tab.ctypes.data, c.ctypes.data, None, None, 100, C.addressof(hms))
    if rc == 0 and hms.value > 0:
        out["hyb"] = {"value": round((24 + 8 * m.nr) * m.n_states / (hms.value * 1e-3) / 1e9, 3), "unit": "GB/s",
                      "ms_per_action": round(hms.value, 4), "bytes_per_state": 24 + 8 * m.nr,
                      "kernel": "reference fspmat_hyb_mv built for sm_100a through HYBMatSet::action, 100 actions"}
    return out


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    steps = max(1, args.steps)
    cb = cpu_oracle_gbs(steps, max(3, args.warmup))
    line = {"impl": "reference", "metric": METRIC, "value": round(cb["value"], 3), "unit": "GB/s",
            "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup, "ms_per_step": round(cb["ms_per_step"], 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload_config(args.gpus),
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": round(cb["value"], 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    gk = reference_gpu_kernel()
    if gk is not None:
        line["reference_gpu_kernel"] = gk
    print(json.dumps(line), flush=True)


def expmv_secondary() -> dict:
    import torch
    from cuda_fsp_b200 import FSPMat, KryExpvFSP, MatrixFormat, models
    m = models.birth_death_2()
    A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    p0 = torch.as_tensor(m.p0(), device="cuda")
    c = m.coefs(0)
    v = p0.clone()
    KryExpvFSP(10.0, A, v, m=30, tol=1e-8, coefs=c).solve()  # warm-up
    reps = 3
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    st = None
    for _ in range(reps):
        v.copy_(p0)
        st = KryExpvFSP(10.0, A, v, m=30, tol=1e-8, coefs=c).solve()
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / reps
    return {"metric": "expmv solves/s", "workload": "birth_death_2, 32,768 states, t = 10, m = 30, tol 1e-8",
            "value": round(1.0 / dt, 3), "ms_per_solve": round(dt * 1e3, 3), "krylov_steps": st["n_steps"],
            "matvecs": st["n_matvec"]}


def expmv_large_secondary(t_final: float = 0.2) -> dict:
    """Krylov exp(tA)p0 on the 255^3 workload (mass_action_3, p0 = Poisson(5)^3, tol 1e-8), timed to
    completion over the stated horizon t = 0.2 (the whole t = 20 needs ~4e4 full-orthogonalisation
    steps: the x1 x2 and x1 x3 propensities make the network stiff), in two configurations:
      m = 30, full orthogonalisation (the reference's default), with its Arnoldi traffic rate against
        the HBM roofline: algorithmic bytes per step (16 (m+1) + 8 (m (m+1) + 2m) + 8 (m+2)) n = 8,672 n;
      m = 60, incomplete orthogonalisation against the last 3 vectors (the reference's IOP option; the
        fastest of m in {30, 45, 60} x q in {full, 2, 3, 4} in the --leg iopsweep measurement), about a
        third of the steps at a cost per step of ~(16 + 8 (2q + 3)) (m + 1) n,
    and the 1-norm difference between the two results."""
    import torch
    from cuda_fsp_b200 import FSPMat, KryExpvFSP, MatrixFormat, models
    mm = models.mass_action_3()
    n = mm.n_states
    A = FSPMat.from_model(mm, MatrixFormat.KRONECKER)
    p0 = torch.as_tensor(mm.p0(), device="cuda")
    out = {"metric": "expmv solves/s", "workload": f"mass_action_3 255^3 = 16,777,216 states, p0 = Poisson(5)^3, "
           f"t = {t_final}, tol 1e-8, timed to completion"}
    res = {}
    for name, kw in (("m30_full", dict(m=30)), ("m60_iop3", dict(m=60, iop=True, q_iop=3))):
        v = p0.clone()
        KryExpvFSP(t_final, A, v, tol=1e-8, coefs=mm.coefs(0), **kw).step()  # warm-up: tables, first launches
        v.copy_(p0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        E = KryExpvFSP(t_final, A, v, tol=1e-8, coefs=mm.coefs(0), **kw)  # a new solve, as a caller makes it
        E.max_nstep = 1 << 20
        st = E.solve()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        res[name] = v
        out[name] = {"solves_per_s": round(1.0 / dt, 4), "s_per_solve": round(dt, 3), "krylov_steps": st["n_steps"],
                     "rejected": st["n_reject"], "matvecs": st["n_matvec"],
                     "ms_per_step": round(dt / st["n_steps"] * 1e3, 3), "mass": round(v.sum().item(), 12)}
        if name == "m30_full":
            bps = (16 * 31 + 8 * (30 * 31 + 60) + 8 * 32) * n
            gbs = st["n_steps"] * bps / dt / 1e9
            peak, _ = measured_peak_hbm()
            out[name].update({"arnoldi_bytes_per_step": bps, "achieved_gbs": round(gbs, 1),
                              "frac_of_measured_hbm": round(gbs / peak, 4)})
    out["value"] = max(out["m30_full"]["solves_per_s"], out["m60_iop3"]["solves_per_s"])
    out["max_1norm_diff_between_configs"] = float((res["m30_full"] - res["m60_iop3"]).abs().sum().item())
    return out


def sparse_secondary(steps: int = 200) -> dict:
    """The sparse-format generator action (CSR/HYB: reaction-major propensity table a_r(x_i)) on the
    255^3 workload, y += A x over 2 rotating (x, y) pairs (537 MB > L2), CUDA events.  Algorithmic
    bytes: x read, y read and written, and the nr-row table read: (24 + 8 nr) B/state."""
    import torch
    from cuda_fsp_b200 import FSPMat, MatrixFormat, models
    m = models.mass_action_3()
    n = m.n_states
    A = FSPMat.from_model(m, MatrixFormat.HYB)
    g = torch.Generator(device="cuda").manual_seed(5)
    xs = [torch.rand(n, dtype=torch.float64, device="cuda", generator=g) for _ in range(2)]
    ys = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(2)]
    for i in range(4):
        A.action(0.0, xs[i % 2], ys[i % 2])
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(steps):
        A.action(0.0, xs[i % 2], ys[i % 2])
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    bps = 24 + 8 * m.nr
    gbs = bps * n / (ms * 1e-3) / 1e9
    peak, _ = measured_peak_hbm()
    return {"metric": "sparse-format matvec GB/s", "workload": "mass_action_3 255^3, HYB (propensity table), y += A x",
            "value": round(gbs, 1), "us_per_action": round(ms * 1e3, 2), "bytes_per_state": bps,
            "frac_of_hbm_peak": round(gbs / peak, 4), "kernel": A.describe()}


def kron_general_secondary(steps: int = 200) -> dict:
    """The KRONECKER action of the 5-species gene network on an HBM-sized box (1,1,1,127,8191) =
    8,388,608 states, outside the plane kernel's shape, through the kernel specialised per network and
    box: y += A x over 2 rotating (x, y) pairs (268 MB > L2), CUDA events, 24 B/state."""
    import torch
    from cuda_fsp_b200 import FSPMat, MatrixFormat, models
    m = models.gene_expression((1, 1, 1, 127, 8191), time_varying=False)
    n = m.n_states
    A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    g = torch.Generator(device="cuda").manual_seed(6)
    xs = [torch.rand(n, dtype=torch.float64, device="cuda", generator=g) for _ in range(2)]
    ys = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(2)]
    c = m.coefs(0)
    for i in range(4):
        A.apply(xs[i % 2], ys[i % 2], coefs=c, beta=1.0)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(steps):
        A.apply(xs[i % 2], ys[i % 2], coefs=c, beta=1.0)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    gbs = BYTES_PER_STATE * n / (ms * 1e-3) / 1e9
    peak, _ = measured_peak_hbm()
    return {"metric": "KRONECKER matvec GB/s (general networks)", "workload": "gene_expression 5 species, box "
            "1x1x1x127x8191 = 8,388,608 states, 12 reactions, y += A x", "value": round(gbs, 1),
            "us_per_action": round(ms * 1e3, 2), "frac_of_hbm_peak": round(gbs / peak, 4), "kernel": A.describe()}


def bdf_secondary() -> dict:
    """BDF leg: the time-varying gene-expression model (131,072 states, switching rate
    k0 sigmoid((t - 5) / 0.5)) from p0 to t = 60 by the device BDF integrator (rtol 1e-8, atol 1e-14;
    the reference's CVODE path).  The oracle's host BDF is timed on the sample [0, 6] (the switch and
    408 of the ~700 steps), with the device solve of the same sample beside it."""
    import torch
    import oracle
    from cuda_fsp_b200 import BDFIntegrator, FSPMat, MatrixFormat, models
    m = models.gene_expression((1, 1, 1, 127, 127), time_varying=True)
    A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    p0 = torch.as_tensor(m.p0(), device="cuda")

    def solve(t_end):
        B = BDFIntegrator(A, rtol=1e-8, atol=1e-14)
        p = p0.clone()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        B.init(0.0, p)
        B.advance(t_end, p)
        torch.cuda.synchronize()
        return time.perf_counter() - t0, B.stats, p

    solve(6.0)  # warm-up
    full, st, p = solve(60.0)
    sample, st6, _ = solve(6.0)
    t0 = time.perf_counter()
    _, rst, rc = oracle.bdf(oracle.assemble_model(m), m.coefs, 0.0, m.p0(), [6.0], rtol=1e-8, atol=1e-14)
    cpu = time.perf_counter() - t0
    return {"metric": "BDF solve s", "workload": "gene_expression 131,072 states, time-varying switch, t = 60, "
            "rtol 1e-8, atol 1e-14", "value": round(full, 4), "steps": st["n_steps"], "order": st["order"],
            "mass": round(p.sum().item(), 12), "sample_t6_s": round(sample, 4), "sample_t6_steps": st6["n_steps"],
            "cpu_oracle_sample_t6_s": round(cpu, 3), "cpu_oracle_sample_t6_steps": rst["n_steps"],
            "cpu_oracle_rc": rc}


def cpu_expmv_ms() -> float:
    """The oracle's host Krylov exp(tA)v on birth_death_2 (same workload as the expmv leg)."""
    import oracle
    from cuda_fsp_b200 import models
    m = models.birth_death_2()
    csr = oracle.assemble_model(m)
    t0 = time.perf_counter()
    w, st, rc = oracle.expv(csr, m.coefs(0), 10.0, m.p0(), m=30, tol=1e-8)
    return (time.perf_counter() - t0) * 1e3


def batched_secondary(n_sets: int = 256, sample: int = 4) -> dict:
    """Batched leg: n_sets parameter sets of the gene-expression model (rates within one decade of nominal,
    mRNA bounds 63..255) solved to t = 30 in one persistent launch; the plain single-instance Krylov
    path is timed on `sample` of the same instances and its results compared (1-norm)."""
    import torch
    from cuda_fsp_b200 import BatchKrylov, FSPMat, KryExpvFSP, MatrixFormat, models
    ms = models.gene_batch(n_sets)
    B = BatchKrylov.from_models(ms, m=30, tol=1e-8)
    p0 = B.pack([mm.p0() for mm in ms])
    p = p0.clone()
    t0 = time.perf_counter()
    B.solve(30.0, p)  # chooses the launch shape (autotuner), captures the graph and warms up; untimed
    tune_s = time.perf_counter() - t0
    p.copy_(p0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    stats = B.solve(30.0, p)
    torch.cuda.synchronize()
    batch_s = time.perf_counter() - t0
    out = B.unpack(p)
    idx = [i * n_sets // sample for i in range(sample)]
    single_s, errs = 0.0, []
    for i in idx:
        mm = ms[i]
        A = FSPMat.from_model(mm, MatrixFormat.KRONECKER)
        v = torch.as_tensor(mm.p0(), device="cuda")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        KryExpvFSP(30.0, A, v, m=30, tol=1e-8, coefs=mm.coefs(0)).solve()
        torch.cuda.synchronize()
        single_s += time.perf_counter() - t0
        errs.append(float(np.abs(v.cpu().numpy() - out[i]).sum()))
    return {"metric": "batched expmv solves/s", "workload": f"{n_sets} gene-expression parameter sets, "
            f"{int(B.sizes.sum())} states in total, t = 30, m = 30, tol 1e-8, one persistent launch",
            "value": round(n_sets / batch_s, 3), "s_per_batch": round(batch_s, 3),
            "single_instance_solves_per_s": round(len(idx) / single_s, 3),
            "single_instance_sample": f"{len(idx)} of the same instances through KryExpvFSP",
            "max_1norm_diff_vs_single": max(errs), "steps_mean": float(np.mean([s_["steps"] for s_ in stats])),
            "launch": B.describe(), "first_call_s": round(tune_s, 1),
            "autotune_s": _autotune_seconds(B.describe())}


def _autotune_seconds(describe: str):
    """The autotuner's own wall time (candidate compiles and trial launches), as the solver reports it;
    None when the launch shape came from the tuning cache or the environment."""
    import re
    hit = re.search(r"autotuner ([0-9.]+) s", describe)
    return float(hit.group(1)) if hit else None


def batched_sharded_secondary(world: int, rank: int, dev, per_rank: int = 256) -> dict | None:
    """Batched leg over N GPUs: per_rank * N parameter sets partitioned by state count over the ranks
    (cuda_fsp_b200.batch.solve_sharded, weak scaling), one final gather of the per-instance results;
    time = max over ranks."""
    import torch
    import torch.distributed as dist
    from cuda_fsp_b200 import models
    from cuda_fsp_b200.batch import solve_sharded
    ms = models.gene_batch(per_rank * world)
    solve_sharded(ms[:world * 8], 1.0, rank, world)  # warm-up: kernel compilation and launch shape
    dist.barrier()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    res = solve_sharded(ms, 30.0, rank, world)
    torch.cuda.synchronize(dev)
    dt = torch.tensor([time.perf_counter() - t0], device=dev)
    dist.all_reduce(dt, op=dist.ReduceOp.MAX)
    if rank != 0:
        return None
    return {"metric": "batched expmv solves/s", "workload": f"{len(ms)} gene-expression parameter sets over "
            f"{world} GPUs ({per_rank} per GPU), t = 30, m = 30, tol 1e-8", "value": round(len(ms) / dt.item(), 3),
            "s_per_batch": round(dt.item(), 3), "scaling": "weak", "failed": sum(1 for r in res if r["status"] != 0)}


def gradient_secondary(n_sets: int = 64, workers: int = 4, sample: int = 8) -> dict:
    """Gradient leg: d log L / d log theta for the 12 rates of the gene-expression model (131,072 states) from
    1,000 seeded-SSA cells at 8 log-spaced times in [1, 60], (n, c) histograms marginalised over the
    gene states, for n_sets parameter sets (rates within half a decade of nominal) at once
    (cufsp_likelihood_grad_batched: `workers` concurrent adjoint solves, each worker's persistent
    Arnoldi passes on an equal share of the SMs, so that one solve's passes overlap the others' host-side
    step control).  The comparator is the same path one set at a time on `sample` of the same sets
    (every n_sets/sample-th: the sets differ in cost, since the step count follows the rates), whose
    results the batched ones must match; one log-likelihood evaluation is timed beside it."""
    import torch
    from cuda_fsp_b200 import Likelihood, generate_data, histograms, models
    m = models.gene_expression((1, 1, 1, 127, 127), time_varying=False)
    times = np.geomspace(1.0, 60.0, 8)
    snaps = generate_data(m, times, [0, 0, 0, 0, 0], 1000, seed=20261205)
    counts, outside = histograms(snaps, m.bounds, n_marginal=3)
    L = Likelihood(m, times, counts, outside=outside, n_marginal=3, kry_tol=1e-8)
    rng = np.random.default_rng(7)
    sets = np.stack([m.coefs(0) * 10.0 ** rng.uniform(-0.5, 0.5, m.nr) for _ in range(n_sets)])
    L.gradient(sets[0])  # warm-up (kernel compilation, graphs)
    torch.cuda.synchronize()
    idx = [i * n_sets // sample for i in range(sample)]
    single, ref = 0.0, []
    for i in idx:
        t0 = time.perf_counter()
        ref.append(L.gradient(sets[i]))
        torch.cuda.synchronize()
        single += time.perf_counter() - t0
    t0 = time.perf_counter()
    ll_b, g_b = L.gradient_batched(sets, workers=workers)
    torch.cuda.synchronize()
    batched = time.perf_counter() - t0
    diff = max(float(np.abs(g_b[i] - g).max() / max(np.abs(g).max(), 1e-300)) for i, (_, g) in zip(idx, ref))
    dll = max(abs(ll_b[i] - l) / abs(l) for i, (l, _) in zip(idx, ref))
    t0 = time.perf_counter()
    L.evaluate(sets[0])
    torch.cuda.synchronize()
    ev = time.perf_counter() - t0
    return {"metric": "grad logL grads/s", "workload": "gene_expression 131,072 states, 12 rates, 8 times in [1, 60], "
            f"1,000 SSA cells per time, marginalised over gene states, {n_sets} parameter sets",
            "value": round(n_sets / batched, 3), "s_per_batch": round(batched, 3), "workers": workers,
            "single_grads_per_s": round(len(idx) / single, 3),
            "single_sample": f"{len(idx)} of the same sets one at a time (cufsp_likelihood_grad)",
            "rel_diff_vs_single": {
                "logL": dll, "grad": diff,
                "note": "the workers' passes run on a quarter of the SMs (37 CTAs against 148) and round "
                        "differently; where that flips an accept/reject decision of the Krylov step control, "
                        "data cells whose probability is below the absolute kry_tol 1e-8 cross the 1e-44 floor "
                        "(up to ~70 in log L each). With equal CTA counts both paths do the same arithmetic "
                        "(test_c5_batched_gradients_equal_single_on_full_gene_box)."},
            "s_per_loglik": round(ev, 3)}


def run_ours(args):
    import torch
    import torch.distributed as dist
    from cuda_fsp_b200 import FSPMat, MatrixFormat, models

    world, rank, local = dist_setup()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=300))
    dev = torch.device("cuda", local if world > 1 else 0)
    torch.cuda.set_device(dev)

    m = models.mass_action_3()
    n = m.n_states
    A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
    c = m.coefs(0)
    n_sets = args.sets  # default 4 rotating (x, y) pairs = 1.07 GB > 126 MB L2 between timed iterations
    g = torch.Generator(device=dev).manual_seed(1234 + rank)
    xs = [torch.rand(n, dtype=torch.float64, device=dev, generator=g) for _ in range(n_sets)]
    ys = [torch.zeros(n, dtype=torch.float64, device=dev) for _ in range(n_sets)]
    stream = torch.cuda.current_stream(dev)

    def step(i):
        A.apply(xs[i % n_sets], ys[i % n_sets], coefs=c, beta=1.0, stream=stream.cuda_stream)

    for i in range(max(3, args.warmup)):
        step(i)
    # Warm-up beyond the W steps: ~30 ms of launches, so the SM clock has left its idle state.  The
    # timed region is then a burst of K launches (the regime of the HBM copy peak it is compared
    # with); the same launches over ~1 s, under the power cap, are reported beside it as `sustained`.
    clocks = ClockSampler(nvml_index(dev))
    clocks.start()
    t_w = time.perf_counter()
    i = 0
    while not args.no_extras and time.perf_counter() - t_w < 0.03:
        for _ in range(20):
            step(i)
            i += 1
        torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    clocks.mark()
    ev0.record(stream)
    for i in range(args.steps):
        step(i)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    clocks.mark()
    ms = ev0.elapsed_time(ev1) / args.steps
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = t.item()
        dist.barrier()
    clk = clocks.stop()
    sustained = None
    if not args.no_extras:  # the same launches over ~1 s (power-capped regime), reported beside
        k_s = max(args.steps, int(1.0 / max(ms * 1e-3, 1e-6)))
        cs = ClockSampler(nvml_index(dev))
        cs.start()
        torch.cuda.synchronize(dev)
        ev0.record(stream)
        for i in range(k_s):
            step(i)
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        ms_s = ev0.elapsed_time(ev1) / k_s
        if world > 1:
            t = torch.tensor([ms_s], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms_s = t.item()
        sustained = {"value": round(BYTES_PER_STATE * n / (ms_s * 1e-3) / 1e9 * world, 3), "unit": "GB/s",
                     "ms_per_step": round(ms_s, 5), "steps": k_s, "clocks": cs.stop()}
    kernel_gbs = BYTES_PER_STATE * n / (ms * 1e-3) / 1e9
    value = kernel_gbs * world
    if args.no_extras:  # profiling runs: the timed generator action only
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": round(value, 3), "unit": "GB/s", "ms_per_step": round(ms, 5),
                              "steps": args.steps, "sets": n_sets, "profiling_run": True, "kernel": A.describe()}),
                  flush=True)
        if world > 1:
            dist.destroy_process_group()
        return

    # e2e through the host-buffer entry point (pinned host memory, copies inside the timed region)
    xh = torch.empty(n, dtype=torch.float64).pin_memory()
    yh = torch.empty(n, dtype=torch.float64).pin_memory()
    xh.copy_(xs[0].cpu())
    yh.zero_()
    e2e_steps = max(2, min(args.steps, 10))
    A.action_host(0.0, xh, yh)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        A.action_host(0.0, xh, yh)
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    if world > 1:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = t.item()
    e2e_gbs = BYTES_PER_STATE * n / e2e_s / 1e9 * world

    secondary = None
    if world > 1:  # the batched form shards over the ranks; every rank takes part
        sharded = batched_sharded_secondary(world, rank, dev)
        if rank == 0:
            secondary = [expmv_secondary(), sharded]
    elif rank == 0:
        secondary = expmv_secondary()
        secondary["cpu_oracle_ms_per_solve"] = round(cpu_expmv_ms(), 1)
        secondary = [secondary, sparse_secondary(), kron_general_secondary(), bdf_secondary(), expmv_large_secondary(), batched_secondary(),
                     gradient_secondary()]
    cpu = cpu_oracle_gbs(max(3, min(args.steps, 20)), 3) if (rank == 0 and world == 1) else None
    peak, peak_kind = measured_peak_hbm()
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 5), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(world),
            "e2e": {"value": round(e2e_gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": 16 * n, "d2h_bytes_per_step": 8 * n,
                    "entry_point": "cufsp_mat_action_host", "ms_per_step": round(e2e_s * 1e3, 3)},
            "roofline": {"bound": "hbm", "achieved": round(kernel_gbs, 3), "peak": peak, "unit": "GB/s",
                         "frac": round(kernel_gbs / peak, 4), "traffic": profile_traffic(),
                         "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured" else "fallback 6.65 TB/s",
                         "kernel": A.describe()},
            "cpu_baseline": ({k: (round(v, 3) if isinstance(v, float) else v) for k, v in cpu.items() if k != "ms_per_step"}
                             if cpu else None),
            "clocks": clk,
            "sustained": sustained,
            "gpu_launches": args.steps,
            "secondary": secondary,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_leg(args):
    """One leg alone, for profiling its kernels under ncu (small steps, one JSON line, no extras):
      sparse  the CSR/HYB generator action y += A x on mass_action_3 (--box, default 255^3)
      kgen    the KRONECKER action of the 5-species gene network (--box, default 1,1,1,127,8191): the
              slab kernel
      kslab3  forward and transposed KRONECKER actions of the 3-species network with two reactions
              moving 2 molecules (--box, default 255^3): the tiled slab kernels
      krylov  Krylov steps exp(tA)p0 on mass_action_3 (--box; above 2^20 states the launch sequence
              of plane-kernel matvecs and the k_mdot / k_mupd / k_comb vector kernels)
      adjoint one log-likelihood gradient on the gene model (--box, default 1,1,1,127,127)
      gradbatch  gradients of --sets parameter sets with --workers concurrent host workers
      bdf     the BDF solve of the time-varying gene model to t = 6 (--box)
      states  state enumeration cufsp_get_states (--box, default 1023,1023,3)
      iopsweep  exp(tA)p0 on mass_action_3 (--box, default 255^3) to t = 0.2 for Krylov dimensions m and
              incomplete orthogonalisation depths q, each timed to completion, with its 1-norm distance
              to an m = 60, tol 1e-11 full-orthogonalisation solution"""
    import torch
    from cuda_fsp_b200 import (BDFIntegrator, FSPMat, KryExpvFSP, Likelihood, MatrixFormat, get_states, models)
    box = [int(v) for v in args.box.split(",")] if args.box else None
    torch.cuda.set_device(0)
    out = {"leg": args.leg, "profiling_run": True}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if args.leg == "sparse":
        m = models.mass_action_3(bounds=box) if box else models.mass_action_3()
        A = FSPMat.from_model(m, MatrixFormat.HYB)
        g = torch.Generator(device="cuda").manual_seed(5)
        xs = [torch.rand(m.n_states, dtype=torch.float64, device="cuda", generator=g) for _ in range(2)]
        ys = [torch.zeros(m.n_states, dtype=torch.float64, device="cuda") for _ in range(2)]
        c = m.coefs(0)
        for i in range(max(3, args.warmup)):
            A.apply(xs[i % 2], ys[i % 2], coefs=c, beta=1.0)
        torch.cuda.synchronize()
        ev0.record()
        for i in range(args.steps):
            A.apply(xs[i % 2], ys[i % 2], coefs=c, beta=1.0)
        ev1.record()
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / args.steps
        bps = 24 + 8 * m.nr
        out.update({"n_states": m.n_states, "us_per_action": round(ms * 1e3, 2), "bytes_per_state": bps,
                    "gbs": round(bps * m.n_states / (ms * 1e-3) / 1e9, 1), "kernel": A.describe()})
    elif args.leg == "kgen":
        m = models.gene_expression(tuple(box) if box else (1, 1, 1, 127, 8191), time_varying=False)
        A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
        g = torch.Generator(device="cuda").manual_seed(6)
        xs = [torch.rand(m.n_states, dtype=torch.float64, device="cuda", generator=g) for _ in range(2)]
        ys = [torch.zeros(m.n_states, dtype=torch.float64, device="cuda") for _ in range(2)]
        c = m.coefs(0)
        for i in range(max(3, args.warmup)):
            A.apply(xs[i % 2], ys[i % 2], coefs=c, beta=1.0)
        torch.cuda.synchronize()
        ev0.record()
        for i in range(args.steps):
            A.apply(xs[i % 2], ys[i % 2], coefs=c, beta=1.0)
        ev1.record()
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / args.steps
        out.update({"n_states": m.n_states, "us_per_action": round(ms * 1e3, 2),
                    "gbs": round(BYTES_PER_STATE * m.n_states / (ms * 1e-3) / 1e9, 1), "kernel": A.describe()})
    elif args.leg == "kslab3":
        # the 3-species network with reactions 0 and 6 moving 2 molecules (outside the plane kernel's
        # shape): forward y += A x and transposed y = A^T x through the slab kernels
        m = models.mass_action_3(bounds=box) if box else models.mass_action_3()
        m.nu[0] = (2, 0, 0)
        m.nu[6] = (0, -2, 1)
        A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
        g = torch.Generator(device="cuda").manual_seed(7)
        xs = [torch.rand(m.n_states, dtype=torch.float64, device="cuda", generator=g) for _ in range(2)]
        ys = [torch.zeros(m.n_states, dtype=torch.float64, device="cuda") for _ in range(2)]
        c = m.coefs(0)
        res = {}
        for form in ("forward", "transposed"):
            def act(i):
                if form == "forward":
                    A.apply(xs[i % 2], ys[i % 2], coefs=c, beta=1.0)
                else:
                    A.apply_transpose(xs[i % 2], ys[i % 2], coefs=c)
            for i in range(max(3, args.warmup)):
                act(i)
            torch.cuda.synchronize()
            ev0.record()
            for i in range(args.steps):
                act(i)
            ev1.record()
            torch.cuda.synchronize()
            ms = ev0.elapsed_time(ev1) / args.steps
            bps = BYTES_PER_STATE if form == "forward" else 16
            res[form] = {"us_per_action": round(ms * 1e3, 2), "bytes_per_state": bps,
                         "gbs": round(bps * m.n_states / (ms * 1e-3) / 1e9, 1)}
        out.update({"n_states": m.n_states, **res, "kernel": A.describe()})
    elif args.leg == "krylov":
        m = models.mass_action_3(bounds=box) if box else models.mass_action_3()
        A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
        v = torch.as_tensor(m.p0(), device="cuda")
        E = KryExpvFSP(20.0, A, v, m=args.krylov_m, tol=1e-8, coefs=m.coefs(0), iop=args.iop > 0, q_iop=max(1, args.iop))
        for _ in range(max(1, args.warmup)):
            E.step()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            E.step()
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / args.steps
        out.update({"n_states": m.n_states, "ms_per_krylov_step": round(dt * 1e3, 3), "t_now": E.stats["t_now"],
                    "m": args.krylov_m, "iop_q": args.iop})
    elif args.leg == "adjoint":
        m = models.gene_expression(tuple(box) if box else (1, 1, 1, 127, 127), time_varying=False)
        times = np.geomspace(1.0, 60.0, 8)
        rng = np.random.default_rng(1)
        counts = rng.integers(0, 3, size=(8, m.n_states // 8)).astype(float)
        L = Likelihood(m, times, counts, n_marginal=3, kry_tol=1e-8)
        L.gradient()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            L.gradient()
        torch.cuda.synchronize()
        out.update({"n_states": m.n_states, "s_per_gradient": round((time.perf_counter() - t0) / args.steps, 4)})
    elif args.leg == "gradbatch":
        m = models.gene_expression(tuple(box) if box else (1, 1, 1, 127, 127), time_varying=False)
        times = np.geomspace(1.0, 60.0, 8)
        rng = np.random.default_rng(1)
        counts = rng.integers(0, 3, size=(8, m.n_states // 8)).astype(float)
        L = Likelihood(m, times, counts, n_marginal=3, kry_tol=1e-8)
        sets = np.stack([m.coefs(0) * 10.0 ** rng.uniform(-0.5, 0.5, m.nr) for _ in range(args.sets)])
        L.gradient(sets[0])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L.gradient_batched(sets, workers=args.workers)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        out.update({"n_states": m.n_states, "sets": args.sets, "workers": args.workers,
                    "grads_per_s": round(args.sets / dt, 3)})
    elif args.leg == "bdf":
        m = models.gene_expression(tuple(box) if box else (1, 1, 1, 127, 127), time_varying=True)
        A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
        p = torch.as_tensor(m.p0(), device="cuda")
        B = BDFIntegrator(A, rtol=1e-8, atol=1e-14)
        t0 = time.perf_counter()
        B.init(0.0, p)
        B.advance(6.0, p)
        torch.cuda.synchronize()
        out.update({"n_states": m.n_states, "s_to_t6": round(time.perf_counter() - t0, 4), "steps": B.stats["n_steps"]})
    elif args.leg == "iopsweep":
        m = models.mass_action_3(bounds=box) if box else models.mass_action_3()
        A = FSPMat.from_model(m, MatrixFormat.KRONECKER)
        p0 = torch.as_tensor(m.p0(), device="cuda")
        T = 0.2

        def solve(tol, **kw):
            v = p0.clone()
            KryExpvFSP(T, A, v, tol=tol, coefs=m.coefs(0), **kw).step()  # warm-up: tables, first launches
            v.copy_(p0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            E = KryExpvFSP(T, A, v, tol=tol, coefs=m.coefs(0), **kw)
            E.max_nstep = 1 << 20
            st = E.solve()
            torch.cuda.synchronize()
            return v, time.perf_counter() - t0, st

        ref, dt_ref, st_ref = solve(1e-11, m=60)
        rows = []
        for mk, q in ((30, 0), (45, 0), (60, 0), (30, 2), (45, 2), (60, 2), (60, 3), (60, 4)):
            kw = dict(m=mk, iop=q > 0, q_iop=max(q, 1))
            v, dt, st = solve(1e-8, **kw)
            rows.append({"m": mk, "q": q or "full", "s": round(dt, 3), "steps": st["n_steps"],
                         "rejected": st["n_reject"], "matvecs": st["n_matvec"],
                         "err_1norm": float((v - ref).abs().sum().item())})
        out.update({"n_states": m.n_states, "t": T, "tol": 1e-8,
                    "reference": {"m": 60, "tol": 1e-11, "s": round(dt_ref, 3), "steps": st_ref["n_steps"]},
                    "configs": rows})
    elif args.leg == "states":
        b = box or [1023, 1023, 3]
        st = get_states(b)
        torch.cuda.synchronize()
        ev0.record()
        for _ in range(args.steps):
            st = get_states(b)
        ev1.record()
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / args.steps
        out.update({"n_states": int(st.shape[0]), "ms_per_call": round(ms, 4),
                    "gbs_written": round(st.numel() * 4 / (ms * 1e-3) / 1e9, 1)})
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--sets", type=int, default=4, help="rotating (x, y) input pairs; parameter sets of the gradbatch leg")
    ap.add_argument("--no-extras", action="store_true",
                    help="time the generator action only (no e2e, expmv or CPU legs); for profiling runs")
    ap.add_argument("--leg", choices=["sparse", "kgen", "kslab3", "krylov", "adjoint", "gradbatch", "bdf", "states",
                                      "iopsweep"],
                    default=None,
                    help="run one leg alone (profiling runs; see run_leg)")
    ap.add_argument("--box", default=None, help="box bounds of the leg, comma separated")
    ap.add_argument("--workers", type=int, default=4, help="host workers of the gradbatch leg")
    ap.add_argument("--krylov-m", type=int, default=30, help="Krylov dimension of the krylov leg")
    ap.add_argument("--iop", type=int, default=0, help="incomplete orthogonalisation depth q of the krylov leg (0: full)")
    args = ap.parse_args()
    if args.leg:
        run_leg(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
