"""Partitioning of batched solves over ranks, and the sharded solve's gather, on CPU ranks (gloo,
world size 2); the per-rank solver is replaced by the oracle so no GPU is needed."""
import os

import numpy as np
import pytest

from cuda_fsp_b200.batch import partition_instances


def test_partition_balances_states_and_covers_every_instance():
    rng = np.random.default_rng(0)
    sizes = rng.integers(1000, 500000, 256)
    for world in (1, 2, 3, 8):
        parts = partition_instances(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(256))
        loads = [int(np.sum(sizes[p])) for p in parts]
        assert max(loads) - min(loads) <= int(sizes.max())  # greedy bound
        assert parts == partition_instances(sizes, world)  # deterministic


def _oracle_solver(sub, t):
    import oracle
    out = []
    for mm in sub:
        csr = oracle.assemble_model(mm)
        w, st, rc = oracle.expv(csr, mm.coefs(0), t, mm.p0(), m=20, tol=1e-8)
        out.append((w, {"steps": st["n_steps"], "status": rc}))
    return out


def _rank_main(rank, world, port, result_dir):
    import torch.distributed as dist
    from cuda_fsp_b200 import models
    from cuda_fsp_b200.batch import solve_sharded
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = models.gene_batch(6, seed=11, lo=3, hi=9)
        res = solve_sharded(ms, 2.0, rank, world, solver=_oracle_solver)
        np.save(os.path.join(result_dir, f"r{rank}.npy"), np.array([[r["mass"], r["steps"], r["status"]] for r in res]))
    finally:
        dist.destroy_process_group()


def test_sharded_solve_gathers_every_instance_on_every_rank(tmp_path):
    import socket

    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    r0, r1 = np.load(tmp_path / "r0.npy"), np.load(tmp_path / "r1.npy")
    assert r0.shape == (6, 3) and np.array_equal(r0, r1)
    assert np.all(r0[:, 2] == 0) and np.all(r0[:, 1] >= 1)
    assert np.all((r0[:, 0] > 0.5) & (r0[:, 0] <= 1.0 + 1e-12))


def _rank_vectors(rank, world, port, result_dir):
    import torch.distributed as dist
    from cuda_fsp_b200 import models
    from cuda_fsp_b200.batch import gradient_sharded, solve_sharded
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = models.gene_batch(5, seed=12, lo=3, hi=9)
        vecs = solve_sharded(ms, 2.0, rank, world, solver=_oracle_solver, gather="vectors")
        np.save(os.path.join(result_dir, f"v{rank}.npy"), np.concatenate(vecs))
        marg = solve_sharded(ms, 2.0, rank, world, solver=_oracle_solver, gather="reduce",
                             reduce=lambda mm, v, st: v.reshape(-1, 8).sum(axis=1).tolist())
        np.save(os.path.join(result_dir, f"m{rank}.npy"), np.concatenate([np.asarray(x) for x in marg]))

        def fake_grad(sets):  # a deterministic stand-in for the GPU gradient: (sum c, c * 2)
            return sets.sum(axis=1), 2.0 * sets
        sets = np.arange(7 * 3, dtype=np.float64).reshape(7, 3)
        ll, g = gradient_sharded(None, sets, rank, world, grad_fn=fake_grad)
        np.save(os.path.join(result_dir, f"g{rank}.npy"), np.concatenate([ll[:, None], g], axis=1))
    finally:
        dist.destroy_process_group()


def test_sharded_vectors_reductions_and_gradients(tmp_path):
    """gather='vectors' returns every instance's solution on every rank (equal to a single-rank
    solve), gather='reduce' a caller-chosen reduction, and gradient_sharded the rows of all
    parameter sets in their original order."""
    import socket

    import torch.multiprocessing as mp
    from cuda_fsp_b200 import models
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    mp.start_processes(_rank_vectors, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    ms = models.gene_batch(5, seed=12, lo=3, hi=9)
    ref = np.concatenate([w for w, _ in _oracle_solver(ms, 2.0)])
    for r in (0, 1):
        assert np.array_equal(np.load(tmp_path / f"v{r}.npy"), ref)
        assert np.allclose(np.load(tmp_path / f"m{r}.npy"),
                           np.concatenate([w.reshape(-1, 8).sum(axis=1) for w, _ in _oracle_solver(ms, 2.0)]))
        sets = np.arange(21, dtype=np.float64).reshape(7, 3)
        got = np.load(tmp_path / f"g{r}.npy")
        assert np.array_equal(got[:, 0], sets.sum(axis=1)) and np.array_equal(got[:, 1:], 2.0 * sets)
