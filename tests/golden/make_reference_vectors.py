"""Writes tests/golden/reference_host.npz: outputs of the reference's own compiled host code, run
through oracle/_ref/libref.so (built by `make -C oracle ref` from the reference sources), for the
oracle tests to check against without the shim:
  * rect_fsp_num_states / indx2state / state2indx (src/cme_util.cu:5-22,55-62) on five boxes, at
    the first and last index and up to 500 seeded random ones;
  * fspmat_sdkron_fill_host_data (src/fspmat_kron_kernels.cu:170-190) factor tables and offsets for
    three networks.
Run from the repository root: python tests/golden/make_reference_vectors.py
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from cuda_fsp_b200 import models  # noqa: E402

BOUNDS = [[3, 4, 2], [0, 5], [7], [1, 1, 1, 127, 127], [30, 2, 0, 4]]


def golden_models():
    return {"toggle_31": models.toggle((31, 31)), "gene_1_1_1_7_9": models.gene_expression((1, 1, 1, 7, 9)),
            "mass_action_3_6": models.mass_action_3(6)}


def main():
    R = oracle.ref()
    if R is None:
        raise SystemExit(f"{oracle.REF_SO} is missing: build it with `make -C oracle ref`")
    out = {}
    for k, bounds in enumerate(BOUNDS):
        b = np.asarray(bounds, np.int32)
        n = int(R.ref_num_states(len(b), b.ctypes.data))
        rng = np.random.default_rng(1)
        idx = np.unique(np.concatenate([[0, n - 1], rng.integers(0, n, size=min(n, 500))])).astype(np.int64)
        states = np.empty((len(idx), len(b)), np.int32)
        back = np.empty(len(idx), np.int64)
        for j, i in enumerate(idx):
            s = np.empty(len(b), np.int32)
            R.ref_indx2state(int(i), s.ctypes.data, len(b), b.ctypes.data)
            states[j] = s
            back[j] = R.ref_state2indx(s.ctypes.data, len(b), b.ctypes.data)
        out[f"box{k}_bounds"] = b
        out[f"box{k}_n"] = np.int64(n)
        out[f"box{k}_idx"] = idx
        out[f"box{k}_states"] = states
        out[f"box{k}_state2indx"] = back
    for name, m in golden_models().items():
        b = np.asarray(m.bounds, np.int32)
        sv, sc, sr = m.stoich_csr()
        vals = np.empty_like(m.tables)
        offs = np.empty((m.nr, m.ns), np.int32)
        tab = np.ascontiguousarray(m.tables)
        R.ref_sdkron_fill(m.ns, b.ctypes.data, m.nr, sv.ctypes.data, sc.ctypes.data, sr.ctypes.data,
                          tab.ctypes.data, vals.ctypes.data, offs.ctypes.data)
        out[f"{name}_vals"] = vals
        out[f"{name}_offsets"] = offs
    path = Path(__file__).with_name("reference_host.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({path.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
