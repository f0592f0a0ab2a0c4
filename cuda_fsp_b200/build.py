"""In-tree build of the cufsp CUDA library for sm_100a (B200).

Products (all git-ignored, all shipped with the source tree):
  cuda_fsp_b200/lib/libcufsp.so         C ABI shared library (static cudart inside)
  cuda_fsp_b200/lib/libcufsp_static.a   relocatable-device-code archive for C++ programs that pass
                                        their own __device__ propensity (PropFun) and link with -rdc
  tests/support/libcufsp_testmodels.so  the library device-linked with the test propensities
  tests/cpp/test_dropin                 C++ drop-in test program (include/cufsp.hpp)

Usage: python -m cuda_fsp_b200.build [--force]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "cuda_fsp_b200"
CSRC = PKG / "csrc"
LIB = PKG / "lib"
OBJ = PKG / "_build"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-rdc=true", "-Xcompiler", "-fPIC,-O2",
                     "-I" + str(ROOT / "include"), "--expt-relaxed-constexpr", "--extended-lambda"]
# The small dense kernels of the host Pade exponential vectorise at -O3 only.
HOST_EXTRA = {"cufsp_expm.cpp": ["-Xcompiler", "-O3"]}
SOURCES = ["cufsp_common.cu", "cufsp_rtc.cu", "cufsp_kron.cu", "cufsp_kron_plane.cu", "cufsp_kron_march.cu", "cufsp_sparse.cu", "cufsp_mat.cu",
           "cufsp_krylov.cu", "cufsp_expm.cpp", "cufsp_noalloc.cu", "cufsp_stats.cu", "cufsp_solver.cu",
           "cufsp_vec.cu", "cufsp_bdf.cu", "cufsp_batch.cu", "cufsp_adjoint.cu", "cufsp_adaptive.cu",
           "cufsp_arnoldi.cu"]
HEADERS = ["cufsp_internal.h", "cufsp_reduce.cuh", "cufsp_march.h", "cufsp_vec.h", "cufsp_plane.cuh", "cufsp_batch.cuh",
           "cufsp_sparse_rtc.cuh", "cufsp_kron_rtc.cuh"]
# Kernel sources compiled at run time by NVRTC are embedded in the library as string literals.
RTC_SOURCES = {"cufsp_plane.cuh": "cufsp_plane_src.inc", "cufsp_batch.cuh": "cufsp_batch_src.inc",
               "cufsp_sparse_rtc.cuh": "cufsp_sparse_src.inc", "cufsp_kron_rtc.cuh": "cufsp_kron_rtc_src.inc"}
LINK_LIBS = ["-L/usr/local/cuda/lib64", "-lnvrtc", "-Xlinker", "-rpath,/usr/local/cuda/lib64"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[-1]}")


def _embed_rtc_sources(force: bool) -> None:
    """Write each NVRTC kernel source as a raw string literal into the build folder."""
    for src, inc in RTC_SOURCES.items():
        text = (CSRC / src).read_text()
        if ")CUFSPSRC" in text:
            raise RuntimeError(f"{src} contains the raw-string delimiter")
        out = OBJ / inc
        body = 'R"CUFSPSRC(' + text + ')CUFSPSRC"\n'
        if force or not out.exists() or out.read_text() != body:
            out.write_text(body)


def _compile(src: Path, obj: Path, extra: list[str], force: bool) -> Path:
    deps = [src] + [CSRC / h for h in HEADERS] + [ROOT / "include" / "cufsp.h", ROOT / "include" / "cufsp.hpp"]
    deps += [OBJ / inc for inc in RTC_SOURCES.values()]
    if force or _stale(obj, deps):
        obj.parent.mkdir(parents=True, exist_ok=True)
        _run([nvcc()] + NVCC_FLAGS + ["-I" + str(OBJ)] + extra + ["-c", str(src), "-o", str(obj)])
    return obj


def build(force: bool = False, verbose: bool = False) -> dict[str, Path]:
    LIB.mkdir(parents=True, exist_ok=True)
    OBJ.mkdir(parents=True, exist_ok=True)
    _embed_rtc_sources(force)
    srcs = [CSRC / s for s in SOURCES]
    support = ROOT / "tests" / "support" / "test_models.cu"
    cpp_test = ROOT / "tests" / "cpp" / "test_dropin.cu"
    jobs = [(s, OBJ / (s.name + ".o")) for s in srcs]
    if support.exists():
        jobs.append((support, OBJ / "test_models.cu.o"))
    if cpp_test.exists():
        jobs.append((cpp_test, OBJ / "test_dropin.cu.o"))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda j: _compile(j[0], j[1], HOST_EXTRA.get(j[0].name, []), force), jobs))
    lib_objs = [str(o) for o in objs[: len(srcs)]]
    out = {}
    so = LIB / "libcufsp.so"
    if force or _stale(so, [Path(o) for o in lib_objs]):
        _run([nvcc()] + ARCH + ["-shared", "-rdc=true", "-Xcompiler", "-fPIC"] + lib_objs + LINK_LIBS + ["-o", str(so)])
    out["libcufsp"] = so
    ar = LIB / "libcufsp_static.a"
    if force or _stale(ar, [Path(o) for o in lib_objs]):
        _run([nvcc()] + ARCH + ["-lib", "-rdc=true"] + lib_objs + ["-o", str(ar)])
    out["libcufsp_static"] = ar
    if support.exists():
        tso = ROOT / "tests" / "support" / "libcufsp_testmodels.so"
        tobj = str(OBJ / "test_models.cu.o")
        if force or _stale(tso, [Path(o) for o in lib_objs] + [Path(tobj)]):
            _run([nvcc()] + ARCH + ["-shared", "-rdc=true", "-Xcompiler", "-fPIC"] + lib_objs + [tobj] + LINK_LIBS
                 + ["-o", str(tso)])
        out["testmodels"] = tso
    if cpp_test.exists():
        exe = ROOT / "tests" / "cpp" / "test_dropin"
        cobj = str(OBJ / "test_dropin.cu.o")
        if force or _stale(exe, [Path(o) for o in lib_objs] + [Path(cobj)]):
            _run([nvcc()] + ARCH + ["-rdc=true", cobj, str(ar)] + LINK_LIBS + ["-o", str(exe)])
        out["test_dropin"] = exe
    if verbose:
        for k, v in out.items():
            print(f"{k}: {v}")
    return out


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
