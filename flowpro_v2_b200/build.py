"""Build libflowgpu.so (the C-ABI library) in-tree with nvcc for sm_100a.

usage: python -m flowpro_v2_b200.build [--verbose]
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libflowgpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr",
         "-Xptxas", "-v" if os.environ.get("FP_PTXAS_VERBOSE") else "-O3"]
SOURCES = ["fp_setup.cpp", "fp_api.cu", "fp_residual.cu", "fp_linalg.cu", "fp_res_ns2e.cu", "fp_res_ns2v.cu",
           "fp_res_ns3.cu", "fp_res_sa2.cu", "fp_res_scalar2.cu", "fp_noalloc.cu", "fp_ilu.cu",
           "fp_res_adiabatic.cu", "fp_io.cpp", "fp_batch.cu"]


def _obj(src):
    return os.path.join(BUILD, os.path.splitext(src)[0] + ".o")


def _stale(src, obj):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh", ".cu", ".cpp"))]
    deps.append(os.path.join(HERE, "..", "include", "flowgpu.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d) and (d.endswith((".h", ".cuh")) or d.endswith(src)))


def _compile(src, verbose):
    obj = _obj(src)
    cmd = [NVCC] + ARCH + FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC, "-x", "cu"] + ARCH + FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}")
    return obj


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    todo = [s for s in SOURCES if force or _stale(s, _obj(s))]
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        list(ex.map(lambda s: _compile(s, verbose), todo))
    if todo or not os.path.exists(LIB):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + [_obj(s) for s in SOURCES] + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force="--force" in sys.argv)
    print(LIB)
