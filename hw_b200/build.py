"""Builds libhw_b200.so (the CUDA kernels + C ABI) in-tree for sm_100a.

    python -m hw_b200.build          # incremental
    python -m hw_b200.build --clean

Numerics flags: -fmad=false keeps every float multiply and add separately
rounded (the reference host path has no fused multiply-adds), so results are
bit-comparable with the CPU oracle; division and square root stay IEEE
(no --use_fast_math).
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libhw_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOST_CXX = "/usr/bin/g++"

SOURCES = ["baseliner.cu", "stats_hist.cu", "dme.cu", "labeler.cu", "pulses.cu", "gen.cu", "mlp.cu", "capi.cu", "fused.cu", "hfmetrics.cu", "repack.cu", "baz.cu", "prehq.cu", "compact.cu"]
HEADERS = ["hw_device.cuh", "hw_math.h", "hw_params.h", "metric_blocks.cuh", "../../include/hw_b200.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "-ccbin", HOST_CXX,
    "--expt-relaxed-constexpr",
]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, verbose=False, extra=()):
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    deps = [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in HEADERS] + [__file__]
    if not _stale(obj, deps):
        return obj, None
    cmd = [NVCC] + NVCC_FLAGS + list(extra) + ["-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, (r.stdout + r.stderr) if verbose else None


def build(verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose or ptxas_info, extra), SOURCES))
    objs = [r[0] for r in results]
    for src, (_, log) in zip(SOURCES, results):
        if log:
            print(f"--- {src}\n{log}")
    if _stale(LIB, objs):
        cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-ccbin", HOST_CXX,
               "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


def clean():
    shutil.rmtree(BUILD, ignore_errors=True)
    if os.path.exists(LIB):
        os.remove(LIB)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v resource usage")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    if a.clean:
        clean()
    print(build(verbose=a.verbose, ptxas_info=a.ptxas))
    sys.exit(0)
