"""Build libkmm_b200.so (the C-ABI of include/kmm.h) for sm_100a with nvcc, in-tree.

    python -m polymer_dns_b200.build [--force] [--verbose]

Objects go to polymer_dns_b200/_build/ (ignored by git); the shared library lands
next to this file so it travels with the source tree.
"""
import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libkmm_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE, "--expt-relaxed-constexpr"]
# per-file flags: the Chebyshev recurrences and tau eliminations keep separate multiply / add
# rounding like the reference's operation sequence
PER_FILE = {"kmm_column.cu": ["-fmad=false"]}
SOURCES = ["kmm_ctx.cu", "kmm_column.cu", "kmm_plane.cu", "kmm_fast.cu", "kmm_fused.cu", "kmm_colblk.cu", "kmm_tracer.cu", "kmm_step.cu", "kmm_noalloc.cu", "kmm_ztma.cu", "kmm_tcdct.cu", "kmm_hoststate.cu"]
HEADERS = ["kmm_internal.cuh", "kmm_warpcol.cuh", "kmm_fft.cuh", "kmm_fused.cuh", "kmm_colblk.cuh", "kmm_async.cuh"]


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found")
    return exe


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=()):
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "kmm.h")]
    objs, cmds = [], []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            cmds.append([nvcc()] + ARCH + COMMON + PER_FILE.get(src, []) + list(extra) + ["-c", s, "-o", o])
    # the translation units compile independently: run them side by side
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        futs = []
        for cmd in cmds:
            if verbose:
                print(" ".join(cmd), flush=True)
            futs.append(ex.submit(subprocess.run, cmd))
        for cmd, f in zip(cmds, futs):
            if f.result().returncode != 0:
                raise subprocess.CalledProcessError(f.result().returncode, cmd)
    if force or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-lpthread", "-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register / shared-memory usage")
    a = ap.parse_args(argv)
    extra = ["-Xptxas", "-v"] if a.ptxas_v else []
    print(build(force=a.force or a.ptxas_v, verbose=a.verbose, extra=extra))


if __name__ == "__main__":
    sys.exit(main())
