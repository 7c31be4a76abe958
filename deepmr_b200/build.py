"""Build the in-tree CUDA library ``deepmr_b200/lib/libdeepmr_b200.so`` for sm_100a.

Each ``csrc/*.cu`` is compiled by nvcc in parallel into ``deepmr_b200/_build``
and linked into one shared library against cuFFT (CUDA runtime linked
statically). Usage::

    python -m deepmr_b200.build [--force] [-v]
"""

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJ_DIR = os.path.join(HERE, "_build")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libdeepmr_b200.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "--expt-relaxed-constexpr",
    "-Xcompiler",
    "-fPIC,-O2",
    "-I" + INCLUDE,
    "-I" + CSRC,
]


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _deps():
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hdrs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return max((os.path.getmtime(h) for h in hdrs), default=0.0)


def _compile(src, force, verbose, extra):
    obj = os.path.join(OBJ_DIR, src[:-3] + ".o")
    path = os.path.join(CSRC, src)
    if (
        not force
        and os.path.exists(obj)
        and os.path.getmtime(obj) >= max(os.path.getmtime(path), _deps())
    ):
        return obj, False
    cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", path, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr, flush=True)
    return obj, True


def build(force=False, verbose=False, extra=()):
    """Compile every CUDA source and link the shared library; returns its path."""
    os.makedirs(OBJ_DIR, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, force, verbose, list(extra)), srcs))
    objs = [o for o, _ in results]
    rebuilt = any(r for _, r in results)
    if rebuilt or force or not os.path.exists(LIB):
        cmd = [
            NVCC,
            *ARCH,
            "-shared",
            "-o",
            LIB,
            *objs,
            "-L" + os.path.join(CUDA_HOME, "lib64"),
            "-lcufft",
            "-Xlinker",
            "-rpath=" + os.path.join(CUDA_HOME, "lib64"),
        ]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers / spills")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas_info else []
    print(build(force=a.force or a.ptxas_info, verbose=a.verbose or a.ptxas_info, extra=extra))
    sys.exit(0)
