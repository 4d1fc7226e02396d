"""Build liblzk_b200.so in-tree: every csrc/*.cu compiled for sm_100a with
nvcc, then linked into one shared library next to this file.

    python -m liblightzk_b200.build [-v] [--debug]

Object files go to _build/ at the repository root; a source is recompiled
only when it or a header under csrc/ or include/ changed.  --debug builds
liblzk_b200_debug.so instead (objects in _build_debug/): the same sources
with LZK_DEBUG_CHECKS, whose kernels check their indices and record
out-of-range ones in an error word (lzk_debug_check_word) instead of
touching memory outside their buffers.
"""
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INC = os.path.join(ROOT, "include")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "liblzk_b200.so")
BUILD_DEBUG = os.path.join(ROOT, "_build_debug")
LIB_DEBUG = os.path.join(PKG, "liblzk_b200_debug.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INC, "-I", CSRC,
                "--expt-relaxed-constexpr", "-Xptxas", "-v", "-ccbin", "/usr/bin/g++"]


def _newest_header():
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INC, "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src, verbose, outdir, extra):
    obj = os.path.join(outdir, os.path.basename(src)[:-3] + ".o")
    log = obj + ".ptxas.log"
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _newest_header()):
        return obj, None
    cmd = [NVCC] + FLAGS + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    with open(log, "w") as f:
        f.write(r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr[-6000:]}")
    if verbose:
        print(f"[build] {os.path.basename(src)}", flush=True)
    return obj, log


def build(verbose=False, jobs=None, debug=False):
    outdir, lib = (BUILD_DEBUG, LIB_DEBUG) if debug else (BUILD, LIB)
    extra = ["-DLZK_DEBUG_CHECKS"] if debug else []
    os.makedirs(outdir, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        objs = [o for o, _ in ex.map(lambda s: _compile(s, verbose, outdir, extra), srcs)]
    if os.path.exists(lib) and os.path.getmtime(lib) >= max(os.path.getmtime(o) for o in objs):
        return lib
    cmd = [NVCC] + ARCH + ["-shared", "-cudart", "shared", "-o", lib] + objs + ["-ccbin", "/usr/bin/g++"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
    if verbose:
        print(f"[build] linked {lib}", flush=True)
    return lib


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, debug="--debug" in sys.argv)
