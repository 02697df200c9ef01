"""Build libnekob200.so in-tree for sm_100a.

Every CUDA translation unit is compiled with
``nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` and linked
into ``neko_b200/libnekob200.so`` next to this file, so the shared library
travels with the source tree.  Objects go to ``neko_b200/_build/``.
Rebuilds only what changed (source or header newer than its object).
"""
import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libnekob200.so")
BUILD = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
NVFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                  "--expt-relaxed-constexpr"]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-I/usr/local/cuda/include"]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu"))) + \
        sorted(glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(HERE, "..", "include", "*.h"))


def _compile(src):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    newest_dep = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in _headers()])
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep:
        return obj, False
    if src.endswith(".cu"):
        cmd = [NVCC] + NVFLAGS + ["-c", src, "-o", obj]
    else:
        cmd = ["g++"] + CXXFLAGS + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, True


def build(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = _sources()
    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(_compile, srcs))
    objs = [o for o, _ in results]
    changed = any(c for _, c in results) or not os.path.exists(OUT) or \
        any(os.path.getmtime(o) > os.path.getmtime(OUT) for o in objs)
    if changed:
        cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose:
            print(f"built {OUT}")
    return OUT


if __name__ == "__main__":
    build(verbose=True)
    sys.exit(0)
