"""Build the in-tree CUDA library libxbg_b200.so (sm_100a only).

    python -m xbeach_gpu_b200.build

Each .cu file of csrc/ compiles in parallel to an object under _build/ (kept
only if its source or a header changed), then nvcc links the shared library
next to this file.  Flags: -gencode arch=compute_100a,code=sm_100a, -O3,
-lineinfo, -prec-div=false -prec-sqrt=false.  The FP32 path is held to the
reference within 1e-5 per step, not bit for bit, so it uses multiply-add
contraction and the full-range 2-ulp float division and square root (no
IEEE slow path, whose branchy subroutine dry cells' zeros kept calling);
double arithmetic is unaffected and the FP64 build agrees with the FP64
oracle to rounding.
"""
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libxbg_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-prec-div=false", "-prec-sqrt=false", "-Xcompiler", "-fPIC",
         "-I", INCLUDE]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))


# per-file extra flags: the sediment pass's float transcendentals (pow, exp,
# log10, sin, cos) in their hardware forms; its FP32 results stay within the
# per-phase bar and the FP64 build is unaffected
FILE_FLAGS = {"sed.cu": ["-use_fast_math"]}


def _compile(src, force=False):
    obj = os.path.join(BUILD, os.path.splitext(os.path.basename(src))[0] + ".o")
    newest = max([os.path.getmtime(src), os.path.getmtime(__file__)] + [os.path.getmtime(h) for h in _headers()])
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj
    cmd = [NVCC] + ARCH + FLAGS + FILE_FLAGS.get(os.path.basename(src), []) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force=False, verbose=True):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
