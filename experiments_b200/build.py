"""Build libb3gpu.so (CUDA sm_100a + host C++) in-tree.

Usage: python -m experiments_b200.build [--force]
The shared library lands in experiments_b200/lib/libb3gpu.so and is loaded by
experiments_b200.b3 through ctypes.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libb3gpu.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                  "-I", os.path.join(ROOT, "include"), "-I", CSRC]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
            "-I", os.path.join(CUDA, "include")]


def _sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp"))
    return cu, cpp


def _headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(ROOT, "include", "b3gpu.h"))
    return max(os.path.getmtime(h) for h in hs)


def _compile(src, force):
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
            and os.path.getmtime(obj) >= _headers_mtime()):
        return obj, None
    if src.endswith(".cu"):
        cmd = [NVCC] + NVFLAGS + ["-c", src, "-o", obj]
    else:
        cmd = ["g++"] + CXXFLAGS + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, "FAILED: " + " ".join(cmd) + "\n" + r.stdout + r.stderr
    return obj, (r.stderr.strip() or None)


def build(force=False, verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    cu, cpp = _sources()
    srcs = [os.path.join(CSRC, f) for f in cu + cpp]
    objs = []
    errors = []
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        for obj, msg in ex.map(lambda s: _compile(s, force), srcs):
            objs.append(obj)
            if msg and msg.startswith("FAILED"):
                errors.append(msg)
            elif msg and verbose:
                print(msg)
    if errors:
        raise RuntimeError("\n".join(errors))
    if (force or not os.path.exists(LIB) or
            max(os.path.getmtime(o) for o in objs) > os.path.getmtime(LIB)):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + [
            "-lcudart", "-Xlinker", "-rpath=" + os.path.join(CUDA, "lib64")]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
