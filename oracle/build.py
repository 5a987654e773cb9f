"""Build the oracle (test infrastructure only).

  oracle/liboracle.so      the single-threaded C++ restatement (b3_oracle.cpp)
  oracle/_ref/libb3ref.so  pieces of the reference compiled from its own
                           sources under /root/reference plus the thin shim in
                           oracle/ref_shim.cpp (built only where that tree
                           exists; the built file travels with the repository
                           snapshot, the sources do not)

Usage: python -m oracle.build [--force]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
LIB_F32 = os.path.join(HERE, "liboracle_f32.so")
LIB_DUAL = os.path.join(HERE, "liboracle_dual.so")
REF_LIB = os.path.join(HERE, "_ref", "libb3ref.so")
BULLET_LIB = os.path.join(HERE, "_ref", "libb3bullet.so")
# the reference tree; B3_REFERENCE_ROOT overrides the default location
REFERENCE = os.environ.get("B3_REFERENCE_ROOT", "/root/reference")

# Reference sources compiled for the pins (paths relative to the reference root).
REF_SOURCES = [
    "opencl/gpu_rigidbody_pipeline2/btPgsJacobiSolver.cpp",
    "opencl/gpu_rigidbody_pipeline2/satClipHullContacts.cpp",
    "opencl/gpu_rigidbody_pipeline/btConvexUtility.cpp",
    "bullet2/LinearMath/btConvexHullComputer.cpp",
    "bullet2/LinearMath/btAlignedAllocator.cpp",
    "bullet2/LinearMath/btGeometryUtil.cpp",
    "bullet2/LinearMath/btQuickprof.cpp",
]


def _stale(out, srcs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs if os.path.exists(s))


def build_oracle(force=False):
    src = os.path.join(HERE, "b3_oracle.cpp")
    dual = os.path.join(HERE, "b3_dual.h")
    for out, extra in ((LIB, []), (LIB_F32, ["-DORACLE_REAL=float"]), (LIB_DUAL, ["-DORACLE_DUAL"])):
        if force or _stale(out, [src, dual]):
            cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math"] + \
                extra + [src, "-o", out]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError("oracle build failed:\n" + r.stderr)
    return LIB


def build_ref(force=False):
    """Compile the reference pieces in place (no copies into this repo)."""
    if not os.path.isdir(REFERENCE):
        return REF_LIB if os.path.exists(REF_LIB) else None
    shims = [os.path.join(HERE, f) for f in ("ref_shim_jacobi.cpp", "ref_shim_hull.cpp", "ref_shim_clip.cpp")]
    srcs = [os.path.join(REFERENCE, s) for s in REF_SOURCES] + shims
    if not force and not _stale(REF_LIB, srcs):
        return REF_LIB
    os.makedirs(os.path.dirname(REF_LIB), exist_ok=True)
    objdir = os.path.join(HERE, "_ref", "obj")
    os.makedirs(objdir, exist_ok=True)
    inc = ["-I", os.path.join(REFERENCE, "bullet2"),
           "-I", os.path.join(REFERENCE, "opencl/gpu_rigidbody_pipeline2"),
           "-I", os.path.join(REFERENCE, "opencl/gpu_rigidbody_pipeline"),
           "-I", os.path.join(REFERENCE, "dynamics/basic_demo/Stubs"),
           "-I", os.path.join(REFERENCE, "opencl")]
    flags = ["-O2", "-fPIC", "-w", "-include", "cstdio", "-include", "cstring", "-include", "cstdlib",
             "-DDISABLE_JOINTS"]
    objs = []
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        cmd = ["g++"] + flags + inc + ["-c", s, "-o", o]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("reference build failed: " + " ".join(cmd) + "\n" + r.stderr[-4000:])
        objs.append(o)
    r = subprocess.run(["g++", "-shared", "-o", REF_LIB] + objs, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference link failed:\n" + r.stderr[-4000:])
    return REF_LIB


def bullet_sources():
    """The reference's bullet2 core: LinearMath, BulletCollision, BulletDynamics."""
    out = []
    for sub in ("LinearMath", "BulletCollision", "BulletDynamics"):
        for root, _, files in os.walk(os.path.join(REFERENCE, "bullet2", sub)):
            out += [os.path.join(root, f) for f in sorted(files) if f.endswith(".cpp")]
    return sorted(out)


def build_bullet(force=False):
    """The reference's CPU rigid-body pipeline (bullet2 btDiscreteDynamicsWorld)
    as a shared library with the C shim oracle/ref_shim_bullet.cpp; the CPU
    baseline of bench.py. Compiled in place from the reference sources with
    g++ -O2; objects go to oracle/_ref/bullet_obj."""
    if not os.path.isdir(REFERENCE):
        return BULLET_LIB if os.path.exists(BULLET_LIB) else None
    shim = os.path.join(HERE, "ref_shim_bullet.cpp")
    srcs = bullet_sources() + [shim]
    if not force and not _stale(BULLET_LIB, srcs):
        return BULLET_LIB
    from concurrent.futures import ThreadPoolExecutor
    objdir = os.path.join(HERE, "_ref", "bullet_obj")
    os.makedirs(objdir, exist_ok=True)
    inc = ["-I", os.path.join(REFERENCE, "bullet2")]

    def compile_one(src):
        rel = os.path.relpath(src, REFERENCE) if src.startswith(REFERENCE) else os.path.basename(src)
        o = os.path.join(objdir, rel.replace(os.sep, "_") + ".o")
        if force or _stale(o, [src]):
            r = subprocess.run(["g++", "-O2", "-fPIC", "-w"] + inc + ["-c", src, "-o", o], capture_output=True,
                               text=True)
            if r.returncode != 0:
                raise RuntimeError("bullet2 build failed: " + src + "\n" + r.stderr[-3000:])
        return o

    with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, srcs))
    r = subprocess.run(["g++", "-shared", "-o", BULLET_LIB] + objs, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("bullet2 link failed:\n" + r.stderr[-4000:])
    return BULLET_LIB


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    print(build_ref(force="--force" in sys.argv))
    print(build_bullet(force="--force" in sys.argv))
