"""C ABI checks that need no GPU: the library loads, exports every function
include/b3gpu.h declares, and the host-side logic behind a host-only
context (device -1) behaves: configuration defaults, hull and body
registration, inertia, error codes and messages."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from experiments_b200 import b3, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(b3_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported():
    lib = b3.load()
    names = declared_functions()
    assert len(names) >= 50
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    names = declared_functions()
    bound = {s[0] for s in b3.SIGNATURES}
    missing = [n for n in sorted(names) if n not in bound]
    assert not missing, missing


def test_struct_layouts_match_reference_sizes():
    # Body 80 B (ST/AdlRigidBody.h:26-45), Inertia 96 B (:47-59),
    # btCollidable 16 B, ConvexPolyhedronCL 96 B, btGpuFace 32 B, Contact4 96 B
    assert C.sizeof(b3.Body) == 80 and C.sizeof(b3.Inertia) == 96
    assert C.sizeof(b3.Collidable) == 16 and C.sizeof(b3.ConvexPolyhedron) == 96
    assert C.sizeof(b3.Face) == 32 and C.sizeof(b3.Contact4) == 96


def test_config_defaults_are_the_reference_constants():
    cfg = b3.default_config()
    assert abs(cfg.dt - 1.0 / 60.0) < 1e-9
    assert cfg.solverIterations == 10
    assert tuple(cfg.gravity) == (0.0, -9.800000190734863, 0.0)
    assert cfg.maxPairsPerBody == 32
    assert all(d & (d - 1) == 0 for d in cfg.gridDims)


def test_host_context_registration(host_ctx):
    sc = scenes.c1(dims=(2, 2, 2))
    w = b3.PhysicsWorld(host_ctx, scenes.world_config(sc))
    scenes.register_scene(w, sc)
    assert w.n == sc.n
    sh = w.shapes()
    nc, npo, nv, nf, ni, ne = sh["counts"]
    assert nc == len(sc.shapes) and npo == len(sc.shapes)
    # the unit cube: 8 vertices, 6 quads, 3 unique edge directions
    cube = sh["polys"][sh["cols"][1].shapeIndex]
    assert (cube.numVertices, cube.numFaces, cube.numUniqueEdges) == (8, 6, 3)
    # inverse inertia from the registration AABB with margin 0.01 and full
    # extents (P1/btGpuNarrowPhaseAndSolver.cpp:566-657): a unit cube of
    # mass 1 -> l = 2 * (0.5 + 0.01) * 2 = 2.04 per axis
    ii = w.inertias()
    dyn = np.where(np.asarray(sc.mass) > 0)[0]
    b0 = dyn[0]
    q = sc.quat[b0]
    if abs(abs(q[3]) - 1) < 1e-7:
        l = 2.04
        expect = 12.0 / (2 * l * l)
        assert np.allclose(ii[b0, :3], expect, rtol=1e-5)
    assert np.all(ii[np.asarray(sc.mass) == 0, :3] == 0)
    w.close()


def test_host_context_refuses_device_work(host_ctx):
    sc = scenes.c1(dims=(2, 2, 2))
    w = b3.PhysicsWorld(host_ctx, scenes.world_config(sc))
    scenes.register_scene(w, sc)
    lib = b3.load()
    assert lib.b3_step(w.h, 1, None) == 5  # B3_ERR_STATE: bodies not written yet
    assert lib.b3_write_bodies(w.h, None) == 4  # B3_ERR_NO_DEVICE
    msg = lib.b3_last_error()
    assert msg and len(msg) > 0
    w.close()


def test_invalid_arguments_are_reported(host_ctx):
    lib = b3.load()
    out = C.c_void_p()
    assert lib.b3_world_create(None, None, C.byref(out)) == 1
    cfg = b3.default_config()
    cfg.gridDims[0] = 100  # not a power of two
    assert lib.b3_world_create(host_ctx.h, C.byref(cfg), C.byref(out)) == 1
    w = b3.PhysicsWorld(host_ctx, b3.default_config())
    col = C.c_int()
    pts = np.zeros((2, 3), np.float32)  # fewer than 4 points: no hull
    assert lib.b3_register_convex_hull(w.h, pts.ctypes.data_as(C.POINTER(C.c_float)), 2, 12, None,
                                       C.byref(col)) != 0
    bid = C.c_int()
    pos = (C.c_float * 3)(0, 0, 0)
    q = (C.c_float * 4)(0, 0, 0, 1)
    assert lib.b3_register_body(w.h, 1.0, pos, q, 7, 0.5, 0.0, 0, C.byref(bid)) == 1  # unknown collidable
    w.close()


def test_tuning_values_round_trip_and_are_checked(host_ctx):
    """b3_get_tuning / b3_set_tuning are host state: ten values (index 8 the
    grid pair search form, index 9 the narrowphase lane-group form), the
    read-only ones ignored on set, every out-of-range value refused."""
    w = b3.PhysicsWorld(host_ctx, b3.default_config())
    t = w.tuning()
    assert len(t) == 10
    assert t[8] in (0, 1) and t[9] in (0, 1)
    want = [4, t[1], 64, t[3], 2, t[5], 1, 1, 1, 0]
    w.set_tuning(want)
    got = w.tuning()
    for i in (0, 2, 4, 6, 7, 8, 9):
        assert got[i] == want[i], i
    # shorter lists keep the later values
    w.set_tuning([2, t[1], 128])
    got2 = w.tuning()
    assert got2[0] == 2 and got2[2] == 128 and got2[8] == 1 and got2[9] == 0
    lib = b3.load()
    for i, bad in ((0, 3), (2, 96), (4, 0), (4, 9), (6, 2), (7, 2), (8, 2), (9, 2), (9, -1)):
        v = list(got2)
        v[i] = bad
        arr = (C.c_int * len(v))(*v)
        assert lib.b3_set_tuning(w.h, arr, len(v)) == 1, (i, bad)  # B3_ERR_INVALID_ARG
    assert w.tuning() == got2  # a refused set changes nothing
    w.close()


def test_scene_generator_is_deterministic():
    a = scenes.c2(dims=(4, 2, 4))
    b = scenes.c2(dims=(4, 2, 4))
    for f in ("pos", "quat", "mass", "friction", "shape"):
        assert np.array_equal(getattr(a, f), getattr(b, f))
    c = scenes.c2(seed=7, dims=(4, 2, 4))
    assert not np.array_equal(a.pos, c.pos)
    # counter-based generator: a prefix does not depend on the length drawn
    u1 = scenes.uniform(5, 3, 10, 0.0, 1.0)
    u2 = scenes.uniform(5, 3, 20, 0.0, 1.0)
    assert np.array_equal(u1, u2[:10])


def test_batch_world_offsets(host_ctx):
    sc = scenes.c3(worlds=16)
    w = b3.PhysicsWorld(host_ctx, scenes.world_config(sc))
    scenes.register_scene(w, sc)
    off = w.world_offsets()
    assert len(off) == 17 and off[0] == 0 and off[-1] == sc.n
    counts = np.bincount(np.asarray(sc.world), minlength=16)
    assert np.array_equal(np.diff(off), counts)
    w.close()


def test_adjoint_call_order(host_ctx):
    lib = b3.load()
    w = b3.PhysicsWorld(host_ctx, b3.default_config())
    a = C.c_void_p()
    # bodies not written (and no device): the adjoint cannot be created
    assert lib.b3_adjoint_create(w.h, 10, 4, C.byref(a)) == 5
    assert lib.b3_adjoint_create(w.h, 0, 4, C.byref(a)) == 1
    assert lib.b3_adjoint_forward(None, None) == 1
    assert lib.b3_adjoint_gradients(None, None, None, None, None) == 1
    w.close()


def test_large_hull_registers_quickly(host_ctx):
    """Registration builds the hull in O(points x faces) on the integer
    grid: 65,536 points of a shell register in well under the time an
    exhaustive plane search would take, and every point lies inside every
    face plane of the result."""
    import time
    rng = np.random.default_rng(5)
    p = rng.normal(size=(65536, 3))
    p /= np.linalg.norm(p, axis=1, keepdims=True)
    p = (p * rng.uniform(0.5, 1.0, (65536, 1))).astype(np.float32)
    w = b3.PhysicsWorld(host_ctx, b3.default_config(maxBodies=4))
    t0 = time.perf_counter()
    w.registerConvexPolyhedron(p)
    assert time.perf_counter() - t0 < 10.0
    sh = w.shapes()
    poly = sh["polys"][0]
    assert poly.numVertices > 100 and poly.numFaces > 100
    planes = np.array([list(sh["faces"][f].plane) for f in range(poly.faceOffset, poly.faceOffset + poly.numFaces)])
    # grid vertices sit within one grid step (extent / 10216) of the input
    assert (p @ planes[:, :3].T + planes[:, 3]).max() < 2.0 / 10216 * 2
    w.close()
