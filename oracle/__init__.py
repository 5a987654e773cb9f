"""ORACLE — test infrastructure only.

Python binding of the single-threaded C++ restatement of the reference
rigid-body step (oracle/b3_oracle.cpp) and of the reference pieces compiled
from the reference's own sources (oracle/_ref/libb3ref.so). Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg use this package, as
the checker; the product (experiments_b200) never imports it.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
LIB_F32 = os.path.join(HERE, "liboracle_f32.so")
LIB_DUAL = os.path.join(HERE, "liboracle_dual.so")
REF_LIB = os.path.join(HERE, "_ref", "libb3ref.so")
BULLET_LIB = os.path.join(HERE, "_ref", "libb3bullet.so")


class OrConfig(C.Structure):
    _fields_ = [("cellSize", C.c_float), ("dims", C.c_int * 3), ("maxBodiesPerCell", C.c_int),
                ("maxPairsPerBody", C.c_int), ("gravity", C.c_float * 3), ("dt", C.c_float),
                ("iterations", C.c_int), ("erp", C.c_float), ("contactBreaking", C.c_float),
                ("contactProcessing", C.c_float), ("slopOffset", C.c_float), ("angularDamping", C.c_float),
                ("frictionCombine", C.c_int), ("numWorlds", C.c_int), ("maxPairs", C.c_int)]


class OrContact(C.Structure):
    _fields_ = [("pos", (C.c_double * 4) * 4), ("normal", C.c_double * 4), ("friction", C.c_double),
                ("pairIndex", C.c_int), ("bodyA", C.c_int), ("bodyB", C.c_int), ("pad", C.c_int)]


# OrContact as a numpy record (same field order and packing)
_OR_CONTACT_DTYPE = np.dtype([("pos", "<f8", (4, 4)), ("normal", "<f8", 4), ("friction", "<f8"),
                              ("pairIndex", "<i4"), ("bodyA", "<i4"), ("bodyB", "<i4"), ("pad", "<i4")])
assert _OR_CONTACT_DTYPE.itemsize == C.sizeof(OrContact)

_ref = None
_bullet = None
_D = C.POINTER(C.c_double)
_F = C.POINTER(C.c_float)
_I = C.POINTER(C.c_int)
_U = C.POINTER(C.c_uint32)
_VP = C.c_void_p


_libs = {}


def lib(f32=False, dual=False):
    """The FP64 oracle; with f32=True the same restatement in FP32 (used to
    tell precision effects from logic differences); with dual=True the FP64
    restatement carrying forward-mode derivatives (tangent-linear build)."""
    kind = "dual" if dual else ("f32" if f32 else "f64")
    if kind not in _libs:
        path = {"f64": LIB, "f32": LIB_F32, "dual": LIB_DUAL}[kind]
        if not os.path.exists(path):
            from . import build
            build.build_oracle()
        L = C.CDLL(path)
        L.or_world_create.restype = _VP
        L.or_world_create.argtypes = [C.POINTER(OrConfig), C.c_int, _F, _F, _F, _I, _I, _I, _F, C.c_int, _I,
                                      C.c_int, _VP, C.c_int, _F, C.c_int, _VP, C.c_int, _I, C.c_int, _F, _F]
        L.or_world_destroy.argtypes = [_VP]
        L.or_set_collidables.argtypes = [_VP, C.c_int, _I, _F, _I, _I, C.c_int, _F, _I]
        L.or_set_state_f32.argtypes = [_VP, _F, _F, _F, _F]
        L.or_set_state_f64.argtypes = [_VP, _D, _D, _D, _D]
        L.or_get_state.argtypes = [_VP, _D, _D, _D, _D]
        for s in ("aabbs", "broadphase", "narrowphase", "solve", "integrate"):
            getattr(L, "or_stage_" + s).argtypes = [_VP]
        L.or_step.argtypes = [_VP, C.c_int]
        L.or_get_aabbs.argtypes = [_VP, _F]
        L.or_get_sorted.argtypes = [_VP, _U, _U, C.c_int]
        L.or_get_pairs.argtypes = [_VP, _I, C.c_int]
        L.or_get_contacts.argtypes = [_VP, C.POINTER(OrContact), C.c_int]
        L.or_get_overflow.argtypes = [_VP, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
        L.or_set_contacts.argtypes = [_VP, C.POINTER(OrContact), C.c_int]
        L.or_set_pairs.argtypes = [_VP, _I, C.c_int]
        L.or_pair_contact.argtypes = [_VP, C.c_int, C.c_int, C.POINTER(OrContact)]
        L.or_clip_reduce.argtypes = [_VP, C.c_int, C.c_int, _D, _D, _D, C.c_int, C.c_double, _D, _D, _I]
        L.or_solve_velocities.argtypes = [_VP, _D, _D]
        L.or_active_hash.argtypes = [_VP, C.POINTER(C.c_uint64), C.c_int]
        L.or_reset_active.argtypes = [_VP]
        L.or_set_params_f64.argtypes = [_VP, _D, _D, _D]
        L.or_clip_face_world.argtypes = [_D, C.c_int, _D, _D, C.c_int, C.c_double, C.c_double, _D]
        L.or_set_tangent.argtypes = [_VP, _D, _D, _D, _D, _D]
        L.or_get_tangent.argtypes = [_VP, _D, _D, _D, _D]
        L.or_set_tangent_pose.argtypes = [_VP, _D, _D]
        L.or_real_kind.restype = C.c_int
        L.or_set_broadphase.argtypes = [_VP, C.c_int]
        L.or_set_solver.argtypes = [_VP, C.c_int]
        L.or_gs_batches.restype = C.c_int
        L.or_gs_batches.argtypes = [_VP, _I, C.c_int]
        L.or_gs_applied.restype = C.c_int
        L.or_gs_applied.argtypes = [_VP, _D, C.c_int]
        L.or_gs_constraint.argtypes = [_D, _D, _D, _D, C.c_double, C.c_double, _D, _D, C.c_double, _D]
        L.or_sap_sorted_pairs.restype = C.c_int
        L.or_sap_sorted_pairs.argtypes = [_F, C.c_int, C.c_int, _I, C.c_int]
        _libs[kind] = L
    return _libs[kind]


def ref_lib():
    """The reference pieces compiled from its sources, or None if absent."""
    global _ref
    if _ref is None and os.path.exists(REF_LIB):
        R = C.CDLL(REF_LIB)
        R.ref_jacobi_solve.argtypes = [C.c_int, _VP, _VP, C.c_int, _VP]
        R.ref_hull.argtypes = [_F, C.c_int, _F, C.c_int, _I, _F, _I, C.c_int, _I, _I, C.c_int, _F, C.c_int, _I]
        R.ref_clip_reduce.argtypes = [_F, _I, _I, _F, _F, _F, C.c_int, _F, _I, C.c_int, _I, C.c_int, _F, _F, _F,
                                      _F, C.c_float, _F, _I]
        _ref = R
    return _ref


def bullet_lib():
    """The reference's CPU rigid-body pipeline (bullet2 btDiscreteDynamicsWorld)
    compiled from its sources, or None if absent."""
    global _bullet
    if _bullet is None and os.path.exists(BULLET_LIB):
        B = C.CDLL(BULLET_LIB)
        B.rb_create.restype = _VP
        B.rb_create.argtypes = [C.c_int, _I, _F, C.c_int, _I, _F, _F, _F, _F, _F, _F, _I, C.c_int, C.c_float,
                                C.c_int, C.c_float, C.c_float, C.c_float]
        B.rb_step.argtypes = [_VP, C.c_int]
        B.rb_positions.argtypes = [_VP, _F]
        B.rb_destroy.argtypes = [_VP]
        B.rb_write_bullet.restype = C.c_int
        B.rb_write_bullet.argtypes = [_VP, C.c_char_p]
        _bullet = B
    return _bullet


def _bullet_points(shape):
    """A scene shape as the shim's point list: hull points, one point
    (radius, 0, 0) for a sphere, two (normal; constant, 0, 0) for a plane."""
    if isinstance(shape, dict):
        if shape["kind"] == "sphere":
            return np.array([[shape["radius"], 0.0, 0.0]], np.float32)
        if shape["kind"] == "plane":
            return np.array([shape["normal"], [shape["constant"], 0.0, 0.0]], np.float32)
        raise NotImplementedError(f"{shape['kind']} shapes in the reference CPU pipeline")
    return np.asarray(shape, np.float32).reshape(-1, 3)


class ReferenceCpuWorld:
    """A scene in the reference's CPU pipeline (btDiscreteDynamicsWorld:
    btDbvtBroadphase + btSequentialImpulseConstraintSolver, 10 iterations);
    boxes as btBoxShape, other hulls as btConvexHullShape of the same points,
    one dynamics world per independent world."""

    def __init__(self, scene, dt=1.0 / 60.0, iterations=10, gravity=(0.0, -9.8, 0.0)):
        B = bullet_lib()
        if B is None:
            raise RuntimeError("oracle/_ref/libb3bullet.so not built")
        self.B = B
        self.n = scene.n
        pts = [_bullet_points(v) for v in scene.shapes]
        offs = np.zeros(len(pts) + 1, np.int32)
        offs[1:] = np.cumsum([len(p) for p in pts])
        allp = np.ascontiguousarray(np.concatenate(pts).astype(np.float32))
        f32 = lambda a, k: np.ascontiguousarray(np.asarray(a, np.float32).reshape(-1, k))
        self._keep = [offs, allp, np.ascontiguousarray(np.asarray(scene.shape, np.int32)), f32(scene.mass, 1),
                      f32(scene.pos, 3), f32(scene.quat, 4), f32(scene.friction, 1), f32(scene.lin, 3),
                      f32(scene.ang, 3), np.ascontiguousarray(np.asarray(scene.world, np.int32))]
        k = self._keep
        self.h = B.rb_create(len(pts), _i(k[0]), _f(k[1]), self.n, _i(k[2]), _f(k[3]), _f(k[4]), _f(k[5]), _f(k[6]),
                             _f(k[7]), _f(k[8]), _i(k[9]), int(scene.num_worlds), float(dt), int(iterations),
                             *[float(g) for g in gravity])

    def step(self, steps=1):
        self.B.rb_step(self.h, int(steps))

    def positions(self):
        out = np.zeros((self.n, 3), np.float32)
        self.B.rb_positions(self.h, _f(out))
        return out

    def write_bullet(self, path):
        """The first world written by bullet2's btDefaultSerializer (a .bullet file)."""
        if self.B.rb_write_bullet(self.h, os.fsencode(path)) != 0:
            raise RuntimeError(f"could not write {path}")

    def close(self):
        if self.h:
            self.B.rb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _f(a):
    return a.ctypes.data_as(_F)


def _i(a):
    return a.ctypes.data_as(_I)


def _d(a):
    return a.ctypes.data_as(_D)


class OracleWorld:
    """Oracle world built from a registered product world's shape tables
    (hull construction is checked separately against btConvexUtility)."""

    def __init__(self, scene, shapes, cfg, inv_inertia, is_large, f32=False, dual=False):
        L = lib(f32, dual)
        self.n = scene.n
        c = OrConfig()
        c.cellSize = cfg.cellSize
        for k in range(3):
            c.dims[k] = cfg.gridDims[k]
            c.gravity[k] = cfg.gravity[k]
        c.maxBodiesPerCell = cfg.maxBodiesPerCell
        c.maxPairsPerBody = cfg.maxPairsPerBody
        c.dt = cfg.dt
        c.iterations = cfg.solverIterations
        c.erp = cfg.erp
        c.contactBreaking = cfg.contactBreaking
        c.contactProcessing = cfg.contactProcessing
        c.slopOffset = cfg.linearSlopOffset
        c.angularDamping = cfg.angularDamping
        c.frictionCombine = cfg.frictionCombine
        c.numWorlds = cfg.numWorlds
        c.maxPairs = cfg.maxPairs
        self.cfg = c
        n = scene.n
        m = np.asarray(scene.mass, np.float64)
        self._keep = dict(
            invMass=np.ascontiguousarray(np.where(m != 0, 1.0 / np.where(m != 0, m, 1), 0).astype(np.float32)),
            fr=np.ascontiguousarray(scene.friction.astype(np.float32)),
            rs=np.zeros(n, np.float32),
            col=np.ascontiguousarray(shapes["col_of_body"].astype(np.int32)),
            wid=np.ascontiguousarray(scene.world.astype(np.int32)),
            large=np.ascontiguousarray(np.asarray(is_large, np.int32)),
            ii=np.ascontiguousarray(np.asarray(inv_inertia, np.float32).reshape(n, 4)),
            colShape=np.ascontiguousarray(np.array([shapes["cols"][k].shapeIndex for k in range(shapes["counts"][0])],
                                                   np.int32)),
            verts=np.ascontiguousarray(shapes["verts"].astype(np.float32)),
            idx=np.ascontiguousarray(shapes["idx"].astype(np.int32)),
            edges=np.ascontiguousarray(shapes["edges"].astype(np.float32)),
            laabb=np.ascontiguousarray(shapes["localAabb"].astype(np.float32)),
        )
        k = self._keep
        nc, npo, nv, nf, ni, ne = shapes["counts"]
        self.h = L.or_world_create(C.byref(c), n, _f(k["invMass"]), _f(k["fr"]), _f(k["rs"]), _i(k["col"]),
                                   _i(k["wid"]), _i(k["large"]), _f(k["ii"]), nc, _i(k["colShape"]), npo,
                                   C.cast(shapes["polys"], _VP), nv, _f(k["verts"]), nf,
                                   C.cast(shapes["faces"], _VP), ni, _i(k["idx"]), ne, _f(k["edges"]),
                                   _f(k["laabb"]))
        self.L = L
        # the collidable table (types other than hulls, compound children)
        cols = shapes["cols"]
        nc = shapes["counts"][0]
        ch = shapes.get("children", [])
        self._keep["colType"] = np.ascontiguousarray(np.array([cols[k].shapeType for k in range(nc)], np.int32))
        self._keep["colRadius"] = np.ascontiguousarray(np.array([cols[k].radius for k in range(nc)], np.float32))
        self._keep["colNum"] = np.ascontiguousarray(np.array([cols[k].numChildShapes for k in range(nc)], np.int32))
        self._keep["colIndex"] = np.ascontiguousarray(np.array([cols[k].shapeIndex for k in range(nc)], np.int32))
        pose = np.zeros((max(len(ch), 1), 8), np.float32)
        ccol = np.zeros(max(len(ch), 1), np.int32)
        for j, c in enumerate(ch):
            pose[j, :4] = list(c.childPosition)
            pose[j, 4:] = list(c.childOrientation)
            ccol[j] = c.shapeIndex
        self._keep["childPose"] = np.ascontiguousarray(pose)
        self._keep["childCol"] = np.ascontiguousarray(ccol)
        k = self._keep
        L.or_set_collidables(self.h, nc, _i(k["colType"]), _f(k["colRadius"]), _i(k["colNum"]), _i(k["colIndex"]),
                             len(ch), _f(k["childPose"]), _i(k["childCol"]))
        if int(getattr(cfg, "flags", 0)) & 1:
            L.or_set_broadphase(self.h, 1)  # sweep and prune
        if int(getattr(cfg, "flags", 0)) & 2:
            L.or_set_solver(self.h, 1)  # batched Gauss-Seidel
        pos4 = np.zeros((n, 4), np.float32)
        pos4[:, :3] = scene.pos
        lin4 = np.zeros((n, 4), np.float32)
        lin4[:, :3] = scene.lin
        ang4 = np.zeros((n, 4), np.float32)
        ang4[:, :3] = scene.ang
        self.set_state_f32(pos4, np.ascontiguousarray(scene.quat.astype(np.float32)), lin4, ang4)

    def set_state_f32(self, pos4, quat4, lin4, ang4):
        arrs = [np.ascontiguousarray(np.asarray(a, np.float32).reshape(self.n, 4)) for a in (pos4, quat4, lin4, ang4)]
        self.L.or_set_state_f32(self.h, *[_f(a) for a in arrs])

    def set_state_f64(self, pos4, quat4, lin4, ang4):
        arrs = [np.ascontiguousarray(np.asarray(a, np.float64).reshape(self.n, 4)) for a in (pos4, quat4, lin4, ang4)]
        self.L.or_set_state_f64(self.h, *[_d(a) for a in arrs])

    def state(self):
        out = [np.zeros((self.n, 4), np.float64) for _ in range(4)]
        self.L.or_get_state(self.h, *[_d(a) for a in out])
        return out

    def stage(self, name):
        getattr(self.L, "or_stage_" + name)(self.h)

    def step(self, steps=1):
        self.L.or_step(self.h, steps)

    def aabbs(self):
        out = np.zeros((self.n, 8), np.float32)
        self.L.or_get_aabbs(self.h, _f(out))
        return out

    def sorted_hash(self):
        cnt = self.L.or_get_sorted(self.h, None, None, 0)
        k = np.zeros(max(cnt, 1), np.uint32)
        v = np.zeros(max(cnt, 1), np.uint32)
        self.L.or_get_sorted(self.h, k.ctypes.data_as(_U), v.ctypes.data_as(_U), cnt)
        return k[:cnt], v[:cnt]

    def pairs(self):
        cnt = self.L.or_get_pairs(self.h, None, 0)
        out = np.zeros((max(cnt, 1), 2), np.int32)
        self.L.or_get_pairs(self.h, _i(out), cnt)
        return out[:cnt]

    def set_pairs(self, pairs):
        p = np.ascontiguousarray(np.asarray(pairs, np.int32).reshape(-1, 2))
        self.L.or_set_pairs(self.h, _i(p), p.shape[0])

    def contacts(self):
        cnt = self.L.or_get_contacts(self.h, None, 0)
        arr = (OrContact * max(cnt, 1))()
        self.L.or_get_contacts(self.h, arr, cnt)
        raw = np.frombuffer(C.string_at(C.addressof(arr), C.sizeof(OrContact) * cnt), np.uint8)
        raw = raw.reshape(cnt, C.sizeof(OrContact)) if cnt else np.zeros((0, C.sizeof(OrContact)), np.uint8)
        d = raw[:, :168].copy().view(np.float64).reshape(cnt, 21) if cnt else np.zeros((0, 21))
        i = raw[:, 168:184].copy().view(np.int32).reshape(cnt, 4) if cnt else np.zeros((0, 4), np.int32)
        return dict(pos=d[:, :16].reshape(-1, 4, 4), normal=d[:, 16:20], friction=d[:, 20], pairIndex=i[:, 0],
                    bodyA=i[:, 1], bodyB=i[:, 2])

    def set_contacts(self, c):
        n = len(c["normal"])
        rec = np.zeros(max(n, 1), dtype=_OR_CONTACT_DTYPE)
        if n:
            rec["pos"][:n] = np.asarray(c["pos"], np.float64).reshape(n, 4, 4)
            rec["normal"][:n] = np.asarray(c["normal"], np.float64).reshape(n, 4)
            rec["friction"][:n] = np.asarray(c["friction"], np.float64)
            rec["pairIndex"][:n] = np.asarray(c["pairIndex"], np.int32)
            rec["bodyA"][:n] = np.asarray(c["bodyA"], np.int32)
            rec["bodyB"][:n] = np.asarray(c["bodyB"], np.int32)
        self.L.or_set_contacts(self.h, C.cast(rec.ctypes.data, C.POINTER(OrContact)), n)

    def overflow(self):
        a, b = C.c_longlong(), C.c_longlong()
        self.L.or_get_overflow(self.h, C.byref(a), C.byref(b))
        return a.value, b.value

    def set_tangent(self, lin=None, ang=None, inv_mass=None, inv_inertia3=None, friction=None):
        """Derivative seeds (tangent-linear build): initial linear / angular
        velocities (n x 3), inverse masses, local inverse inertia diagonals
        (n x 3) and friction coefficients; None means zero."""
        keep = []
        for a, cols in ((lin, 4), (ang, 4), (inv_mass, 1), (inv_inertia3, 3), (friction, 1)):
            if a is None:
                keep.append(None)
                continue
            a = np.asarray(a, np.float64).reshape(self.n, -1)
            b = np.zeros((self.n, cols))
            b[:, :a.shape[1]] = a
            keep.append(np.ascontiguousarray(b))
        self.L.or_set_tangent(self.h, *[None if a is None else _d(a) for a in keep])

    def set_tangent_pose(self, pos=None, quat=None):
        """Derivative seeds of the positions and quaternions (n x 4; None
        leaves zero), after set_tangent, which zeroes them."""
        arrs = [None if a is None else np.ascontiguousarray(np.asarray(a, np.float64).reshape(self.n, 4))
                for a in (pos, quat)]
        self.L.or_set_tangent_pose(self.h, *[None if a is None else _d(a) for a in arrs])

    def tangent(self):
        """Derivatives of (pos, quat, lin, ang), each n x 4."""
        out = [np.zeros((self.n, 4), np.float64) for _ in range(4)]
        self.L.or_get_tangent(self.h, *[_d(a) for a in out])
        return out

    def gs_batches(self):
        """(cell, batch) per manifold from the last batched Gauss-Seidel solve (M x 2)."""
        m = self.L.or_gs_batches(self.h, None, 0)
        out = np.zeros((max(m, 1), 2), np.int32)
        self.L.or_gs_batches(self.h, _i(out), m)
        return out[:m]

    def gs_applied(self):
        """Accumulated impulses per manifold from the last batched Gauss-Seidel
        solve: M x 6 (normal [4], friction [2])."""
        m = self.L.or_gs_applied(self.h, None, 0)
        out = np.zeros((max(m, 1), 6))
        self.L.or_gs_applied(self.h, _d(out), m)
        return out[:m]

    def solve_velocities(self):
        lin = np.zeros((self.n, 4))
        ang = np.zeros((self.n, 4))
        self.L.or_solve_velocities(self.h, _d(lin), _d(ang))
        return lin, ang

    def set_params_f64(self, inv_mass=None, friction=None, inv_inertia3=None):
        """Override body parameters in FP64 (None leaves a set unchanged)."""
        keep = [None if a is None else np.ascontiguousarray(np.asarray(a, np.float64).reshape(-1))
                for a in (inv_mass, friction, inv_inertia3)]
        self.L.or_set_params_f64(self.h, *[None if a is None else _d(a) for a in keep])

    def active_hash(self):
        """Per-world signatures of the discrete choices since the last reset,
        shape (worlds, 2): contact topology (pairs with manifolds, clip
        sizes, reduced points) and row clamp states."""
        nw = max(1, int(self.cfg.numWorlds))
        out = np.zeros((nw, 2), np.uint64)
        self.L.or_active_hash(self.h, out.ctypes.data_as(C.POINTER(C.c_uint64)), nw)
        return out

    def reset_active(self):
        self.L.or_reset_active(self.h)

    def close(self):
        if self.h:
            self.L.or_world_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def oracle_from_world(world, scene, cfg=None, f32=False, dual=False):
    """Build an OracleWorld from a registered PhysicsWorld (host-only
    context suffices) and its scene."""
    cfg = cfg or world.cfg
    sh = world.shapes()
    n_shapes = len(scene.shapes)
    # body collidable index = scene.shape (shapes are registered in scene order)
    sh["col_of_body"] = np.asarray(scene.shape, np.int32)
    assert sh["counts"][0] == n_shapes
    arr, cnt = world.child_shapes()
    sh["children"] = [arr[j] for j in range(cnt)]
    inv_inertia = world.inertias()
    # large-body classification rule (half-diagonal of the registration AABB)
    is_large = large_flags(world, scene, cfg)
    return OracleWorld(scene, sh, cfg, inv_inertia, is_large, f32=f32, dual=dual)


def large_flags(world, scene, cfg):
    """Registration-AABB half-diagonal > maxSmallProxySize / 2, computed from
    the scene and the local AABBs (G3/btGpu3DGridBroadphase.cpp:385-391)."""
    sh = world.shapes()
    la = sh["localAabb"].astype(np.float64)
    c = np.asarray(scene.shape)
    lmin, lmax = la[c, :3], la[c, 4:7]
    he = 0.5 * (lmax - lmin) + 0.01
    q = scene.quat.astype(np.float64)
    x, y, z, w = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    s = 2.0 / (x * x + y * y + z * z + w * w)
    R = np.stack([np.stack([1 - (y * y + z * z) * s, (x * y - w * z) * s, (x * z + w * y) * s], 1),
                  np.stack([(x * y + w * z) * s, 1 - (x * x + z * z) * s, (y * z - w * x) * s], 1),
                  np.stack([(x * z - w * y) * s, (y * z + w * x) * s, 1 - (x * x + y * y) * s], 1)], 1)
    e = np.einsum("nij,nj->ni", np.abs(R), he)
    r = np.linalg.norm(e, axis=1)
    return (r > 0.5 * cfg.maxSmallProxySize).astype(np.int32)


def sap_sorted_pairs(sorted_aabbs, axis=0):
    """computePairsKernel restatement on caller-sorted n x 8 float32 AABB
    records; returns the pairs (n_pairs x 2 int32) in the device order."""
    a = np.ascontiguousarray(np.asarray(sorted_aabbs, np.float32).reshape(-1, 8))
    L = lib()
    n = L.or_sap_sorted_pairs(_f(a), a.shape[0], axis, None, 0)
    out = np.zeros((max(n, 1), 2), np.int32)
    L.or_sap_sorted_pairs(_f(a), a.shape[0], axis, _i(out), n)
    return out[:n]


def gs_constraint(pos4x4, normal4, posA, posB, inv_mass_a, inv_mass_b, inv_inertia_a, inv_inertia_b, dt):
    """setConstraint4 of the batched Gauss-Seidel restatement on one manifold:
    (jacCoeffInv[4], b[4], center[3], fJacCoeffInv[2])."""
    out = np.zeros(13)
    arr = [np.ascontiguousarray(np.asarray(a, np.float64).reshape(-1))
           for a in (pos4x4, normal4, posA, posB, inv_inertia_a, inv_inertia_b)]
    lib().or_gs_constraint(_d(arr[0]), _d(arr[1]), _d(arr[2]), _d(arr[3]), float(inv_mass_a), float(inv_mass_b),
                           _d(arr[4]), _d(arr[5]), float(dt), _d(out))
    return out[:4], out[4:8], out[8:11], out[11:13]
