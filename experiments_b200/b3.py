"""ctypes binding of libb3gpu (include/b3gpu.h) and a Python mirror of the
reference pipeline's object API.

The reference objects (C++ over OpenCL) and their counterparts here:
  btFillCL            -> Fill           (BB/btFillCL.h:85-126)
  btPrefixScanCL      -> PrefixScan     (BB/btPrefixScanCL.h:9-35)
  btRadixSort32CL     -> RadixSort32    (BB/btRadixSort32CL.h:14-74)
  btBoundSearchCL     -> BoundSearch    (BB/btBoundSearchCL.h:30-63)
  btGpuNarrowphaseAndSolver + btGridBroadphaseCl + CLPhysicsDemo
                      -> PhysicsWorld   (P1/btGpuNarrowPhaseAndSolver.h:63-123,
                                         BB/btGridBroadphaseCL.h:32-73,
                                         P2/CLPhysicsDemo.h:30-81)
Errors raise B3Error carrying the status code and the library's message,
where the reference would assert (oclCHECKERROR) or truncate silently.
The compute path is the CUDA library only: loading fails loudly if
libb3gpu.so is missing or no sm_100 device is present.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libb3gpu.so")
B3_WORLD_SAP_BROADPHASE = 1  # b3WorldConfig.flags: sweep-and-prune broadphase
BULLET_KEEP_STATIC_OBJECTS = 1  # b3_load_bullet_file_ex flags (B3_BULLET_*)
BULLET_SPHERES_AND_PLANES = 2
B3_WORLD_BATCHED_GS_SOLVER = 2  # b3WorldConfig.flags: the reference GPU solver (batched Gauss-Seidel)

B3_OK = 0
STATUS = {0: "OK", 1: "INVALID_ARG", 2: "CUDA", 3: "CAPACITY", 4: "NO_DEVICE", 5: "STATE",
          6: "TIMEOUT", 7: "UNSUPPORTED"}


class B3Error(RuntimeError):
    def __init__(self, code, where, msg):
        super().__init__(f"{where}: {STATUS.get(code, code)} ({msg})")
        self.code = code


class Body(C.Structure):
    _fields_ = [("pos", C.c_float * 4), ("quat", C.c_float * 4), ("linVel", C.c_float * 4),
                ("angVel", C.c_float * 4), ("collidableIdx", C.c_uint32), ("invMass", C.c_float),
                ("restitution", C.c_float), ("friction", C.c_float)]


class Inertia(C.Structure):
    _fields_ = [("invInertiaWorld", C.c_float * 12), ("initInvInertia", C.c_float * 12)]


class Collidable(C.Structure):
    _fields_ = [("numChildShapes", C.c_int), ("radius", C.c_float), ("shapeType", C.c_int),
                ("shapeIndex", C.c_int)]


class ChildShape(C.Structure):
    _fields_ = [("childPosition", C.c_float * 4), ("childOrientation", C.c_float * 4), ("shapeIndex", C.c_int),
                ("unused", C.c_int * 3)]


SHAPE_CONVEX_HULL, SHAPE_PLANE, SHAPE_CONCAVE_TRIMESH, SHAPE_COMPOUND, SHAPE_SPHERE = 3, 4, 5, 6, 7


class ConvexPolyhedron(C.Structure):
    _fields_ = [("localCenter", C.c_float * 4), ("extents", C.c_float * 4), ("mC", C.c_float * 4),
                ("mE", C.c_float * 4), ("radius", C.c_float), ("faceOffset", C.c_int),
                ("numFaces", C.c_int), ("numVertices", C.c_int), ("vertexOffset", C.c_int),
                ("uniqueEdgesOffset", C.c_int), ("numUniqueEdges", C.c_int), ("unused", C.c_int)]


class Face(C.Structure):
    _fields_ = [("plane", C.c_float * 4), ("indexOffset", C.c_int), ("numIndices", C.c_int),
                ("pad", C.c_int * 2)]


class Contact4(C.Structure):
    _fields_ = [("worldPos", (C.c_float * 4) * 4), ("worldNormal", C.c_float * 4),
                ("friction", C.c_float), ("pairIndex", C.c_int), ("bodyAPtrAndSignBit", C.c_int),
                ("bodyBPtrAndSignBit", C.c_int)]


class Constraint4(C.Structure):
    _fields_ = [("linear", C.c_float * 4), ("worldPos", (C.c_float * 4) * 4), ("center", C.c_float * 4),
                ("jacCoeffInv", C.c_float * 4), ("b", C.c_float * 4), ("appliedRambdaDt", C.c_float * 4),
                ("fJacCoeffInv", C.c_float * 2), ("fAppliedRambdaDt", C.c_float * 2), ("bodyA", C.c_uint32),
                ("bodyB", C.c_uint32), ("batchIdx", C.c_int32), ("padding", C.c_uint32)]


class Counters(C.Structure):
    _fields_ = [("numPairs", C.c_int32), ("numManifolds", C.c_int32), ("numContactPoints", C.c_int32),
                ("pairOverflow", C.c_int32), ("cellOverflow", C.c_int32), ("timeouts", C.c_int32),
                ("clipOverflow", C.c_int32), ("steps", C.c_int32), ("refinedAxes", C.c_int32),
                ("refinedClips", C.c_int32)]

    def as_dict(self):
        return {f: int(getattr(self, f)) for f, _ in self._fields_}


class WorldConfig(C.Structure):
    _fields_ = [("maxBodies", C.c_int32), ("maxPairs", C.c_int32), ("numWorlds", C.c_int32),
                ("cellSize", C.c_float), ("gridDims", C.c_int32 * 3), ("maxBodiesPerCell", C.c_int32),
                ("maxPairsPerBody", C.c_int32), ("maxSmallProxySize", C.c_float),
                ("gravity", C.c_float * 3), ("dt", C.c_float), ("solverIterations", C.c_int32),
                ("erp", C.c_float), ("contactBreaking", C.c_float), ("contactProcessing", C.c_float),
                ("linearSlopOffset", C.c_float), ("angularDamping", C.c_float),
                ("frictionCombine", C.c_int32), ("useGraph", C.c_int32), ("flags", C.c_int32)]


assert C.sizeof(Body) == 80 and C.sizeof(Inertia) == 96 and C.sizeof(Collidable) == 16
assert C.sizeof(ConvexPolyhedron) == 96 and C.sizeof(Face) == 32 and C.sizeof(Contact4) == 96

BUF = {"pos": 0, "quat": 1, "linVel": 2, "angVel": 3, "aabbMin": 4, "aabbMax": 5, "pairs": 6,
       "contacts": 7, "counters": 8, "invMass": 9}

_lib = None

# (name, restype, argtypes) of every exported entry point of include/b3gpu.h
_P = C.c_void_p
_I = C.c_int
_I64 = C.c_int64
_FP = C.POINTER(C.c_float)
_IP = C.POINTER(C.c_int)
_U32P = C.POINTER(C.c_uint32)
SIGNATURES = [
    ("b3_context_create", _I, [_I, C.POINTER(_P)]),
    ("b3_context_destroy", _I, [_P]),
    ("b3_sync", _I, [_P, _P]),
    ("b3_context_info", _I, [_P, C.c_char_p, _I]),
    ("b3_last_error", C.c_char_p, []),
    ("b3_fill_u32", _I, [_P, _P, C.c_uint32, _I64, _I64, _P]),
    ("b3_fill_int2", _I, [_P, _P, C.c_int32, C.c_int32, _I64, _I64, _P]),
    ("b3_prefix_scan_u32", _I, [_P, _P, _P, _I64, _P, _U32P, _P]),
    ("b3_prefix_scan_u32_static", _I, [_P, _P, _I64, _P, _P, _P]),
    ("b3_radix_sort32_kv", _I, [_P, _P, _P, _I64, _I, _P]),
    ("b3_radix_sort32_keys", _I, [_P, _P, _I64, _I, _P]),
    ("b3_bound_search", _I, [_P, _P, _I64, _P, _I64, _I, _P]),
    ("b3_set_wait_limits", _I, [_P, _I, _I]),
    ("b3_register_sphere", _I, [_P, C.c_float, _IP]),
    ("b3_register_plane", _I, [_P, _FP, C.c_float, _IP]),
    ("b3_register_compound", _I, [_P, _P, _I, _IP]),
    ("b3_register_concave_mesh", _I, [_P, _FP, _I, _IP, _I, _FP, _IP]),
    ("b3_get_child_shapes", _I, [_P, _P, _I, _IP]),
    ("b3_radix_sort32_kv_out", _I, [_P, _P, _P, _P, _P, _I64, _I, _P]),
    ("b3_radix_sort32_sortdata", _I, [_P, _P, _I64, _I, _P]),
    ("b3_bound_search_sortdata", _I, [_P, _P, _I64, _P, _I64, _I, _P]),
    ("b3_world_config_default", None, [C.POINTER(WorldConfig)]),
    ("b3_world_create", _I, [_P, C.POINTER(WorldConfig), C.POINTER(_P)]),
    ("b3_world_destroy", _I, [_P]),
    ("b3_register_convex_hull", _I, [_P, _FP, _I, _I, _FP, _IP]),
    ("b3_register_body", _I, [_P, C.c_float, _FP, _FP, _I, C.c_float, C.c_float, _I, _IP]),
    ("b3_register_bodies", _I, [_P, _I, _FP, _FP, _FP, _IP, _FP, _FP, _IP, _IP]),
    ("b3_write_bodies", _I, [_P, _P]),
    ("b3_write_velocities", _I, [_P, _FP, _FP, _P]),
    ("b3_step", _I, [_P, _I, _P]),
    ("b3_read_bodies", _I, [_P, C.POINTER(Body), _I, _P]),
    ("b3_read_state", _I, [_P, _FP, _FP, _FP, _FP, _P]),
    ("b3_write_state", _I, [_P, _FP, _FP, _FP, _FP, _P]),
    ("b3_get_num_bodies", _I, [_P, _IP]),
    ("b3_get_counters", _I, [_P, C.POINTER(Counters), _P]),
    ("b3_reset_counters", _I, [_P, _P]),
    ("b3_stage_aabbs", _I, [_P, _P]),
    ("b3_stage_broadphase", _I, [_P, _P]),
    ("b3_stage_narrowphase", _I, [_P, _P]),
    ("b3_stage_solve", _I, [_P, _P]),
    ("b3_stage_integrate", _I, [_P, _P]),
    ("b3_grid_broadphase_calculate_overlapping_pairs", _I, [_P, _P]),
    ("b3_sap_broadphase_calculate_overlapping_pairs", _I, [_P, _P]),
    ("b3_sap_compute_pairs", _I, [_P, _P, _I, _I, _P, _I, _P, _P]),
    ("b3_grid_broadphase_get_pair_count", _I, [_P, _IP, _P]),
    ("b3_narrowphase_compute_contacts", _I, [_P, _P, _I, _P]),
    ("b3_solver_solve_jacobi", _I, [_P, _P]),
    ("b3_solver_solve_batched_gs", _I, [_P, _P]),
    ("b3_load_bullet_file", _I, [_P, C.c_char_p, _I, _IP]),
    ("b3_load_bullet_file_ex", _I, [_P, C.c_char_p, _I, _IP]),
    ("b3_get_gs_batches", _I, [_P, _IP, _I, _IP, _P]),
    ("b3_get_gs_constraints", _I, [_P, C.POINTER(Constraint4), _I, _IP, _P]),
    ("b3_integrate", _I, [_P, _P]),
    ("b3_get_aabbs", _I, [_P, _FP, _I, _P]),
    ("b3_get_sorted_hash", _I, [_P, _U32P, _U32P, _I, _IP, _P]),
    ("b3_get_pairs", _I, [_P, _IP, _I, _IP, _P]),
    ("b3_get_contacts", _I, [_P, C.POINTER(Contact4), _I, _IP, _P]),
    ("b3_get_shape_sizes", _I, [_P, _IP, _IP, _IP, _IP, _IP, _IP]),
    ("b3_get_shapes", _I, [_P, C.POINTER(Collidable), C.POINTER(ConvexPolyhedron), _FP,
                           C.POINTER(Face), _IP, _FP, _FP]),
    ("b3_get_inertias", _I, [_P, C.POINTER(Inertia), _I]),
    ("b3_get_device_buffer", _I, [_P, _I, C.POINTER(_P), C.POINTER(_I64)]),
    ("b3_set_stage_timing", _I, [_P, _I]),
    ("b3_get_stage_times", _I, [_P, _FP, _I, _IP]),
    ("b3_batch_world_stats", _I, [_P, _FP, _I, _P]),
    ("b3_batch_world_offsets", _I, [_P, _IP, _I, _IP]),
    ("b3_autotune", _I, [_P, _I, _P]),
    ("b3_get_tuning", _I, [_P, _IP, _I, _IP]),
    ("b3_set_tuning", _I, [_P, _IP, _I]),
    ("b3_adjoint_create", _I, [_P, _I, _I, C.POINTER(_P)]),
    ("b3_adjoint_destroy", _I, [_P]),
    ("b3_adjoint_forward", _I, [_P, _P]),
    ("b3_adjoint_backward", _I, [_P, _FP, _FP, _FP, _FP, _P]),
    ("b3_adjoint_gradients", _I, [_P, _FP, _FP, _FP, _FP]),
    ("b3_adjoint_info", _I, [_P, _IP]),
]


def load(path=None):
    """Load libb3gpu.so (no compute happens here)."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise B3Error(4, "load", f"{p} missing; run `python -m experiments_b200.build`")
    lib = C.CDLL(p)
    for name, res, args in SIGNATURES:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _check(code, where):
    if code != B3_OK:
        msg = _lib.b3_last_error().decode(errors="replace") if _lib else ""
        raise B3Error(code, where, msg)


def fptr(a):
    return a.ctypes.data_as(_FP)


def iptr(a):
    return a.ctypes.data_as(_IP)


def _stream(s):
    if s is None:
        return None
    if hasattr(s, "cuda_stream"):
        return C.c_void_p(s.cuda_stream)
    return C.c_void_p(int(s))


class Context:
    """Device + library handle (replaces the OpenCL context/queue pair)."""

    def __init__(self, device=0):
        lib = load()
        h = C.c_void_p()
        _check(lib.b3_context_create(device, C.byref(h)), "b3_context_create")
        self.h = h
        self.lib = lib

    def info(self):
        buf = C.create_string_buffer(256)
        _check(self.lib.b3_context_info(self.h, buf, 256), "b3_context_info")
        return buf.value.decode()

    def sync(self, stream=None):
        _check(self.lib.b3_sync(self.h, _stream(stream)), "b3_sync")

    def close(self):
        if self.h:
            self.lib.b3_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Primitive objects (device pointers are torch CUDA tensors)
# ---------------------------------------------------------------------------
def _dptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


class Fill:
    """btFillCL: fill a device range."""

    def __init__(self, ctx):
        self.ctx = ctx

    def execute(self, dst, value, n=None, offset=0, stream=None):
        n = dst.numel() - offset if n is None else n
        if dst.dim() == 2 and dst.shape[-1] == 2:
            _check(self.ctx.lib.b3_fill_int2(self.ctx.h, _dptr(dst), int(value[0]), int(value[1]), n,
                                             offset, _stream(stream)), "b3_fill_int2")
        else:
            _check(self.ctx.lib.b3_fill_u32(self.ctx.h, _dptr(dst), int(value) & 0xFFFFFFFF, n, offset,
                                            _stream(stream)), "b3_fill_u32")


class PrefixScan:
    """btPrefixScanCL: exclusive scan; returns the total like execute(..., &sum)."""

    def __init__(self, ctx):
        self.ctx = ctx

    def execute(self, src, dst, n=None, stream=None):
        n = src.numel() if n is None else n
        total = C.c_uint32(0)
        _check(self.ctx.lib.b3_prefix_scan_u32(self.ctx.h, _dptr(src), _dptr(dst), n, None,
                                               C.byref(total), _stream(stream)), "b3_prefix_scan_u32")
        return int(total.value)


class RadixSort32:
    """btRadixSort32CL: stable in-place key-value (or keys-only) sort."""

    def __init__(self, ctx):
        self.ctx = ctx

    def execute(self, keys, values=None, n=None, key_bits=32, stream=None):
        n = keys.numel() if n is None else n
        if values is None:
            _check(self.ctx.lib.b3_radix_sort32_keys(self.ctx.h, _dptr(keys), n, key_bits, _stream(stream)),
                   "b3_radix_sort32_keys")
        else:
            _check(self.ctx.lib.b3_radix_sort32_kv(self.ctx.h, _dptr(keys), _dptr(values), n, key_bits,
                                                   _stream(stream)), "b3_radix_sort32_kv")

    def execute_out(self, keys_in, keys_out, values_in=None, values_out=None, n=None, key_bits=32, stream=None):
        """execute(keysIn, keysOut, valuesIn, valuesOut, n, sortBits): out of place."""
        n = keys_in.numel() if n is None else n
        _check(self.ctx.lib.b3_radix_sort32_kv_out(self.ctx.h, _dptr(keys_in), _dptr(keys_out), _dptr(values_in),
                                                   _dptr(values_out), n, key_bits, _stream(stream)),
               "b3_radix_sort32_kv_out")

    def execute_sortdata(self, key_values, n=None, key_bits=32, stream=None):
        """execute(btOpenCLArray<btSortData>&, sortBits): (n, 2) int32 records in place."""
        n = key_values.shape[0] if n is None else n
        _check(self.ctx.lib.b3_radix_sort32_sortdata(self.ctx.h, _dptr(key_values), n, key_bits, _stream(stream)),
               "b3_radix_sort32_sortdata")


class SapPairs:
    """computePairsKernel (BB/sapFast.cl:48-150) on caller-sorted device
    AABBs in btAabbCL layout (n x 8 float32: min xyz, id bits, max xyz, w)."""

    def __init__(self, ctx):
        self.ctx = ctx

    def execute(self, sorted_aabbs, pairs, count, n=None, axis=0, max_pairs=None, stream=None):
        n = sorted_aabbs.shape[0] if n is None else n
        max_pairs = pairs.shape[0] if max_pairs is None else max_pairs
        _check(self.ctx.lib.b3_sap_compute_pairs(self.ctx.h, _dptr(sorted_aabbs), n, axis, _dptr(pairs),
                                                 max_pairs, _dptr(count), _stream(stream)),
               "b3_sap_compute_pairs")


class BoundSearch:
    """btBoundSearchCL: LOWER = 0, UPPER = 1, COUNT = 2."""
    LOWER, UPPER, COUNT = 0, 1, 2

    def __init__(self, ctx):
        self.ctx = ctx

    def execute(self, sorted_keys, n_src, dst, n_dst, mode, stream=None):
        _check(self.ctx.lib.b3_bound_search(self.ctx.h, _dptr(sorted_keys), n_src, _dptr(dst), n_dst, mode,
                                            _stream(stream)), "b3_bound_search")

    def execute_sortdata(self, sorted_key_values, n_src, dst, n_dst, mode=0, stream=None):
        """execute(btOpenCLArray<btSortData>& src, nSrc, dst, nDst, option)."""
        _check(self.ctx.lib.b3_bound_search_sortdata(self.ctx.h, _dptr(sorted_key_values), n_src, _dptr(dst), n_dst,
                                                     mode, _stream(stream)), "b3_bound_search_sortdata")


# ---------------------------------------------------------------------------
# World (CLPhysicsDemo + btGpuNarrowphaseAndSolver + btGridBroadphaseCl)
# ---------------------------------------------------------------------------
def default_config(**kw):
    load()
    cfg = WorldConfig()
    _lib.b3_world_config_default(C.byref(cfg))
    for k, v in kw.items():
        if k == "gridDims":
            for i in range(3):
                cfg.gridDims[i] = int(v[i])
        elif k == "gravity":
            for i in range(3):
                cfg.gravity[i] = float(v[i])
        else:
            setattr(cfg, k, v)
    return cfg


class PhysicsWorld:
    """Rigid-body world with the reference facade's calls:
    registerConvexPolyhedron, registerPhysicsInstance, writeBodiesToGpu,
    stepSimulation, plus stage entry points and readbacks."""

    def __init__(self, ctx, cfg):
        self.ctx = ctx
        self.lib = ctx.lib
        self.cfg = cfg
        h = C.c_void_p()
        _check(self.lib.b3_world_create(ctx.h, C.byref(cfg), C.byref(h)), "b3_world_create")
        self.h = h
        self.n = 0

    # registration -------------------------------------------------------
    def registerConvexPolyhedron(self, vertices, scaling=(1.0, 1.0, 1.0)):
        v = np.ascontiguousarray(np.asarray(vertices, dtype=np.float32).reshape(-1, 3))
        s = np.asarray(scaling, dtype=np.float32)
        out = C.c_int()
        _check(self.lib.b3_register_convex_hull(self.h, fptr(v), v.shape[0], 12, fptr(s), C.byref(out)),
               "b3_register_convex_hull")
        return out.value

    def registerSphereShape(self, radius):
        out = C.c_int()
        _check(self.lib.b3_register_sphere(self.h, float(radius), C.byref(out)), "b3_register_sphere")
        return out.value

    def registerPlaneShape(self, normal, constant):
        n = np.ascontiguousarray(np.asarray(normal, np.float32).reshape(3))
        out = C.c_int()
        _check(self.lib.b3_register_plane(self.h, fptr(n), float(constant), C.byref(out)), "b3_register_plane")
        return out.value

    def registerCompoundShape(self, children):
        """children: list of (convex hull collidable, position xyz, orientation xyzw)."""
        arr = (ChildShape * len(children))()
        for k, (col, pos, orn) in enumerate(children):
            arr[k].shapeIndex = int(col)
            for i in range(3):
                arr[k].childPosition[i] = float(pos[i])
            for i in range(4):
                arr[k].childOrientation[i] = float(orn[i])
        out = C.c_int()
        _check(self.lib.b3_register_compound(self.h, arr, len(children), C.byref(out)), "b3_register_compound")
        return out.value

    def registerConcaveMesh(self, vertices, indices, scaling=(1.0, 1.0, 1.0)):
        v = np.ascontiguousarray(np.asarray(vertices, np.float32).reshape(-1, 3))
        ix = np.ascontiguousarray(np.asarray(indices, np.int32).reshape(-1))
        sc = np.ascontiguousarray(np.asarray(scaling, np.float32).reshape(3))
        out = C.c_int()
        _check(self.lib.b3_register_concave_mesh(self.h, fptr(v), v.shape[0], iptr(ix), ix.shape[0], fptr(sc),
                                                 C.byref(out)), "b3_register_concave_mesh")
        return out.value

    def child_shapes(self):
        cnt = C.c_int()
        _check(self.lib.b3_get_child_shapes(self.h, None, 0, C.byref(cnt)), "b3_get_child_shapes")
        arr = (ChildShape * max(cnt.value, 1))()
        _check(self.lib.b3_get_child_shapes(self.h, arr, cnt.value, C.byref(cnt)), "b3_get_child_shapes")
        return arr, cnt.value

    def registerPhysicsInstance(self, mass, position, orientation, collidable, friction=1.0,
                                restitution=0.0, world_id=0):
        p = np.asarray(position, dtype=np.float32)
        q = np.asarray(orientation, dtype=np.float32)
        out = C.c_int()
        _check(self.lib.b3_register_body(self.h, float(mass), fptr(p), fptr(q), int(collidable), float(friction),
                                         float(restitution), int(world_id), C.byref(out)), "b3_register_body")
        self.n = out.value + 1
        return out.value

    def register_bodies(self, mass, pos, quat, collidable, friction=None, restitution=None, world=None):
        """Bulk registerPhysicsInstance; returns the first body id."""
        n = len(mass)
        m = np.ascontiguousarray(np.asarray(mass, np.float32))
        p = np.ascontiguousarray(np.asarray(pos, np.float32).reshape(n, 3))
        q = np.ascontiguousarray(np.asarray(quat, np.float32).reshape(n, 4))
        c = np.ascontiguousarray(np.asarray(collidable, np.int32))
        f = np.ascontiguousarray(np.ones(n, np.float32) if friction is None else np.asarray(friction, np.float32))
        r = np.ascontiguousarray(np.zeros(n, np.float32) if restitution is None else np.asarray(restitution, np.float32))
        wv = np.ascontiguousarray(np.zeros(n, np.int32) if world is None else np.asarray(world, np.int32))
        out = C.c_int()
        _check(self.lib.b3_register_bodies(self.h, n, fptr(m), fptr(p), fptr(q), iptr(c), fptr(f), fptr(r),
                                           iptr(wv), C.byref(out)), "b3_register_bodies")
        self.n = out.value + n
        return out.value

    def writeBodiesToGpu(self, stream=None):
        _check(self.lib.b3_write_bodies(self.h, _stream(stream)), "b3_write_bodies")

    def write_velocities(self, lin=None, ang=None, stream=None):
        la = None if lin is None else np.ascontiguousarray(np.asarray(lin, np.float32).reshape(-1, 3))
        aa = None if ang is None else np.ascontiguousarray(np.asarray(ang, np.float32).reshape(-1, 3))
        _check(self.lib.b3_write_velocities(self.h, None if la is None else fptr(la),
                                            None if aa is None else fptr(aa), _stream(stream)),
               "b3_write_velocities")

    # stepping -----------------------------------------------------------
    def stepSimulation(self, steps=1, stream=None):
        _check(self.lib.b3_step(self.h, int(steps), _stream(stream)), "b3_step")

    def stage(self, name, stream=None):
        f = getattr(self.lib, "b3_stage_" + name)
        _check(f(self.h, _stream(stream)), "b3_stage_" + name)

    # readback -----------------------------------------------------------
    def read_state(self, stream=None, out=None):
        """(pos, quat, linVel, angVel) as (n, 4) float32 arrays; `out` gives
        the four arrays to fill (e.g. pinned host buffers)."""
        n = self.n
        if out is not None:
            pos, quat, lin, ang = out
            for a in out:
                assert a.dtype == np.float32 and a.shape == (n, 4) and a.flags["C_CONTIGUOUS"]
        else:
            pos = np.zeros((n, 4), np.float32)
            quat = np.zeros((n, 4), np.float32)
            lin = np.zeros((n, 4), np.float32)
            ang = np.zeros((n, 4), np.float32)
        _check(self.lib.b3_read_state(self.h, fptr(pos), fptr(quat), fptr(lin), fptr(ang), _stream(stream)),
               "b3_read_state")
        return pos, quat, lin, ang

    def write_state(self, pos=None, quat=None, lin=None, ang=None, stream=None):
        arrs = [None if a is None else np.ascontiguousarray(np.asarray(a, np.float32).reshape(-1, 4))
                for a in (pos, quat, lin, ang)]
        _check(self.lib.b3_write_state(self.h, *[None if a is None else fptr(a) for a in arrs],
                                       _stream(stream)), "b3_write_state")

    def read_bodies(self):
        arr = (Body * self.n)()
        _check(self.lib.b3_read_bodies(self.h, arr, self.n, None), "b3_read_bodies")
        return arr

    def counters(self):
        c = Counters()
        _check(self.lib.b3_get_counters(self.h, C.byref(c), None), "b3_get_counters")
        return c.as_dict()

    def counters_status(self):
        """(status, counters): b3_get_counters without raising on
        B3_ERR_TIMEOUT (a bounded device wait gave up)."""
        c = Counters()
        rc = self.lib.b3_get_counters(self.h, C.byref(c), None)
        if rc not in (0, 6):
            _check(rc, "b3_get_counters")
        return rc, c.as_dict()

    def set_wait_limits(self, spin_limit=0, hold_micros=0):
        _check(self.lib.b3_set_wait_limits(self.h, int(spin_limit), int(hold_micros)), "b3_set_wait_limits")

    def reset_counters(self):
        _check(self.lib.b3_reset_counters(self.h, None), "b3_reset_counters")

    def aabbs(self):
        out = np.zeros((self.n, 8), np.float32)
        _check(self.lib.b3_get_aabbs(self.h, fptr(out), self.n, None), "b3_get_aabbs")
        return out

    def sorted_hash(self):
        cnt = C.c_int()
        keys = np.zeros(self.n, np.uint32)
        vals = np.zeros(self.n, np.uint32)
        _check(self.lib.b3_get_sorted_hash(self.h, keys.ctypes.data_as(_U32P), vals.ctypes.data_as(_U32P),
                                           self.n, C.byref(cnt), None), "b3_get_sorted_hash")
        return keys[:cnt.value], vals[:cnt.value]

    def pairs(self):
        cnt = C.c_int()
        _check(self.lib.b3_get_pairs(self.h, None, 0, C.byref(cnt), None), "b3_get_pairs")
        out = np.zeros((max(cnt.value, 1), 2), np.int32)
        _check(self.lib.b3_get_pairs(self.h, iptr(out), cnt.value, C.byref(cnt), None), "b3_get_pairs")
        return out[:cnt.value]

    def contacts(self):
        cnt = C.c_int()
        _check(self.lib.b3_get_contacts(self.h, None, 0, C.byref(cnt), None), "b3_get_contacts")
        arr = (Contact4 * max(cnt.value, 1))()
        _check(self.lib.b3_get_contacts(self.h, arr, cnt.value, C.byref(cnt), None), "b3_get_contacts")
        return contacts_to_numpy(arr, cnt.value)

    def shapes(self):
        n = [C.c_int() for _ in range(6)]
        _check(self.lib.b3_get_shape_sizes(self.h, *[C.byref(x) for x in n]), "b3_get_shape_sizes")
        nc, npo, nv, nf, ni, ne = [x.value for x in n]
        cols = (Collidable * max(nc, 1))()
        polys = (ConvexPolyhedron * max(npo, 1))()
        verts = np.zeros((max(nv, 1), 4), np.float32)
        faces = (Face * max(nf, 1))()
        idx = np.zeros(max(ni, 1), np.int32)
        edges = np.zeros((max(ne, 1), 4), np.float32)
        laabb = np.zeros((max(nc, 1), 8), np.float32)
        _check(self.lib.b3_get_shapes(self.h, cols, polys, fptr(verts), faces, iptr(idx), fptr(edges),
                                      fptr(laabb)), "b3_get_shapes")
        return dict(cols=cols, polys=polys, verts=verts[:nv], faces=faces, idx=idx[:ni], edges=edges[:ne],
                    localAabb=laabb[:nc], counts=(nc, npo, nv, nf, ni, ne))

    def inertias(self):
        arr = (Inertia * self.n)()
        _check(self.lib.b3_get_inertias(self.h, arr, self.n), "b3_get_inertias")
        return np.array([[a.initInvInertia[0], a.initInvInertia[5], a.initInvInertia[10], 0.0] for a in arr],
                        np.float32).reshape(-1, 4)

    def autotune(self, trial_steps=3, stream=None):
        """b3_autotune: time the candidate launch shapes on the current scene
        and keep the fastest; the body state is left as it was."""
        _check(self.lib.b3_autotune(self.h, int(trial_steps), _stream(stream)), "b3_autotune")

    def tuning(self):
        """(narrowphase warps/CTA, pair CTA size, solver CTA size, kernels per
        captured step, Jacobi blocks per SM cap, configurations timed,
        Jacobi mode, Jacobi gather, grid pair search form, narrowphase lane groups)."""
        v = (C.c_int * 10)()
        cnt = C.c_int()
        _check(self.lib.b3_get_tuning(self.h, v, 10, C.byref(cnt)), "b3_get_tuning")
        return list(v)[:cnt.value]

    def set_tuning(self, values):
        v = (C.c_int * len(values))(*[int(x) for x in values])
        _check(self.lib.b3_set_tuning(self.h, v, len(values)), "b3_set_tuning")

    def set_stage_timing(self, on=True):
        _check(self.lib.b3_set_stage_timing(self.h, 1 if on else 0), "b3_set_stage_timing")

    def stage_times(self):
        ms = np.zeros(16, np.float32)
        cnt = C.c_int()
        _check(self.lib.b3_get_stage_times(self.h, fptr(ms), 16, C.byref(cnt)), "b3_get_stage_times")
        return ms[:cnt.value].tolist()

    def world_stats(self, num_worlds):
        out = np.zeros((num_worlds, 4), np.float32)
        _check(self.lib.b3_batch_world_stats(self.h, fptr(out), num_worlds, None), "b3_batch_world_stats")
        return out

    def world_offsets(self):
        """Body-count prefix sums per world (numWorlds + 1 entries)."""
        nw = C.c_int()
        _check(self.lib.b3_batch_world_offsets(self.h, None, 0, C.byref(nw)), "b3_batch_world_offsets")
        out = np.zeros(nw.value + 1, np.int32)
        _check(self.lib.b3_batch_world_offsets(self.h, iptr(out), len(out), C.byref(nw)), "b3_batch_world_offsets")
        return out

    def sap_calculate_overlapping_pairs(self, stream=None):
        """btGpuSapBroadphase::calculateOverlappingPairs on a world created
        with flags=B3_WORLD_SAP_BROADPHASE (from the current AABBs)."""
        _check(self.lib.b3_sap_broadphase_calculate_overlapping_pairs(self.h, _stream(stream)),
               "b3_sap_broadphase_calculate_overlapping_pairs")

    def load_bullet_file(self, path, keep_static_objects=False, spheres_and_planes=False):
        """btBulletDataExtractor::convertAllObjects on a .bullet scene file:
        registers its box and convex-hull shapes and its rigid bodies (see
        b3_load_bullet_file); with spheres_and_planes also its sphere and
        static plane shapes (b3_load_bullet_file_ex,
        B3_BULLET_SPHERES_AND_PLANES). Returns the number of bodies added."""
        n = C.c_int()
        if spheres_and_planes:
            flags = BULLET_SPHERES_AND_PLANES | (BULLET_KEEP_STATIC_OBJECTS if keep_static_objects else 0)
            _check(self.lib.b3_load_bullet_file_ex(self.h, os.fsencode(path), flags, C.byref(n)),
                   "b3_load_bullet_file_ex")
        else:
            _check(self.lib.b3_load_bullet_file(self.h, os.fsencode(path), 1 if keep_static_objects else 0,
                                                C.byref(n)), "b3_load_bullet_file")
        total = C.c_int()
        _check(self.lib.b3_get_num_bodies(self.h, C.byref(total)), "b3_get_num_bodies")
        self.n = total.value
        return n.value

    def solve_batched_gs(self, stream=None):
        """Solver::batchContacts + convertToConstraints + solveContactConstraint
        on a world created with flags=B3_WORLD_BATCHED_GS_SOLVER."""
        _check(self.lib.b3_solver_solve_batched_gs(self.h, _stream(stream)), "b3_solver_solve_batched_gs")

    def gs_batches(self):
        """(cell, batch) per manifold from the last batched Gauss-Seidel solve (M x 2)."""
        cnt = C.c_int()
        _check(self.lib.b3_get_gs_batches(self.h, None, 0, C.byref(cnt), None), "b3_get_gs_batches")
        out = np.zeros((max(cnt.value, 1), 2), np.int32)
        _check(self.lib.b3_get_gs_batches(self.h, iptr(out), cnt.value, C.byref(cnt), None), "b3_get_gs_batches")
        return out[:cnt.value]

    def gs_constraints(self):
        """Constraint4 per manifold after the last batched Gauss-Seidel solve:
        dict of arrays (applied impulses included)."""
        cnt = C.c_int()
        _check(self.lib.b3_get_gs_constraints(self.h, None, 0, C.byref(cnt), None), "b3_get_gs_constraints")
        n = cnt.value
        arr = (Constraint4 * max(n, 1))()
        _check(self.lib.b3_get_gs_constraints(self.h, arr, n, C.byref(cnt), None), "b3_get_gs_constraints")
        raw = np.frombuffer(arr, np.float32).reshape(-1, 44)[:n]
        ints = raw.view(np.int32)
        return dict(linear=raw[:, 0:4], worldPos=raw[:, 4:20].reshape(-1, 4, 4), center=raw[:, 20:24],
                    jacCoeffInv=raw[:, 24:28], b=raw[:, 28:32], applied=raw[:, 32:36], fJacCoeffInv=raw[:, 36:38],
                    fApplied=raw[:, 38:40], bodyA=ints[:, 40], bodyB=ints[:, 41], batchIdx=ints[:, 42])

    def compute_contacts(self, d_pairs=None, num_pairs=0, stream=None):
        """Narrowphase on caller device pairs (int2) or, with None, on the
        world's own broadphase pairs."""
        _check(self.lib.b3_narrowphase_compute_contacts(self.h, d_pairs, num_pairs, stream),
               "b3_narrowphase_compute_contacts")

    def device_buffer(self, which):
        p = C.c_void_p()
        nb = C.c_int64()
        _check(self.lib.b3_get_device_buffer(self.h, BUF[which], C.byref(p), C.byref(nb)),
               "b3_get_device_buffer")
        return p.value, nb.value

    def close(self):
        if self.h:
            self.lib.b3_world_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Adjoint:
    """Reverse-mode gradients of a loss of the final state with respect to
    the initial velocities, masses and friction coefficients
    (b3_adjoint_*): forward() runs num_steps steps with checkpoints every
    checkpoint_every steps, backward(seeds) runs the reverse sweep."""

    def __init__(self, world, num_steps, checkpoint_every):
        self.world = world
        self.lib = world.lib
        h = _P()
        _check(self.lib.b3_adjoint_create(world.h, int(num_steps), int(checkpoint_every), C.byref(h)),
               "b3_adjoint_create")
        self.h = h

    def forward(self, stream=None):
        _check(self.lib.b3_adjoint_forward(self.h, _stream(stream)), "b3_adjoint_forward")

    def backward(self, d_pos=None, d_quat=None, d_lin=None, d_ang=None, stream=None):
        n = self.world.n

        def arr(x):
            if x is None:
                return None
            a = np.zeros((n, 4), np.float32)
            x = np.asarray(x, np.float32).reshape(n, -1)
            a[:, :x.shape[1]] = x
            return a

        keep = [arr(x) for x in (d_pos, d_quat, d_lin, d_ang)]
        ptrs = [fptr(a) if a is not None else None for a in keep]
        _check(self.lib.b3_adjoint_backward(self.h, *ptrs, _stream(stream)), "b3_adjoint_backward")

    def gradients(self):
        n = self.world.n
        gl = np.zeros((n, 4), np.float32)
        ga = np.zeros((n, 4), np.float32)
        gm = np.zeros(n, np.float32)
        gf = np.zeros(n, np.float32)
        _check(self.lib.b3_adjoint_gradients(self.h, fptr(gl), fptr(ga), fptr(gm), fptr(gf)), "b3_adjoint_gradients")
        return dict(lin=gl[:, :3], ang=ga[:, :3], mass=gm, friction=gf)

    def unclassified(self):
        v = C.c_int()
        _check(self.lib.b3_adjoint_info(self.h, C.byref(v)), "b3_adjoint_info")
        return v.value

    def close(self):
        if self.h:
            self.lib.b3_adjoint_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def contacts_to_numpy(arr, n):
    """Contact4 array -> dict of numpy arrays (pos (n,4,4), normal (n,4), ...)."""
    raw = np.frombuffer(C.string_at(C.addressof(arr), 96 * max(n, 0)), dtype=np.uint8).reshape(-1, 96) \
        if n > 0 else np.zeros((0, 96), np.uint8)
    f = raw.view(np.float32).reshape(-1, 24)
    i = raw.view(np.int32).reshape(-1, 24)
    return dict(pos=f[:, :16].reshape(-1, 4, 4).copy(), normal=f[:, 16:20].copy(), friction=f[:, 20].copy(),
                pairIndex=i[:, 21].copy(), bodyA=i[:, 22].copy(), bodyB=i[:, 23].copy())
