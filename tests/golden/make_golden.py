"""Generate the golden fixtures under tests/golden/ from the reference tree
(run here, where /root/reference exists; the fixtures are committed so the
tests need no reference at run time).

clip_faces_k11.npz
    The reference's own recorded test vector for the clipping kernel:
    testdata/clipFacesAndContactReductionKernel.7z holds the argument dump of
    clipFacesAndContactReductionKernel (satClipHullContacts.cl:1845-1952)
    before and after one launch, in the btLauncherCL serialisation
    (BB/btLauncherCL.h:216-273: int nArgs, then per argument {isBuffer,
    argIndex, sizeBytes, 16-byte value} followed by the buffer's bytes, then
    int numWorkItems), the format the reference's own test
    (opencl/tests/main.cpp:249-334) replays. Per pair with a separating
    axis: the reference face's world vertices and normal, the incident
    polygon, and the kernel's output points and count.

jacobi_pins.npz
    Outputs of the reference's btPgsJacobiSolver::solveContacts
    (P2/btPgsJacobiSolver.cpp:171-189), compiled from the reference sources
    into oracle/_ref/libb3ref.so, on the manifolds of three settled piles
    (random_pile seeds 21-23, 40 bodies, 40 oracle steps): the Body /
    Inertia / Contact4 arrays it was given and the velocities it returned.

sap_kernel_args.npz
    The reference's recorded arguments of its sweep-and-prune pair kernel:
    testdata/m_sapKernelArgs.zip holds m_sapKernelArgs.bin, the btLauncherCL
    dump of computePairsKernel (BB/sapFast.cl:48-150) taken before a launch
    (P2/btGpuSapBroadphase.cpp:349-371), the file opencl/tests/main.cpp:
    110-190 replays: the sorted AABB array (btAabbCL records), the pair and
    count buffers, numObjects, axis and maxPairs. The fixture keeps the
    sorted AABBs and the scalars (the output buffers were not yet written).

gs_solve_args.npz
    The reference's recorded arguments of its batched Gauss-Seidel solve
    kernel: testdata/m_batchSolveKernel.7z holds m_batchSolveKernel.bin, the
    btLauncherCL dump of one BatchSolveKernelContact launch
    (ST/solveContact.cl:400-476; ST/Solver.cpp:561-640 sets its arguments):
    the Body array (96-byte records of that revision: position, orientation,
    linear and angular velocity, then inverse mass at float 18), the Shape
    array (world and local inverse inertia), the Constraint4 array (176
    bytes, ST/AdlConstraint4.h:23-47) as ContactToConstraintKernel
    (ST/solverSetup.cl:614-655) and the batching kernel left it, and the
    per-cell counts and offsets of the 16 x 16 grid; maxBatch, the parity
    class and N_SPLIT. The fixture keeps the used constraints, the bodies'
    positions, inverse masses and world inverse inertias, and the grid.

pile.bullet, pile_bullet.npz
    A .bullet scene file written by the reference's own serializer: a seeded
    pile (random_pile seed 61, 40 bodies: unit cubes, which the reference
    CPU pipeline builds as btBoxShape, and 12-point hulls as
    btConvexHullShape) on a static ground box, put into bullet2's
    btDiscreteDynamicsWorld (oracle/_ref/libb3bullet.so, compiled from the
    reference's bullet2 sources) and written by btDefaultSerializer. The npz
    keeps the scene it was made from (positions, orientations, masses,
    shape of each body and the shapes' points).

spheres.bullet, spheres_bullet.npz
    The same writer on 24 spheres (spheres_on_plane seed 84: radii
    U(0.2, 0.5), btSphereShape) above a static plane y = 0
    (btStaticPlaneShape); the npz keeps each body's position, orientation,
    mass and radius and the plane.

hull_pins.npz
    btConvexUtility::initializePolyhedralFeatures
    (P1/btConvexUtility.cpp:31-270) on every distinct shape of the plain and
    batched workloads: vertices, face planes, face vertex cycles and unique
    edges.

The .7z container is read by the small reader below: one LZMA folder,
LZMA-coded header (the layout both files in testdata/ use); Python's lzma
module decodes the raw LZMA1 streams.

Usage: python tests/golden/make_golden.py
"""
import lzma
import os
import struct

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference tree; B3_REFERENCE_ROOT overrides the default location
REFERENCE = os.environ.get("B3_REFERENCE_ROOT", "/root/reference")


def _num(b, i):
    """7z variable-length number."""
    first = b[i]
    i += 1
    mask = 0x80
    val = 0
    for k in range(8):
        if first & mask == 0:
            return val | ((first & (mask - 1)) << (8 * k)), i
        val |= b[i] << (8 * k)
        i += 1
        mask >>= 1
    return val, i


def _lzma1(data, props, size):
    lc = props[0] % 9
    lp = (props[0] // 9) % 5
    pb = props[0] // 45
    dict_size = struct.unpack("<I", props[1:5])[0]
    dec = lzma.LZMADecompressor(format=lzma.FORMAT_RAW,
                                filters=[{"id": lzma.FILTER_LZMA1, "dict_size": dict_size, "lc": lc, "lp": lp,
                                          "pb": pb}])
    out = dec.decompress(data, max_length=size)
    if len(out) != size:
        raise ValueError("short LZMA stream")
    return out


def _streams_info(h, i):
    """PackInfo + one-folder LZMA UnpackInfo (+ SubStreamsInfo sizes)."""
    info = {}
    while True:
        t = h[i]
        i += 1
        if t == 0x00:
            return info, i
        if t == 0x06:  # PackInfo
            info["packPos"], i = _num(h, i)
            n, i = _num(h, i)
            assert n == 1
            assert h[i] == 0x09
            info["packSize"], i = _num(h, i + 1)
            while h[i] != 0x00:  # skip CRCs if present
                i += 1
            i += 1
        elif t == 0x07:  # UnpackInfo
            assert h[i] == 0x0B
            nf, i = _num(h, i + 1)
            assert nf == 1 and h[i] == 0x00
            i += 1
            nc, i = _num(h, i)
            assert nc == 1
            flags = h[i]
            i += 1
            idsize = flags & 0x0F
            codec = h[i:i + idsize]
            i += idsize
            assert codec == b"\x03\x01\x01", "only LZMA folders"
            if flags & 0x20:
                psz, i = _num(h, i)
                info["props"] = h[i:i + psz]
                i += psz
            assert h[i] == 0x0C
            info["unpackSize"], i = _num(h, i + 1)
            if h[i] == 0x0A:  # folder CRC
                i += 1 + 1 + 4
            assert h[i] == 0x00
            i += 1
        elif t == 0x08:  # SubStreamsInfo
            sizes = []
            if h[i] == 0x0D:
                nstreams, i = _num(h, i + 1)
            else:
                nstreams = 1
            if h[i] == 0x09:
                i += 1
                for _ in range(nstreams - 1):
                    v, i = _num(h, i)
                    sizes.append(v)
            info["subsizes"] = sizes
            while h[i] != 0x00:  # CRC digests
                if h[i] == 0x0A:
                    i += 1
                    alldef = h[i]
                    i += 1
                    assert alldef == 1
                    i += 4 * nstreams
                else:
                    break
            assert h[i] == 0x00
            i += 1
        else:
            raise ValueError(f"unsupported 7z property {t:#x}")


def read_7z(path):
    """{file name: bytes} of a single-folder LZMA 7z archive."""
    d = open(path, "rb").read()
    assert d[:6] == b"7z\xbc\xaf\x27\x1c"
    off, size = struct.unpack("<QQ", d[12:28])
    h = d[32 + off:32 + off + size]
    if h[0] == 0x17:  # encoded header
        info, _ = _streams_info(h, 1)
        h = _lzma1(d[32 + info["packPos"]:32 + info["packPos"] + info["packSize"]], info["props"],
                   info["unpackSize"])
    assert h[0] == 0x01 and h[1] == 0x04  # Header, MainStreamsInfo
    info, i = _streams_info(h, 2)
    data = _lzma1(d[32 + info["packPos"]:32 + info["packPos"] + info["packSize"]], info["props"],
                  info["unpackSize"])
    sizes = info.get("subsizes", [])
    sizes = sizes + [len(data) - sum(sizes)]
    # FilesInfo: names (UTF-16LE, NUL-terminated)
    names = []
    j = h.index(b"\x11", i)
    ln, j = _num(h, j + 1)
    assert h[j] == 0x00
    raw = h[j + 1:j + ln].decode("utf-16-le")
    names = [x for x in raw.split("\x00") if x]
    out, p = {}, 0
    for name, sz in zip(names, sizes):
        out[name] = data[p:p + sz]
        p += sz
    return out


def launcher_args(blob):
    """btLauncherCL argument dump -> (list of (isBuffer, bytes or 16-byte value), numWorkItems)."""
    nargs = struct.unpack("<i", blob[:4])[0]
    p = 4
    args = []
    for _ in range(nargs):
        is_buf, idx, sz = struct.unpack("<iii", blob[p:p + 12])
        val = blob[p + 12:p + 28]
        p += 28
        if is_buf:
            args.append((True, blob[p:p + sz]))
            p += sz
        else:
            args.append((False, val))
    work = struct.unpack("<i", blob[p:p + 4])[0]
    return args, work


def make_clip_faces():
    files = read_7z(os.path.join(REFERENCE, "testdata", "clipFacesAndContactReductionKernel.7z"))
    before_name = [k for k in files if k.endswith("_before.bin")][0]
    after_name = [k for k in files if k.endswith("_after.bin")][0]
    before, work = launcher_args(files[before_name])
    after, _ = launcher_args(files[after_name])
    f4 = lambda b: np.frombuffer(b, np.float32).reshape(-1, 4)
    i4 = lambda b: np.frombuffer(b, np.int32)
    cap = struct.unpack("<i", before[11][1][:4])[0]
    num_pairs = struct.unpack("<i", before[12][1][:4])[0]
    has_sep = i4(before[3][1])
    faces_b = i4(before[5][1]).reshape(-1, 4)
    faces_a = i4(after[5][1]).reshape(-1, 4)
    vA = f4(before[6][1]).reshape(-1, cap, 4)
    nA = f4(before[7][1])
    vB1 = f4(before[8][1]).reshape(-1, cap, 4)
    out1 = f4(after[8][1]).reshape(-1, cap, 4)
    out2 = f4(after[9][1]).reshape(-1, cap, 4)
    keep = [p for p in range(num_pairs) if has_sep[p] and faces_b[p, 0] >= 0]
    rec = dict(pairs=np.array(keep, np.int32), cap=np.int32(cap), numPairs=np.int32(num_pairs),
               numWorkItems=np.int32(work))
    nAv = faces_b[keep, 2]
    nBv = faces_b[keep, 3]
    rec["numVertsA"] = nAv.astype(np.int32)
    rec["numVertsB"] = nBv.astype(np.int32)
    rec["numOut"] = faces_a[keep, 3].astype(np.int32)
    mA, mB = int(nAv.max()), int(nBv.max())
    rec["vertsA"] = vA[keep, :mA].astype(np.float32)
    rec["normalA"] = nA[keep].astype(np.float32)
    rec["polyB"] = vB1[keep, :mB].astype(np.float32)
    # the depth-filtered points are written through pVtxOut, which after the
    # side planes' swaps names worldVertsB2 for an even number of planes and
    # worldVertsB1 for an odd one
    mO = max(int(faces_a[keep, 3].max()), 1)
    outs = np.where((nAv % 2 == 0)[:, None, None], out2[keep, :mO], out1[keep, :mO])
    rec["points"] = outs.astype(np.float32)
    np.savez_compressed(os.path.join(HERE, "clip_faces_k11.npz"), **rec)
    return rec


def _import_tests():
    import sys
    root = os.path.dirname(os.path.dirname(HERE))
    for p in (root, os.path.join(root, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)


def make_jacobi():
    _import_tests()
    import ctypes as C
    import oracle
    from experiments_b200 import b3, scenes
    from helpers import host_oracle
    ref = oracle.ref_lib()
    hc = b3.Context(-1)
    rec = {}
    for seed in (21, 22, 23):
        sc = scenes.random_pile(seed, n=40, velocity=0.5)
        w, o = host_oracle(hc, sc)
        o.step(40)
        o.stage("aabbs")
        o.stage("broadphase")
        o.stage("narrowphase")
        cts = o.contacts()
        m = len(cts["normal"])
        q = np.round(np.clip(cts["friction"], 0, 1) * 65535.0)
        pos, quat, lin, ang = [a.astype(np.float32) for a in o.state()]
        mass = np.asarray(sc.mass, np.float64)
        body = np.zeros(sc.n, dtype=np.dtype([("pos", "<f4", 4), ("quat", "<f4", 4), ("lin", "<f4", 4),
                                               ("ang", "<f4", 4), ("shape", "<u4"), ("invMass", "<f4"),
                                               ("rest", "<f4"), ("fric", "<f4")]))
        body["pos"], body["quat"], body["lin"], body["ang"] = pos, quat, lin, ang
        body["invMass"] = np.where(mass != 0, 1.0 / np.where(mass != 0, mass, 1), 0)
        body["fric"] = sc.friction
        ii = w.inertias()
        inert = np.zeros((sc.n, 24), np.float32)
        for k in range(3):
            inert[:, k * 4 + k] = ii[:, k]
            inert[:, 12 + k * 4 + k] = ii[:, k]
        c4 = np.zeros(m, dtype=np.dtype([("pos", "<f4", (4, 4)), ("nrm", "<f4", 4), ("rest", "<u2"),
                                          ("fric", "<u2"), ("batch", "<i4"), ("a", "<i4"), ("b", "<i4")]))
        c4["pos"] = cts["pos"]
        c4["nrm"] = cts["normal"]
        c4["fric"] = q.astype(np.uint16)
        c4["a"] = np.abs(cts["bodyA"])
        c4["b"] = np.abs(cts["bodyB"])
        given = body.copy()
        assert ref.ref_jacobi_solve(sc.n, body.ctypes.data, inert.ctypes.data, m, c4.ctypes.data) == 0
        rec[f"s{seed}_body"] = given.view(np.uint8)
        rec[f"s{seed}_inertia"] = inert
        rec[f"s{seed}_contacts"] = c4.view(np.uint8)
        rec[f"s{seed}_bodyA"] = cts["bodyA"].astype(np.int32)
        rec[f"s{seed}_bodyB"] = cts["bodyB"].astype(np.int32)
        rec[f"s{seed}_lin"] = body["lin"].copy()
        rec[f"s{seed}_ang"] = body["ang"].copy()
        w.close()
        o.close()
    np.savez_compressed(os.path.join(HERE, "jacobi_pins.npz"), **rec)
    return rec


def make_sap():
    import zipfile
    blob = zipfile.ZipFile(os.path.join(REFERENCE, "testdata", "m_sapKernelArgs.zip")).read("m_sapKernelArgs.bin")
    args, work = launcher_args(blob)
    scalar = lambda k: struct.unpack("<i", args[k][1][:4])[0]
    aabbs = np.frombuffer(args[0][1], np.float32).reshape(-1, 8).copy()
    rec = dict(sorted_aabbs=aabbs, numObjects=np.int32(scalar(3)), axis=np.int32(scalar(4)),
               maxPairs=np.int32(scalar(5)), numWorkItems=np.int32(work))
    np.savez_compressed(os.path.join(HERE, "sap_kernel_args.npz"), **rec)
    return rec


def make_gs():
    files = read_7z(os.path.join(REFERENCE, "testdata", "m_batchSolveKernel.7z"))
    args, work = launcher_args(files["m_batchSolveKernel.bin"])
    scalar = lambda k: struct.unpack("<i", args[k][1][:4])[0]
    gN = np.frombuffer(args[3][1], np.int32).copy()
    gO = np.frombuffer(args[4][1], np.int32).copy()
    n = int(gN.sum())
    cf = np.frombuffer(args[2][1], np.float32)[:44 * n].reshape(n, 44)
    ci = np.frombuffer(args[2][1], np.int32)[:44 * n].reshape(n, 44)
    bodies = np.frombuffer(args[0][1], np.float32).reshape(-1, 24)
    shapes = np.frombuffer(args[1][1], np.float32).reshape(-1, 24)
    used = np.unique(ci[:, 40:42])
    rec = dict(cellCount=gN, cellOffset=gO, numWorkItems=np.int32(work), maxBatch=np.int32(scalar(6)),
               classIdx=np.int32(scalar(7)), nSplit=np.int32(scalar(8)),
               linear=cf[:, 0:4].copy(), worldPos=cf[:, 4:20].reshape(n, 4, 4).copy(), center=cf[:, 20:24].copy(),
               jacCoeffInv=cf[:, 24:28].copy(), b=cf[:, 28:32].copy(), applied=cf[:, 32:36].copy(),
               fJacCoeffInv=cf[:, 36:38].copy(), fApplied=cf[:, 38:40].copy(), bodyAB=ci[:, 40:42].copy(),
               batchIdx=ci[:, 42].copy(), bodies=used.astype(np.int32),
               bodyPos=bodies[used, 0:4].copy(), bodyLinVel=bodies[used, 8:12].copy(),
               bodyAngVel=bodies[used, 12:16].copy(), bodyInvMass=bodies[used, 18].copy(),
               bodyInvInertiaWorld=shapes[used, 0:12].reshape(-1, 3, 4)[:, :, :3].copy())
    np.savez_compressed(os.path.join(HERE, "gs_solve_args.npz"), **rec)
    return rec


def make_bullet_scene():
    _import_tests()
    import oracle
    from experiments_b200 import scenes
    sc = scenes.random_pile(61, n=40, hull_frac=0.5, pool=4)
    ref = oracle.ReferenceCpuWorld(sc)
    ref.write_bullet(os.path.join(HERE, "pile.bullet"))
    ref.close()
    pts = [np.asarray(v, np.float32).reshape(-1, 3) for v in sc.shapes]
    offs = np.concatenate([[0], np.cumsum([len(p) for p in pts])]).astype(np.int32)
    rec = dict(pos=np.asarray(sc.pos, np.float32), quat=np.asarray(sc.quat, np.float32),
               mass=np.asarray(sc.mass, np.float32), shape=np.asarray(sc.shape, np.int32),
               points=np.concatenate(pts).astype(np.float32), shapeOffsets=offs)
    np.savez_compressed(os.path.join(HERE, "pile_bullet.npz"), **rec)
    return sc.n


def make_bullet_spheres():
    """spheres.bullet: 24 spheres on a static plane written by the
    reference's serializer (btSphereShape, btStaticPlaneShape)."""
    _import_tests()
    import oracle
    from experiments_b200 import scenes
    sc = scenes.spheres_on_plane(84, n=24)
    ref = oracle.ReferenceCpuWorld(sc)
    ref.write_bullet(os.path.join(HERE, "spheres.bullet"))
    ref.close()
    radius = np.array([sc.shapes[k]["radius"] if sc.shapes[k]["kind"] == "sphere" else 0.0 for k in sc.shape],
                      np.float32)
    rec = dict(pos=np.asarray(sc.pos, np.float32), quat=np.asarray(sc.quat, np.float32),
               mass=np.asarray(sc.mass, np.float32), shape=np.asarray(sc.shape, np.int32), radius=radius,
               plane=np.array(list(sc.shapes[0]["normal"]) + [sc.shapes[0]["constant"]], np.float32))
    np.savez_compressed(os.path.join(HERE, "spheres_bullet.npz"), **rec)
    return sc.n


def make_hulls():
    _import_tests()
    import test_cpu_pins as pins
    from experiments_b200 import scenes
    rec = {}
    k = 0
    for sc in (scenes.c2(dims=(4, 2, 4)), scenes.c3(worlds=4)):
        for pts in sc.shapes:
            v, p, faces, e = pins.ref_hull(pts)
            rec[f"h{k}_points"] = np.asarray(pts, np.float32)
            rec[f"h{k}_verts"] = v
            rec[f"h{k}_planes"] = p
            rec[f"h{k}_faces"] = np.concatenate([[len(f)] + list(f) for f in faces]).astype(np.int32)
            rec[f"h{k}_edges"] = e
            k += 1
    rec["count"] = np.int32(k)
    np.savez_compressed(os.path.join(HERE, "hull_pins.npz"), **rec)
    return k


if __name__ == "__main__":
    r = make_clip_faces()
    print("clip_faces_k11.npz:", len(r["pairs"]), "pairs with a clip, of", int(r["numPairs"]))
    r = make_jacobi()
    print("jacobi_pins.npz:", len(r) // 7, "piles")
    print("hull_pins.npz:", make_hulls(), "shapes")
    r = make_sap()
    print("sap_kernel_args.npz:", int(r["numObjects"]), "sorted AABBs")
    r = make_gs()
    print("gs_solve_args.npz:", len(r["batchIdx"]), "constraints")
    print("pile.bullet:", make_bullet_scene(), "bodies")
    print("spheres.bullet:", make_bullet_spheres(), "bodies")
