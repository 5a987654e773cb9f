"""Spheres, planes, compounds and triangle meshes (the reference's
non-hull collision paths): registration tables, and the oracle's contacts
pinned by known answers.

The reference ships no recorded data for these paths, so its restatement is
pinned analytically: a sphere on a plane and two spheres against the closed
forms of computeContactPlaneConvex and the sphere-sphere branch of
clipHullHullKernel (P2/satClipHullContacts.cl:957-1124); a compound against
its children registered as separate bodies at the same poses (a compound
pair is its child pairs, P2/sat.cl:639-926, P2/satClipHullContacts.cl:
1184-1318); a mesh's triangle against the plane a cube rests on
(findSeparatingAxisKernel's triangle polytope, P2/sat.cl:970-1191)."""
import numpy as np
import pytest

import oracle
from experiments_b200 import b3, scenes

from helpers import host_oracle

CUBE = scenes.box_vertices(0.5, 0.5, 0.5)
GROUND = scenes.box_vertices(20.0, 0.5, 20.0)
Q0 = [0.0, 0.0, 0.0, 1.0]


def scene_of(shapes, bodies, cell=1.0, dims=(32, 32, 32)):
    """bodies: (shape index, mass, position, orientation)."""
    sh = [b[0] for b in bodies]
    b = scenes._bodies(sh, [x[1] for x in bodies], [x[2] for x in bodies], [x[3] for x in bodies],
                       [0.6] * len(bodies), [0] * len(bodies))
    return scenes.Scene(name="shapes", shapes=shapes, num_worlds=1,
                        config=dict(cellSize=cell, gridDims=dims), steps=1, **b)


def contacts_of(host_ctx, sc):
    w, o = host_oracle(host_ctx, sc)
    for s in ("aabbs", "broadphase", "narrowphase"):
        o.stage(s)
    return w, o, o.contacts()


def test_registration_tables(host_ctx):
    w = b3.PhysicsWorld(host_ctx, b3.default_config(maxBodies=8))
    cube = w.registerConvexPolyhedron(CUBE)
    sph = w.registerSphereShape(0.25)
    pl = w.registerPlaneShape([0, 1, 0], 0.5)
    comp = w.registerCompoundShape([(cube, (0.6, 0, 0), Q0), (cube, (-0.6, 0, 0), Q0)])
    tri = np.array([[0, 0, 0], [2, 0, 0], [0, 0, -2], [2, 0, -2]], np.float32)
    mesh = w.registerConcaveMesh(tri, [0, 1, 2, 2, 1, 3], scaling=(1, 1, 1))
    sh = w.shapes()
    cols = sh["cols"]
    assert [cols[k].shapeType for k in (cube, sph, pl, comp, mesh)] == [3, 7, 4, 6, 5]
    assert cols[sph].radius == 0.25
    f = sh["faces"][cols[pl].shapeIndex]
    assert list(f.plane) == [0.0, 1.0, 0.0, 0.5] and cols[pl].radius == 0.5
    ch, n = w.child_shapes()
    assert n == 2 and cols[comp].numChildShapes == 2 and cols[comp].shapeIndex == 0
    assert ch[0].shapeIndex == cube and abs(ch[0].childPosition[0] - 0.6) < 1e-7
    # compound local AABB: the union of the two cubes
    la = sh["localAabb"][comp]
    assert np.allclose(la[:3], [-1.1, -0.5, -0.5], atol=1e-6) and np.allclose(la[4:7], [1.1, 0.5, 0.5], atol=1e-6)
    # mesh: its own entry (a face per triangle), then one polytope per triangle
    mp = sh["polys"][cols[mesh].shapeIndex]
    assert mp.numFaces == 2 and cols[mesh].numChildShapes == 2 and mp.unused == cols[mesh].shapeIndex + 1
    for t in range(2):
        tp = sh["polys"][mp.unused + t]
        assert tp.numVertices == 3 and tp.numFaces == 5 and tp.numUniqueEdges == 3
        fr = sh["faces"][tp.faceOffset]
        bk = sh["faces"][tp.faceOffset + 1]
        # the triangles' normal is +y (CCW seen from above), the back face -y
        assert np.allclose(list(fr.plane)[:3], [0, 1, 0], atol=1e-7)
        assert np.allclose(list(bk.plane)[:3], [0, -1, 0], atol=1e-7)
        # edge planes: unit normals in the triangle's plane, outward
        v = sh["verts"][tp.vertexOffset:tp.vertexOffset + 3, :3]
        c = v.mean(0)
        for e in range(3):
            pe = np.array(list(sh["faces"][tp.faceOffset + 2 + e].plane))
            assert abs(np.linalg.norm(pe[:3]) - 1) < 1e-6 and abs(pe[1]) < 1e-7
            assert pe[:3] @ c + pe[3] < 0  # the centre is inside
    w.close()


@pytest.mark.parametrize("h", [0.24, 0.2, 0.26])
def test_sphere_on_plane_known_answer(host_ctx, h):
    r = 0.25
    sc = scene_of([{"kind": "plane", "normal": [0, 1, 0], "constant": 0.0}, {"kind": "sphere", "radius": r}],
                  [(0, 0.0, (0, 0, 0), Q0), (1, 1.0, (0.3, h, -0.2), Q0)])
    w, o, c = contacts_of(host_ctx, sc)
    if h - r >= 0:
        assert len(c["normal"]) == 0  # computeContactPlaneConvex: a contact below the plane only
    else:
        assert len(c["normal"]) == 1
        assert int(c["normal"][0][3]) == 1 and np.allclose(c["normal"][0][:3], [0, 1, 0])
        assert np.allclose(c["pos"][0][0][:3], [0.3, h - r, -0.2], atol=1e-12)
        assert abs(c["pos"][0][0][3] - (np.float32(h) - r)) < 1e-7
        assert abs(c["bodyA"][0]) == 0 and c["bodyB"][0] == 1  # the plane's body is side A
    w.close()


def test_sphere_sphere_known_answer(host_ctx):
    sc = scene_of([GROUND, {"kind": "sphere", "radius": 0.5}, {"kind": "sphere", "radius": 0.3}],
                  [(0, 0.0, (0, -30, 0), Q0), (1, 1.0, (0, 5, 0), Q0), (2, 1.0, (0.6, 5.2, 0.1), Q0)])
    w, o, c = contacts_of(host_ctx, sc)
    assert len(c["normal"]) == 1
    A, B = c["bodyA"][0], c["bodyB"][0]
    pA, pB = np.asarray(sc.pos[A], np.float64), np.asarray(sc.pos[B], np.float64)
    rA, rB = (0.5, float(np.float32(0.3))) if A == 1 else (float(np.float32(0.3)), 0.5)
    d = pA - pB
    L = np.linalg.norm(d)
    nB = d / L
    assert np.allclose(c["normal"][0][:3], -nB, atol=1e-12)  # from A to B
    assert np.allclose(c["pos"][0][0][:3], pB + nB * rB, atol=1e-12)
    assert abs(c["pos"][0][0][3] - (L - rA - rB)) < 1e-12
    w.close()


def test_compound_is_its_children(host_ctx):
    """A compound of two cubes resting tilted on the ground gives the two
    manifolds the same cubes give as separate bodies at the children's
    poses (the composed poses are FP32, as the device computes them)."""
    yaw = scenes.yaw_quat(np.array([0.3]))[0]
    tilt = np.array([np.sin(0.02), 0, 0, np.cos(0.02)])
    cp = [(0.7, 0.0, 0.1), (-0.7, 0.02, 0.0)]
    comp = scene_of([GROUND, CUBE, {"kind": "compound", "children": [(1, cp[0], Q0), (1, cp[1], tilt)]}],
                    [(0, 0.0, (0, -0.5, 0), Q0), (2, 1.0, (0.2, 0.49, -0.3), yaw)])
    w, o, c = contacts_of(host_ctx, comp)
    assert len(c["normal"]) == 2
    # the same children as bodies, at the composed poses
    poses = [oracle_child_pose((0.2, 0.49, -0.3), yaw, p, q) for p, q in ((cp[0], Q0), (cp[1], tilt))]
    sep = scene_of([GROUND, CUBE], [(0, 0.0, (0, -0.5, 0), Q0)] + [(1, 1.0, p, q) for p, q in poses])
    w2, o2, c2 = contacts_of(host_ctx, sep)
    assert len(c2["normal"]) == 2
    for k in range(2):
        n = int(c["normal"][k][3])
        assert n == int(c2["normal"][k][3])
        assert np.allclose(c["normal"][k][:3], c2["normal"][k][:3], atol=1e-12)
        a = c["pos"][k][:n]
        b = c2["pos"][k][:n]
        assert np.abs(a[np.lexsort(a[:, :3].T)] - b[np.lexsort(b[:, :3].T)]).max() < 1e-9
    # both manifolds are the compound body's
    assert set(np.abs(c["bodyA"]).tolist() + np.abs(c["bodyB"]).tolist()) == {0, 1}
    w.close()
    w2.close()


def oracle_child_pose(pos, q, cp, cq):
    """qtRotate(q, cp) + pos and qtMul(q, cq) in FP32, the oracle's and the
    device's operation order (findCompoundPairsKernel, P2/sat.cl:774-781)."""
    f = np.float32
    q = np.asarray(q, f)
    cq = np.asarray(cq, f)

    def qmul(a, b):
        c0 = f(a[1] * b[2]) - f(a[2] * b[1])
        c1 = f(a[2] * b[0]) - f(a[0] * b[2])
        c2 = f(a[0] * b[1]) - f(a[1] * b[0])
        r = np.array([c0 + (f(a[3] * b[0]) + f(b[3] * a[0])), c1 + (f(a[3] * b[1]) + f(b[3] * a[1])),
                      c2 + (f(a[3] * b[2]) + f(b[3] * a[2])),
                      f(a[3] * b[3]) - ((f(a[0] * b[0]) + f(a[1] * b[1])) + f(a[2] * b[2]))], f)
        return r
    v = np.array([cp[0], cp[1], cp[2], 0], f)
    r = qmul(qmul(q, v), np.array([-q[0], -q[1], -q[2], q[3]], f))
    return tuple((r[:3] + np.asarray(pos, f)).tolist()), tuple(qmul(q, cq).tolist())


def test_cube_on_mesh_known_answer(host_ctx):
    """A cube resting slightly into a flat two-triangle mesh square: each
    triangle under the cube gives a manifold on the triangle's front face,
    and together their points are the cube's bottom corners (and the cuts
    of its bottom face by the diagonal), all at the cube's depth."""
    sq = np.array([[-3, 0, 3], [3, 0, 3], [-3, 0, -3], [3, 0, -3]], np.float32)
    yaw = scenes.yaw_quat(np.array([0.4]))[0]
    sc = scene_of([{"kind": "mesh", "vertices": sq, "indices": [0, 1, 2, 2, 1, 3]}, CUBE],
                  [(0, 0.0, (0, 0, 0), Q0), (1, 1.0, (0.3, 0.49, 0.2), yaw)])
    w, o, c = contacts_of(host_ctx, sc)
    assert len(c["normal"]) == 2  # the cube straddles the diagonal
    pts = []
    for k in range(2):
        assert abs(c["bodyA"][k]) == 0 and c["bodyB"][k] == 1  # the mesh is side A
        assert np.allclose(c["normal"][k][:3], [0, 1, 0], atol=1e-9)
        n = int(c["normal"][k][3])
        pts.append(c["pos"][k][:n])
    pts = np.concatenate(pts)
    assert np.allclose(pts[:, 3], 0.49 - 0.5, atol=1e-6) and np.allclose(pts[:, 1], -0.01, atol=1e-6)
    # every point lies inside the cube's footprint
    R = np.array([[np.cos(0.4), 0, np.sin(0.4)], [0, 1, 0], [-np.sin(0.4), 0, np.cos(0.4)]])
    local = (pts[:, :3] - [0.3, 0.49, 0.2]) @ R
    assert np.abs(local[:, [0, 2]]).max() <= 0.5 + 1e-6
    w.close()


def test_dynamics_rest(host_ctx):
    """Stepped by the oracle, a sphere rests on a plane, a compound on a
    ground box and a cube on a mesh, without falling through. (The mesh body
    stays at the origin: its triangles' local AABBs are culled against world
    AABBs, as in the reference.)"""
    sq = np.array([[-5, 0, 5], [5, 0, 5], [-5, 0, -5], [5, 0, -5]], np.float32)
    sc = scene_of([{"kind": "plane", "normal": [0, 1, 0], "constant": 0.0}, {"kind": "sphere", "radius": 0.3},
                   CUBE, {"kind": "compound", "children": [(2, (0.55, 0, 0), Q0), (2, (-0.55, 0, 0), Q0)]},
                   {"kind": "mesh", "vertices": sq, "indices": [0, 1, 2, 2, 1, 3]}, GROUND],
                  [(0, 0.0, (0, 0, 0), Q0), (1, 1.0, (10, 1.0, 10), Q0), (4, 0.0, (0, 0, 0), Q0),
                   (3, 2.0, (-30, 1.5, -30), Q0), (2, 1.0, (2, 1.0, 2), Q0), (5, 0.0, (-30, -0.5, -30), Q0)],
                  dims=(64, 64, 64))
    w, o = host_oracle(host_ctx, sc)
    o.step(150)
    p, _, v, _ = o.state()
    assert abs(p[1][1] - 0.3) < 0.02 and abs(v[1][1]) < 0.05      # sphere on the plane
    assert abs(p[3][1] - 0.5) < 0.03 and abs(v[3][1]) < 0.1       # compound on the ground box
    assert abs(p[4][1] - 0.5) < 0.03 and abs(v[4][1]) < 0.1       # cube on the mesh square
    w.close()
