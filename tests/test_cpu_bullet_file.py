""".bullet scene files (b3_load_bullet_file, btBulletDataExtractor::
convertAllObjects) against a file the reference's own serializer wrote.

tests/golden/pile.bullet is bullet2's btDefaultSerializer output for a seeded
pile of 40 bodies (unit cubes as btBoxShape, 12-point hulls as
btConvexHullShape) on a static ground box; tests/golden/pile_bullet.npz holds
the scene it was made from. Loading the file must give back every body (the
static ground only when static objects are kept) with its position, its
orientation (up to the quaternion's sign), its mass, and a shape whose hull
equals the hull of the original points; without static objects the demo's
50 x 50 ground tiles are added instead."""
import os

import numpy as np
import pytest

from experiments_b200 import b3, scenes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FILE = os.path.join(GOLDEN, "pile.bullet")


def _world(host_ctx, n):
    return b3.PhysicsWorld(host_ctx, b3.default_config(maxBodies=n, gridDims=(16, 16, 16)))


def _hull_vertices(w, col):
    sh = w.shapes()
    poly = sh["polys"][int(sh["cols"][col].shapeIndex)]
    v = sh["verts"][poly.vertexOffset:poly.vertexOffset + poly.numVertices, :3]
    return np.array(sorted(map(tuple, np.round(v.astype(np.float64), 5))))


def _reference_hulls(host_ctx, g):
    """The product's hull of each original shape's points."""
    w = _world(host_ctx, 8)
    out = []
    for k in range(len(g["shapeOffsets"]) - 1):
        pts = g["points"][g["shapeOffsets"][k]:g["shapeOffsets"][k + 1]]
        out.append(_hull_vertices(w, w.registerConvexPolyhedron(pts)))
    w.close()
    return out


@pytest.mark.parametrize("keep_static", [True, False])
def test_loaded_scene_matches_the_written_one(host_ctx, keep_static):
    g = np.load(os.path.join(GOLDEN, "pile_bullet.npz"))
    n = len(g["mass"])
    w = _world(host_ctx, n + 2600)
    added = w.load_bullet_file(FILE, keep_static_objects=keep_static)
    dyn = g["mass"] > 0
    expect = n if keep_static else int(dyn.sum()) + 2500
    assert added == expect == w.n
    bodies = w.read_bodies()
    hulls = _reference_hulls(host_ctx, g)
    matched = 0
    for i in range(w.n):
        b = bodies[i]
        p = np.array(b.pos[:3])
        d = np.linalg.norm(g["pos"] - p, axis=1)
        j = int(np.argmin(d))
        if not keep_static and b.invMass == 0:
            continue  # a ground tile (checked below)
        assert d[j] < 1e-6, f"body {i} at {p} has no counterpart"
        q = np.array(b.quat, np.float64)
        assert abs(abs(q @ g["quat"][j].astype(np.float64)) - 1.0) < 2e-6
        mass = 0.0 if b.invMass == 0 else 1.0 / b.invMass
        assert mass == pytest.approx(float(g["mass"][j]), rel=2e-6)
        assert b.friction == 1.0
        got = _hull_vertices(w, b.collidableIdx)
        want = hulls[int(g["shape"][j])]
        assert got.shape == want.shape and np.abs(got - want).max() < 2e-5
        matched += 1
    assert matched == (n if keep_static else int(dyn.sum()))
    if not keep_static:
        tiles = [bodies[i] for i in range(w.n) if bodies[i].invMass == 0]
        assert len(tiles) == 2500
        xs = sorted({round(t.pos[0], 3) for t in tiles})
        assert len(xs) == 50 and xs[0] == pytest.approx(-120.0) and xs[1] - xs[0] == pytest.approx(5.01, abs=1e-4)
    # bodies come grouped by shape: one run of bodies per shape
    cols = [int(bodies[i].collidableIdx) for i in range(w.n)]
    runs = [c for k, c in enumerate(cols) if k == 0 or c != cols[k - 1]]
    assert len(runs) == len(set(runs))
    w.close()


def test_rejects_what_is_not_a_single_precision_bullet_file(host_ctx, tmp_path):
    w = _world(host_ctx, 8)
    bad = tmp_path / "x.bullet"
    bad.write_bytes(b"not a bullet file at all")
    with pytest.raises(b3.B3Error):
        w.load_bullet_file(str(bad))
    raw = bytearray(open(FILE, "rb").read())
    raw[6] = ord("d")  # double precision: refused, as in the reference demo
    bad.write_bytes(bytes(raw))
    with pytest.raises(b3.B3Error):
        w.load_bullet_file(str(bad))
    with pytest.raises(b3.B3Error):
        w.load_bullet_file(str(tmp_path / "missing.bullet"))
    w.close()


def test_fixture_is_the_seeded_scene():
    """The committed scene record is the seeded pile the file was written
    from (tests/golden/make_golden.py)."""
    g = np.load(os.path.join(GOLDEN, "pile_bullet.npz"))
    sc = scenes.random_pile(61, n=40, hull_frac=0.5, pool=4)
    assert np.array_equal(np.asarray(sc.pos, np.float32), g["pos"])
    assert np.array_equal(np.asarray(sc.mass, np.float32), g["mass"])


@pytest.mark.gpu
def test_loaded_file_steps_on_the_device(ctx):
    """The loaded scene (static ground kept) steps on the device: the pile
    falls and comes to rest on the ground, nothing passes through it."""
    g = np.load(os.path.join(GOLDEN, "pile_bullet.npz"))
    # the world configuration the pile's own tests use (large ground proxy)
    w = b3.PhysicsWorld(ctx, scenes.world_config(scenes.random_pile(61, n=40, hull_frac=0.5, pool=4)))
    assert w.load_bullet_file(FILE, keep_static_objects=True) == len(g["mass"])
    w.writeBodiesToGpu()
    w.stepSimulation(240)
    pos, _, lin, _ = w.read_state()
    dyn = np.array([b.invMass != 0 for b in w.read_bodies()])
    # every centre stays above the ground's top face (y = 0): flat hulls
    # rest about 0.1 m above it, cubes 0.5 m
    assert np.isfinite(pos).all() and np.all(pos[dyn, 1] > 0.0)
    assert np.abs(lin[dyn, :3]).max() < 1.0
    assert w.counters()["timeouts"] == 0
    w.close()


def _hull_count_offsets(raw):
    """Byte offsets of m_numUnscaledPoints in the file's convex hull shape
    records (64-bit pointers, little endian): a chunk header is code, length,
    old pointer (8), struct index, count; btConvexHullShapeData holds the
    convex-internal part (56 bytes: name pointer, shape type, padding,
    scaling, dimensions, margin, padding), two point pointers, then the
    count."""
    out, o = [], 12
    while o + 24 <= len(raw):
        code = bytes(raw[o:o + 4])
        length = int.from_bytes(raw[o + 4:o + 8], "little")
        data = o + 24
        if code == b"ENDB":
            break
        if code == b"SHAP" and int.from_bytes(raw[data + 8:data + 12], "little") == 4:
            out.append(data + 72)
        o = data + length
    return out


@pytest.mark.parametrize("count", [100, 0x10000000, 1 << 20])
def test_hull_point_counts_are_checked_before_anything_registers(host_ctx, tmp_path, count):
    """A hull record whose point count exceeds its point data (100), whose
    byte size overflows 32-bit arithmetic (2^28 points x 16 bytes = 2^32) or
    exceeds the 65,536-point limit is refused, and the world is left with
    nothing registered."""
    raw = bytearray(open(FILE, "rb").read())
    offs = _hull_count_offsets(raw)
    assert offs and all(int.from_bytes(raw[o:o + 4], "little") == 12 for o in offs)
    raw[offs[-1]:offs[-1] + 4] = int(count).to_bytes(4, "little")
    bad = tmp_path / "corrupt.bullet"
    bad.write_bytes(bytes(raw))
    w = _world(host_ctx, 3000)
    with pytest.raises(b3.B3Error):
        w.load_bullet_file(str(bad), keep_static_objects=False)
    assert w.n == 0 and w.shapes()["counts"][:2] == (0, 0)
    # the intact file still loads into the same world afterwards
    assert w.load_bullet_file(FILE, keep_static_objects=True) == w.n > 0
    w.close()


def test_a_file_that_does_not_fit_registers_nothing(host_ctx):
    g = np.load(os.path.join(GOLDEN, "pile_bullet.npz"))
    w = _world(host_ctx, len(g["mass"]) - 1)
    with pytest.raises(b3.B3Error):
        w.load_bullet_file(FILE, keep_static_objects=True)
    assert w.n == 0 and w.shapes()["counts"][:2] == (0, 0)
    w.close()


SPHERES = os.path.join(GOLDEN, "spheres.bullet")


def test_spheres_and_planes_are_skipped_as_in_the_reference(host_ctx):
    """The reference's extractor skips sphere and plane shapes
    (createSphereShape / createPlaneShape return -1), and so does the
    default load: of the spheres-on-a-plane file only the replacement
    ground registers."""
    w = _world(host_ctx, 2600)
    assert w.load_bullet_file(SPHERES) == 2500
    w.close()


@pytest.mark.parametrize("keep_static", [True, False])
def test_spheres_and_planes_load_on_request(host_ctx, keep_static):
    """With B3_BULLET_SPHERES_AND_PLANES every sphere registers as a sphere
    of its radius (implicit dimension x times scaling x) at its position and
    mass; the static plane body registers with keepStaticObjects."""
    g = np.load(os.path.join(GOLDEN, "spheres_bullet.npz"))
    n = len(g["mass"])
    dyn = g["mass"] > 0
    w = _world(host_ctx, n + 2600)
    added = w.load_bullet_file(SPHERES, keep_static_objects=keep_static, spheres_and_planes=True)
    assert added == (n if keep_static else int(dyn.sum()) + 2500) == w.n
    bodies = w.read_bodies()
    cols = w.shapes()["cols"]
    spheres = planes = 0
    for i in range(w.n):
        b = bodies[i]
        c = cols[int(b.collidableIdx)]
        if c.shapeType == 7:  # sphere
            p = np.array(b.pos[:3])
            j = int(np.argmin(np.linalg.norm(g["pos"] - p, axis=1)))
            assert np.abs(g["pos"][j] - p).max() == 0.0
            assert c.radius == pytest.approx(float(g["radius"][j]), rel=1e-6)
            assert 1.0 / b.invMass == pytest.approx(float(g["mass"][j]), rel=2e-6)
            spheres += 1
        elif c.shapeType == 4:  # plane
            assert b.invMass == 0 and c.radius == pytest.approx(float(g["plane"][3]))
            face = w.shapes()["faces"][int(c.shapeIndex)]
            assert np.allclose(np.array(face.plane[:3]), g["plane"][:3])
            planes += 1
    assert spheres == int(dyn.sum())
    assert planes == (1 if keep_static else 0)
    w.close()


def test_spheres_fixture_is_the_seeded_scene():
    g = np.load(os.path.join(GOLDEN, "spheres_bullet.npz"))
    sc = scenes.spheres_on_plane(84, n=24)
    assert np.array_equal(np.asarray(sc.pos, np.float32), g["pos"])
    assert np.array_equal(np.asarray(sc.mass, np.float32), g["mass"])


@pytest.mark.gpu
def test_loaded_spheres_rest_on_the_plane(ctx):
    """The spheres-on-a-plane file loaded with its spheres and plane steps
    on the device: no sphere passes through the plane, nearly all of them
    come to rest on it (a few may rest on others), none moves vertically."""
    g = np.load(os.path.join(GOLDEN, "spheres_bullet.npz"))
    w = b3.PhysicsWorld(ctx, scenes.world_config(scenes.spheres_on_plane(84, n=24)))
    w.load_bullet_file(SPHERES, keep_static_objects=True, spheres_and_planes=True)
    w.writeBodiesToGpu()
    w.stepSimulation(300)
    pos, _, lin, _ = w.read_state()
    bodies = w.read_bodies()
    cols = w.shapes()["cols"]
    on_plane = 0
    for i in range(w.n):
        if bodies[i].invMass == 0:
            continue
        r = cols[int(bodies[i].collidableIdx)].radius
        assert pos[i, 1] > r - 0.03
        on_plane += abs(pos[i, 1] - r) < 0.03
    assert on_plane >= 0.8 * (w.n - 1)
    # spheres keep rolling (no rolling friction), but nothing moves vertically
    assert np.abs(lin[[b.invMass != 0 for b in bodies], 1]).max() < 0.1
    assert w.counters()["timeouts"] == 0
    w.close()
