"""Seeded synthetic scenes for the rigid-body step.

Every random draw comes from a counter-based generator (splitmix64 of
seed, stream and index), so a scene is a pure function of its seed and
parameters; the same arrays feed the CUDA world, the oracle and the CPU
baseline. Workloads (no public dataset exists for this path):

  c1  4,096 unit cubes, 16^3 lattice at 1.05 m, 1 m above a 200x1x200 m
      static ground box, position jitter U(+-0.02), yaw U(0, 2pi),
      mass 1, friction 0.6, cell 1.0 m
  c2  131,072 bodies, 64x32x64 lattice at 1.2 m: 1/2 unit cubes, 1/4 hulls
      of 12 points on a radius-0.5 sphere, 1/4 42-vertex icospheres of
      radius 0.5; mass U(0.5, 2), friction U(0.3, 0.9), yaw U(0, 2pi),
      cell 1.2 m
  c3  4,096 independent worlds, N ~ log-uniform[8, 512] bodies each, cubes
      and 12-point hulls 50/50, uniform positions over a 4 m x 4 m
      footprint, velocities N(0, 0.5), one ground box per world
  c4  256 worlds x 64 unit cubes (4^3 lattice at 1.05 m), velocities
      N(0, 1), mass U(0.5, 2), friction U(0.3, 0.9), target U(+-3)^3
  c5  1,048,576 unit cubes, 128x64x128 lattice at 1.05 m, jitter U(+-0.02)

12-point hull shapes are drawn from a seeded pool of distinct hulls (64 by
default) that bodies share, so the hull tables stay small enough to stay
on chip.
"""
from dataclasses import dataclass, field

import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix64(x):
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & _M64
    z = x
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _M64
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _M64
    return z ^ (z >> np.uint64(31))


def uniform(seed, stream, n, lo=0.0, hi=1.0):
    """U[lo, hi) doubles from counter (seed, stream, i), i < n."""
    with np.errstate(over="ignore"):
        base = _splitmix64(np.uint64(seed) * np.uint64(0x100000001B3) + np.uint64(stream))
        idx = np.arange(n, dtype=np.uint64)
        r = _splitmix64(base ^ (idx * np.uint64(0xD1B54A32D192ED03)))
    u = (r >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))
    return lo + (hi - lo) * u


def normal(seed, stream, n, sigma=1.0):
    u1 = uniform(seed, stream, n)
    u2 = uniform(seed, stream + 7919, n)
    return sigma * np.sqrt(-2.0 * np.log(np.maximum(u1, 1e-300))) * np.cos(2 * np.pi * u2)


# ---------------------------------------------------------------------------
# Shapes
# ---------------------------------------------------------------------------
def box_vertices(hx, hy, hz):
    return np.array([[sx * hx, sy * hy, sz * hz] for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)],
                    np.float32)


def sphere_points(seed, n=12, radius=0.5, stream=0):
    z = uniform(seed, 1000 + 2 * stream, n, -1.0, 1.0)
    phi = uniform(seed, 1001 + 2 * stream, n, 0.0, 2 * np.pi)
    r = np.sqrt(np.maximum(0.0, 1 - z * z))
    return (radius * np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)).astype(np.float32)


def icosphere_vertices(radius=0.5):
    """Icosahedron subdivided once: 12 + 30 = 42 vertices on the sphere."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    v = [np.array(p, np.float64) / np.linalg.norm(p) for p in v]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    mids = {}
    for a, b, c in f:
        for i, j in ((a, b), (b, c), (c, a)):
            k = (min(i, j), max(i, j))
            if k not in mids:
                m = v[i] + v[j]
                mids[k] = len(v)
                v.append(m / np.linalg.norm(m))
    return (radius * np.array(v)).astype(np.float32)


def yaw_quat(angle):
    h = 0.5 * np.asarray(angle, np.float64)
    q = np.zeros((np.size(h), 4))
    q[:, 1] = np.sin(h)
    q[:, 3] = np.cos(h)
    return q


# ---------------------------------------------------------------------------
# Scene container
# ---------------------------------------------------------------------------
@dataclass
class Scene:
    name: str
    shapes: list                     # list of (vertices (k,3) float32)
    shape: np.ndarray                # (n,) int shape index per body
    mass: np.ndarray                 # (n,) float32, 0 = static
    pos: np.ndarray                  # (n,3)
    quat: np.ndarray                 # (n,4) x,y,z,w
    friction: np.ndarray             # (n,)
    world: np.ndarray                # (n,) world id
    lin: np.ndarray                  # (n,3)
    ang: np.ndarray                  # (n,3)
    num_worlds: int = 1
    config: dict = field(default_factory=dict)
    steps: int = 1
    extra: dict = field(default_factory=dict)

    @property
    def n(self):
        return int(self.mass.shape[0])


def _concat(parts):
    keys = ["shape", "mass", "pos", "quat", "friction", "world", "lin", "ang"]
    return {k: np.concatenate([p[k] for p in parts]) for k in keys}


def _bodies(shape, mass, pos, quat, friction, world, lin=None, ang=None):
    n = len(shape)
    return dict(shape=np.asarray(shape, np.int32), mass=np.asarray(mass, np.float32),
                pos=np.asarray(pos, np.float32).reshape(n, 3), quat=np.asarray(quat, np.float32).reshape(n, 4),
                friction=np.asarray(friction, np.float32), world=np.asarray(world, np.int32),
                lin=np.zeros((n, 3), np.float32) if lin is None else np.asarray(lin, np.float32).reshape(n, 3),
                ang=np.zeros((n, 3), np.float32) if ang is None else np.asarray(ang, np.float32).reshape(n, 3))


def ground(world=0, friction=0.6, size=200.0, y_top=0.0):
    return _bodies([0], [0.0], [[0.0, y_top - 0.5, 0.0]], [[0, 0, 0, 1]], [friction], [world])


def lattice_scene(name, seed, dims, spacing, shapes_of, mass_of, fric_of, jitter=0.02, yaw=True, y0=1.0,
                  ground_friction=0.6, config=None, steps=1, extra_shapes=()):
    nx, ny, nz = dims
    n = nx * ny * nz
    ix, iy, iz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ix, iy, iz = ix.ravel(), iy.ravel(), iz.ravel()
    j = uniform(seed, 1, 3 * n, -jitter, jitter).reshape(n, 3) if jitter > 0 else np.zeros((n, 3))
    pos = np.stack([(ix - (nx - 1) / 2.0) * spacing, y0 + 0.5 + iy * spacing, (iz - (nz - 1) / 2.0) * spacing], 1) + j
    quat = yaw_quat(uniform(seed, 2, n, 0.0, 2 * np.pi)) if yaw else np.tile([0, 0, 0, 1.0], (n, 1))
    shapes = [box_vertices(100.0, 0.5, 100.0)] + list(extra_shapes)
    body_shape = shapes_of(n)
    parts = [ground(friction=ground_friction),
             _bodies(body_shape, mass_of(n), pos, quat, fric_of(n), np.zeros(n))]
    b = _concat(parts)
    return Scene(name=name, shapes=shapes, num_worlds=1, config=config or {}, steps=steps, **b)


def c1(seed=1, dims=(16, 16, 16), steps=300):
    """4,096 unit cubes over a static ground box (config 1)."""
    return lattice_scene("c1_cubes_4096" if dims == (16, 16, 16) else f"cubes_{dims}", seed, dims, 1.05,
                         lambda n: np.ones(n, np.int32), lambda n: np.ones(n), lambda n: np.full(n, 0.6),
                         config=dict(cellSize=1.0, gridDims=(64, 64, 64)), steps=steps,
                         extra_shapes=[box_vertices(0.5, 0.5, 0.5)])


def hull_pool(seed, count=64):
    return [sphere_points(seed, 12, 0.5, stream=k) for k in range(count)]


def c2(seed=2, dims=(64, 32, 64), steps=1000, pool=64):
    """131,072 mixed hulls (config 2)."""
    n = dims[0] * dims[1] * dims[2]
    hulls = hull_pool(seed, pool)
    extra = [box_vertices(0.5, 0.5, 0.5), icosphere_vertices(0.5)] + hulls

    def shapes_of(n):
        kind = np.zeros(n, np.int32)
        perm = np.argsort(uniform(seed, 3, n))
        kind[perm[n // 2: n // 2 + n // 4]] = 1    # 12-point hull
        kind[perm[n // 2 + n // 4:]] = 2            # icosphere
        sid = np.ones(n, np.int32)                 # cube -> shape 1
        sid[kind == 2] = 2
        pick = (uniform(seed, 4, n) * pool).astype(np.int32) % pool
        sid[kind == 1] = 3 + pick[kind == 1]
        return sid

    return lattice_scene("c2_mixed_131072" if dims == (64, 32, 64) else f"mixed_{dims}", seed, dims, 1.2,
                         shapes_of, lambda n: uniform(seed, 5, n, 0.5, 2.0),
                         lambda n: uniform(seed, 6, n, 0.3, 0.9),
                         config=dict(cellSize=1.2, gridDims=(128, 64, 128)), steps=steps, extra_shapes=extra)


def c3(seed=3, worlds=4096, nmin=8, nmax=512, steps=600, pool=64):
    """Batched independent piles (config 3)."""
    hulls = hull_pool(seed, pool)
    shapes = [box_vertices(10.0, 0.5, 10.0), box_vertices(0.5, 0.5, 0.5)] + hulls
    counts = np.floor(np.exp(uniform(seed, 10, worlds, np.log(nmin), np.log(nmax + 1)))).astype(np.int64)
    counts = np.clip(counts, nmin, nmax)
    total = int(counts.sum())
    wid = np.repeat(np.arange(worlds), counts)
    # position: 4 m x 4 m footprint; height range grows with N to keep the
    # initial density near one body per 1.5 m^3
    h = 4.0 * np.maximum(1.0, counts / 42.0)
    u = uniform(seed, 11, 3 * total).reshape(total, 3)
    pos = np.stack([u[:, 0] * 4.0 - 2.0, 1.0 + u[:, 1] * h[wid], u[:, 2] * 4.0 - 2.0], 1)
    kind = (uniform(seed, 12, total) < 0.5)
    sid = np.where(kind, 1, 2 + ((uniform(seed, 13, total) * pool).astype(np.int32) % pool)).astype(np.int32)
    quat = yaw_quat(uniform(seed, 14, total, 0.0, 2 * np.pi))
    lin = normal(seed, 15, 3 * total, 0.5).reshape(total, 3)
    grounds = _bodies(np.zeros(worlds), np.zeros(worlds), np.tile([0.0, -0.5, 0.0], (worlds, 1)),
                      np.tile([0, 0, 0, 1.0], (worlds, 1)), np.full(worlds, 0.6), np.arange(worlds))
    dyn = _bodies(sid, np.ones(total), pos, quat, np.full(total, 0.6), wid, lin=lin)
    b = _concat([grounds, dyn])
    return Scene(name=f"c3_batched_{worlds}", shapes=shapes, num_worlds=worlds,
                 config=dict(cellSize=1.0, gridDims=(16, 16, 16)), steps=steps,
                 extra=dict(counts=counts), **b)


def c4(seed=4, worlds=256, steps=120):
    """Differentiable throw: 256 worlds x 64 cubes (config 4)."""
    shapes = [box_vertices(10.0, 0.5, 10.0), box_vertices(0.5, 0.5, 0.5)]
    per = 64
    total = worlds * per
    ix, iy, iz = np.meshgrid(np.arange(4), np.arange(4), np.arange(4), indexing="ij")
    local = np.stack([(ix.ravel() - 1.5) * 1.05, 1.5 + iy.ravel() * 1.05, (iz.ravel() - 1.5) * 1.05], 1)
    pos = np.tile(local, (worlds, 1))
    wid = np.repeat(np.arange(worlds), per)
    lin = normal(seed, 20, 3 * total, 1.0).reshape(total, 3)
    mass = uniform(seed, 21, total, 0.5, 2.0)
    fr = uniform(seed, 22, total, 0.3, 0.9)
    target = uniform(seed, 23, 3 * worlds, -3.0, 3.0).reshape(worlds, 3)
    grounds = _bodies(np.zeros(worlds), np.zeros(worlds), np.tile([0.0, -0.5, 0.0], (worlds, 1)),
                      np.tile([0, 0, 0, 1.0], (worlds, 1)), np.full(worlds, 0.6), np.arange(worlds))
    dyn = _bodies(np.ones(total), mass, pos, np.tile([0, 0, 0, 1.0], (total, 1)), fr, wid, lin=lin)
    b = _concat([grounds, dyn])
    return Scene(name=f"c4_throw_{worlds}x64", shapes=shapes, num_worlds=worlds,
                 config=dict(cellSize=1.0, gridDims=(16, 16, 16)), steps=steps, extra=dict(target=target), **b)


def c5(seed=5, dims=(128, 64, 128), steps=32):
    """1,048,576 unit cubes (config 5)."""
    return lattice_scene("c5_cubes_1048576" if dims == (128, 64, 128) else f"cubes_{dims}", seed, dims, 1.05,
                         lambda n: np.ones(n, np.int32), lambda n: np.ones(n), lambda n: np.full(n, 0.6),
                         config=dict(cellSize=1.0, gridDims=(256, 128, 256),
                                     maxPairs=8 * (dims[0] * dims[1] * dims[2] + 1)), steps=steps,
                         extra_shapes=[box_vertices(0.5, 0.5, 0.5)])


def random_pile(seed, n=64, worlds=1, box=4.0, hull_frac=0.5, pool=8, velocity=0.5, orient="random"):
    """Small test pile: uniformly placed cubes / 12-point hulls, random
    orientations, one ground per world."""
    hulls = hull_pool(seed, pool)
    shapes = [box_vertices(10.0, 0.5, 10.0), box_vertices(0.5, 0.5, 0.5), icosphere_vertices(0.5)] + hulls
    total = n * worlds
    wid = np.repeat(np.arange(worlds), n)
    u = uniform(seed, 31, 3 * total).reshape(total, 3)
    pos = np.stack([u[:, 0] * box - box / 2, 0.3 + u[:, 1] * box, u[:, 2] * box - box / 2], 1)
    k = uniform(seed, 32, total)
    sid = np.where(k < 1 - hull_frac, 1, 3 + (uniform(seed, 33, total) * pool).astype(np.int32) % pool)
    if orient == "random":
        q = normal(seed, 34, 4 * total).reshape(total, 4)
        q /= np.linalg.norm(q, axis=1, keepdims=True)
    else:
        q = np.tile([0, 0, 0, 1.0], (total, 1))
    lin = normal(seed, 35, 3 * total, velocity).reshape(total, 3)
    ang = normal(seed, 36, 3 * total, velocity).reshape(total, 3)
    mass = uniform(seed, 37, total, 0.5, 2.0)
    fr = uniform(seed, 38, total, 0.3, 0.9)
    grounds = _bodies(np.zeros(worlds), np.zeros(worlds), np.tile([0.0, -0.5, 0.0], (worlds, 1)),
                      np.tile([0, 0, 0, 1.0], (worlds, 1)), np.full(worlds, 0.6), np.arange(worlds))
    dyn = _bodies(sid, mass, pos, q, fr, wid, lin=lin, ang=ang)
    b = _concat([grounds, dyn])
    return Scene(name=f"pile_{n}x{worlds}", shapes=shapes, num_worlds=worlds,
                 config=dict(cellSize=1.0, gridDims=(16, 16, 16), maxPairs=max(4096, 40 * total)), steps=1, **b)


SCENES = {"c1": c1, "c2": c2, "c3": c3, "c4": c4, "c5": c5}


def world_config(scene, **over):
    """b3WorldConfig fields for a scene."""
    from . import b3
    n = scene.n
    kw = dict(maxBodies=n, numWorlds=scene.num_worlds, maxPairsPerBody=32, maxBodiesPerCell=64,
              maxSmallProxySize=4.0 * scene.config.get("cellSize", 1.0), solverIterations=10,
              dt=1.0 / 60.0)
    kw["maxPairs"] = max(4096, 16 * n)
    kw.update(scene.config)
    kw.update(over)
    return b3.default_config(**kw)


def register_shape(w, entry):
    """Register one scene shape: an array of points (a convex hull), or a
    dict {"kind": "sphere", "radius"}, {"kind": "plane", "normal",
    "constant"}, {"kind": "compound", "children": [(shape index, position,
    orientation), ...]} (children are earlier shapes of the scene, which are
    collidables in registration order) or {"kind": "mesh", "vertices",
    "indices", "scaling"}."""
    if not isinstance(entry, dict):
        return w.registerConvexPolyhedron(entry)
    kind = entry["kind"]
    if kind == "sphere":
        return w.registerSphereShape(entry["radius"])
    if kind == "plane":
        return w.registerPlaneShape(entry["normal"], entry["constant"])
    if kind == "compound":
        return w.registerCompoundShape(entry["children"])
    if kind == "mesh":
        return w.registerConcaveMesh(entry["vertices"], entry["indices"], entry.get("scaling", (1.0, 1.0, 1.0)))
    raise ValueError(f"unknown shape kind {kind}")


def register_scene(w, scene):
    """Register the scene's shapes and bodies on a PhysicsWorld (host only)."""
    cols = np.array([register_shape(w, v) for v in scene.shapes], np.int32)
    w.register_bodies(scene.mass, scene.pos, scene.quat, cols[scene.shape], friction=scene.friction,
                      world=scene.world)
    return cols


def build_world(ctx, scene, **over):
    """Create a PhysicsWorld holding the scene (registered + written)."""
    from . import b3
    w = b3.PhysicsWorld(ctx, world_config(scene, **over))
    register_scene(w, scene)
    w.writeBodiesToGpu()
    if np.any(scene.lin) or np.any(scene.ang):
        w.write_velocities(scene.lin, scene.ang)
    return w


def select_worlds(scene, world_ids):
    """Sub-scene holding only the given worlds, renumbered 0..k-1 (a single
    world becomes a plain one-world scene)."""
    world_ids = list(world_ids)
    remap = {w: i for i, w in enumerate(world_ids)}
    keep = np.isin(scene.world, world_ids)
    b = dict(shape=scene.shape[keep], mass=scene.mass[keep], pos=scene.pos[keep], quat=scene.quat[keep],
             friction=scene.friction[keep], world=np.array([remap[int(w)] for w in scene.world[keep]], np.int32),
             lin=scene.lin[keep], ang=scene.ang[keep])
    cfg = dict(scene.config)
    cfg.pop("maxPairs", None)
    return Scene(name=f"{scene.name}_sel{len(world_ids)}", shapes=scene.shapes, num_worlds=len(world_ids),
                 config=cfg, steps=scene.steps, **b)


def lattice_block(scene, dims, block, blocks=(4, 4)):
    """Sub-scene of a lattice scene: the static ground plus the column of
    bodies whose lattice x and z indices fall in block `block` of a
    blocks[0] x blocks[1] tiling of the footprint (all layers). The blocks
    tile the scene, so running every block covers every body once."""
    nx, ny, nz = dims
    bx, bz = nx // blocks[0], nz // blocks[1]
    ix, iy, iz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ix, iz = ix.ravel(), iz.ravel()
    x0, z0 = (block // blocks[1]) * bx, (block % blocks[1]) * bz
    sel = (ix >= x0) & (ix < x0 + bx) & (iz >= z0) & (iz < z0 + bz)
    idx = np.concatenate([[0], 1 + np.nonzero(sel)[0]])  # body 0 is the ground
    b = dict(shape=scene.shape[idx], mass=scene.mass[idx], pos=scene.pos[idx], quat=scene.quat[idx],
             friction=scene.friction[idx], world=scene.world[idx], lin=scene.lin[idx], ang=scene.ang[idx])
    return Scene(name=f"{scene.name}_block{block}", shapes=scene.shapes, num_worlds=1, config=dict(scene.config),
                 steps=scene.steps, **b)


def spheres_on_plane(seed=81, n=200, box=6.0):
    """Spheres of radius U(0.2, 0.5) dropped as a random pile onto a static
    plane y = 0 (the reference's sphere and plane shapes)."""
    radii = uniform(seed, 1, n, 0.2, 0.5)
    shapes = [{"kind": "plane", "normal": [0.0, 1.0, 0.0], "constant": 0.0}] + \
        [{"kind": "sphere", "radius": float(r)} for r in radii]
    u = uniform(seed, 2, 3 * n).reshape(n, 3)
    pos = np.stack([u[:, 0] * box - box / 2, 0.6 + u[:, 1] * box, u[:, 2] * box - box / 2], 1)
    lin = normal(seed, 3, 3 * n, 0.5).reshape(n, 3)
    parts = [_bodies([0], [0.0], [[0, 0, 0]], [[0, 0, 0, 1.0]], [0.6], [0]),
             _bodies(np.arange(1, n + 1), uniform(seed, 4, n, 0.5, 2.0), pos, np.tile([0, 0, 0, 1.0], (n, 1)),
                     uniform(seed, 5, n, 0.3, 0.9), np.zeros(n), lin=lin)]
    b = _concat(parts)
    return Scene(name=f"spheres_{n}", shapes=shapes, num_worlds=1,
                 config=dict(cellSize=1.0, gridDims=(32, 32, 32)), steps=1, **b)


def compound_pile(seed=82, n=120, spacing=4.0):
    """Compounds of unit cubes (two-cube bars and three-cube L shapes,
    children at fixed offsets and turns) mixed with 12-point hulls, in
    random orientations on a jittered 4 x k x 4 lattice (spacing beyond any
    two bodies' reach, so nothing starts interpenetrating), dropped onto a
    static ground box."""
    q90 = [0.0, np.sin(np.pi / 4), 0.0, np.cos(np.pi / 4)]
    shapes = [box_vertices(10.0, 0.5, 10.0), box_vertices(0.5, 0.5, 0.5)] + hull_pool(seed, 4)
    shapes.append({"kind": "compound", "children": [(1, (0.55, 0.0, 0.0), [0, 0, 0, 1.0]),
                                                    (1, (-0.55, 0.0, 0.0), [0, 0, 0, 1.0])]})
    shapes.append({"kind": "compound", "children": [(1, (0.0, 0.0, 0.0), [0, 0, 0, 1.0]),
                                                    (1, (1.05, 0.0, 0.0), q90), (1, (0.0, 0.0, 1.05), q90)]})
    k = uniform(seed, 1, n)
    sid = np.where(k < 0.35, 6, np.where(k < 0.7, 7, 2 + (uniform(seed, 2, n) * 4).astype(np.int32) % 4))
    i = np.arange(n)
    lat = np.stack([i % 4, i // 16, (i // 4) % 4], 1).astype(np.float64)
    pos = (lat - [1.5, 0.0, 1.5]) * spacing + [0.0, 2.0, 0.0] + uniform(seed, 3, 3 * n, -0.2, 0.2).reshape(n, 3)
    q = normal(seed, 4, 4 * n).reshape(n, 4)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    parts = [ground(), _bodies(sid, uniform(seed, 5, n, 0.5, 2.0), pos, q, uniform(seed, 6, n, 0.3, 0.9), np.zeros(n),
                               lin=normal(seed, 7, 3 * n, 0.5).reshape(n, 3))]
    b = _concat(parts)
    return Scene(name=f"compounds_{n}", shapes=shapes, num_worlds=1,
                 config=dict(cellSize=1.5, gridDims=(32, 32, 32)), steps=1, **b)


def mesh_terrain(seed=83, n=150, cells=16, size=16.0, box=6.0):
    """A static triangle-mesh terrain (cells x cells squares of two
    triangles, heights U(0, 0.3)) at the origin, with unit cubes and
    12-point hulls dropped as a random pile onto it."""
    g = cells + 1
    hx = (np.arange(g) / cells - 0.5) * size
    X, Z = np.meshgrid(hx, hx, indexing="ij")
    Y = uniform(seed, 1, g * g, 0.0, 0.3).reshape(g, g)
    verts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1).astype(np.float32)
    idx = []
    for i in range(cells):
        for j in range(cells):
            a, b_, c, d = i * g + j, (i + 1) * g + j, i * g + j + 1, (i + 1) * g + j + 1
            idx += [a, c, b_, b_, c, d]  # counter-clockwise seen from above (+y)
    shapes = [{"kind": "mesh", "vertices": verts, "indices": np.array(idx, np.int32)},
              box_vertices(0.5, 0.5, 0.5)] + hull_pool(seed, 4)
    k = uniform(seed, 2, n)
    sid = np.where(k < 0.5, 1, 2 + (uniform(seed, 3, n) * 4).astype(np.int32) % 4)
    u = uniform(seed, 4, 3 * n).reshape(n, 3)
    pos = np.stack([u[:, 0] * box - box / 2, 1.2 + u[:, 1] * 2 * box, u[:, 2] * box - box / 2], 1)
    q = normal(seed, 5, 4 * n).reshape(n, 4)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    parts = [_bodies([0], [0.0], [[0, 0, 0]], [[0, 0, 0, 1.0]], [0.6], [0]),
             _bodies(sid, uniform(seed, 6, n, 0.5, 2.0), pos, q, uniform(seed, 7, n, 0.3, 0.9), np.zeros(n))]
    b = _concat(parts)
    return Scene(name=f"terrain_{n}", shapes=shapes, num_worlds=1,
                 config=dict(cellSize=1.0, gridDims=(32, 32, 32)), steps=1, **b)
