"""The batched Gauss-Seidel restatement (the reference's GPU solver,
B3_WORLD_BATCHED_GS_SOLVER) on the CPU.

* Its Constraint4 setup (setConstraint4, ST/solverSetup.cl:520-609) is pinned
  to the reference's own recorded constraints: tests/golden/gs_solve_args.npz
  holds the argument dump of one BatchSolveKernelContact launch
  (testdata/m_batchSolveKernel.7z), whose Constraint4 records carry the
  effective masses, position terms, friction centres and friction effective
  masses that ContactToConstraintKernel computed from the recorded bodies.
  The normal rows and centres match value for value; the friction rows of
  that recorded revision use another tangent basis (checked separately), so
  the restatement's friction is pinned through the basis-independent sum.
* The recorded batching shows the invariant the solve relies on: inside a
  cell the constraints are sorted by batch and no dynamic body appears twice
  in a batch.
* On workload scenes the colouring is valid (no dynamic body twice in a
  (class, batch) group) and greedy (a manifold in batch b met, in every
  earlier batch of its class, an earlier manifold on one of its dynamic
  bodies), and stacks rest under the solver."""
import os

import numpy as np
import pytest

import oracle
from experiments_b200 import scenes
from helpers import host_oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _golden():
    return np.load(os.path.join(GOLDEN, "gs_solve_args.npz"))


def test_setconstraint4_matches_the_recorded_constraints():
    g = _golden()
    row = {int(b): k for k, b in enumerate(g["bodies"])}
    dt = float(np.float32(1.0 / 60.0))  # P1/btGpuNarrowPhaseAndSolver.cpp:1082
    n = len(g["batchIdx"])
    assert n == int(g["cellCount"].sum()) > 300
    checked = 0
    for j in range(n):
        a, b = (row[int(x)] for x in g["bodyAB"][j])
        jac = g["jacCoeffInv"][j]
        npts = int(np.count_nonzero(jac))
        assert npts >= 1 and np.all(jac[npts:] == 0)
        lin = g["linear"][j]
        assert lin[3] == np.float32(0.7)  # friction coefficient of the constraint
        normal4 = [-lin[0], -lin[1], -lin[2], npts]
        jc, bb, center, fj = oracle.gs_constraint(
            g["worldPos"][j], normal4, g["bodyPos"][a][:3], g["bodyPos"][b][:3], g["bodyInvMass"][a],
            g["bodyInvMass"][b], g["bodyInvInertiaWorld"][a], g["bodyInvInertiaWorld"][b], dt)
        np.testing.assert_allclose(jc[:npts], jac[:npts], rtol=2e-6, atol=1e-7)
        np.testing.assert_allclose(bb[:npts], g["b"][j][:npts], rtol=2e-6, atol=1e-7)
        np.testing.assert_allclose(center, g["center"][j][:3], rtol=0, atol=2e-6)
        # friction: the recorded revision spanned the tangent plane with
        # t0 = normalize(n x (p0 - center)), t1 = normalize(t0 x n) (the
        # alternative left in ST/Solver.cpp:403-408); the current source,
        # restated here, uses btPlaneSpace1. The two bases differ by a
        # rotation about n, which leaves the sum of the two directions'
        # effective-mass denominators unchanged.
        rec = g["fJacCoeffInv"][j].astype(np.float64)
        np.testing.assert_allclose(1.0 / fj[0] + 1.0 / fj[1], 1.0 / rec[0] + 1.0 / rec[1], rtol=2e-6)
        n3 = -lin[:3].astype(np.float64)
        t0 = np.cross(n3, g["worldPos"][j][0][:3] - g["center"][j][:3])
        t0 /= np.linalg.norm(t0)
        t1 = np.cross(t0, n3)
        t1 /= np.linalg.norm(t1)
        pa, pb = g["bodyPos"][a][:3], g["bodyPos"][b][:3]
        for t, want in ((t0, rec[0]), (t1, rec[1])):
            ang0 = -np.cross(g["center"][j][:3] - pa, t)
            ang1 = np.cross(g["center"][j][:3] - pb, t)
            den = (g["bodyInvMass"][a] + ang0 @ g["bodyInvInertiaWorld"][a] @ ang0 + g["bodyInvMass"][b] +
                   ang1 @ g["bodyInvInertiaWorld"][b] @ ang1)
            np.testing.assert_allclose(-1.0 / den, want, rtol=2e-5)
        checked += 1
    assert checked == n


def test_recorded_batches_share_no_dynamic_body_within_a_cell():
    g = _golden()
    row = {int(b): k for k, b in enumerate(g["bodies"])}
    dyn = lambda body: g["bodyInvMass"][row[int(body)]] != 0
    cells = 0
    for cnt, off in zip(g["cellCount"], g["cellOffset"]):
        if cnt == 0:
            continue
        cells += 1
        bi = g["batchIdx"][off:off + cnt]
        assert np.all(np.diff(bi) >= 0) and bi.max() < int(g["maxBatch"])
        for b in np.unique(bi):
            bodies = [x for j in np.nonzero(bi == b)[0] for x in g["bodyAB"][off + j] if dyn(x)]
            assert len(bodies) == len(set(bodies))
    assert cells == int(np.count_nonzero(g["cellCount"]))


def _check_colouring(o, inv_mass):
    contacts = o.contacts()
    cb = o.gs_batches()
    m = len(cb)
    assert m == len(contacts["normal"]) > 0
    cell, batch = cb[:, 0], cb[:, 1]
    cls = (cell & 1) + 2 * ((cell // 16) & 1)
    assert np.all(batch >= 0)
    A = np.abs(contacts["bodyA"])
    B = np.abs(contacts["bodyB"])
    dyn_bodies = [[x for x in (A[k], B[k]) if inv_mass[x] != 0] for k in range(m)]
    # rank inside a class: (cell, manifold) order
    rank = np.lexsort((np.arange(m), cell, cls))
    pos = np.empty(m, np.int64)
    pos[rank] = np.arange(m)
    for c in range(4):
        members = np.nonzero(cls == c)[0]
        if len(members) == 0:
            continue
        nb = batch[members].max() + 1
        groups = [members[batch[members] == b] for b in range(nb)]
        for grp in groups:
            assert len(grp) > 0  # batches are dense
            bodies = [x for k in grp for x in dyn_bodies[k]]
            assert len(bodies) == len(set(bodies))
        # greedy: a manifold in batch b was blocked in every earlier batch
        for b in range(1, nb):
            for k in groups[b]:
                mine = set(dyn_bodies[k])
                for e in range(b):
                    assert any(pos[k2] < pos[k] and mine & set(dyn_bodies[k2]) for k2 in groups[e]), (k, b, e)
    return int(batch.max()) + 1


@pytest.mark.parametrize("name", ["pile", "stack"])
def test_colouring_is_valid_and_greedy(host_ctx, name):
    sc = scenes.random_pile(41, n=160, hull_frac=0.5) if name == "pile" else scenes.c1(dims=(6, 6, 6))
    w, o = host_oracle(host_ctx, sc, flags=2)
    o.step(12 if name == "pile" else 30)
    nb = _check_colouring(o, np.asarray(sc.mass, np.float64) > 0)
    assert nb >= 2


def _column(height=3):
    """A column of unit cubes standing on the ground, faces touching."""
    return scenes.lattice_scene(f"column_{height}", 7, (1, height, 1), 1.0, lambda n: np.ones(n, np.int32),
                                lambda n: np.ones(n), lambda n: np.full(n, 0.6), jitter=0.0, yaw=False, y0=0.0,
                                config=dict(cellSize=1.0, gridDims=(16, 16, 16), maxPairs=4096),
                                extra_shapes=[scenes.box_vertices(0.5, 0.5, 0.5)])


def test_column_rests_under_the_batched_solver(host_ctx):
    sc = _column(3)
    w, o = host_oracle(host_ctx, sc, flags=2)
    o.step(120)
    pos, _, lin, ang = o.state()
    dyn = np.asarray(sc.mass) > 0
    # the boxes stay stacked where they stood: the column neither sinks nor
    # drifts, and comes to rest
    np.testing.assert_allclose(pos[dyn, 1], [0.5, 1.5, 2.5], atol=0.03)
    # sideways drift of the top box stays within 2 cm over the 2 s; its
    # exact value depends on the order in which the solver visits the
    # contact points, which follows the start vertex of each face's cycle
    assert np.abs(pos[dyn][:, [0, 2]]).max() < 0.02
    assert np.abs(lin[dyn, :3]).max() < 0.05 and np.abs(ang[dyn, :3]).max() < 0.05
