"""The batched Gauss-Seidel solver (B3_WORLD_BATCHED_GS_SOLVER) on the device
against its FP64 restatement.

Bit-exact: every manifold's cell and batch (the colouring is integer work on
the same FP32 positions and the same manifold order). From the same FP32
state: one step's positions within 1e-5 m and velocities within 1e-4 m/s;
accumulated impulses within 1e-4 of the restatement's, relative to the
largest. The device colouring is valid and greedy on a workload scene, and
graph replays are bitwise deterministic (the counting sort places each
batch's constraints in any order; batches share no dynamic body, so the
result cannot depend on it), whatever the width of the cooperative grid."""
import numpy as np
import pytest

from experiments_b200 import scenes

from helpers import make_pair
from test_cpu_gs import _check_colouring, _column

pytestmark = pytest.mark.gpu

POS_TOL = 1e-5
VEL_TOL = 1e-4
GS = 2  # B3_WORLD_BATCHED_GS_SOLVER


def _scenes():
    return {
        "column": _column(4),
        "c1_8": scenes.c1(dims=(8, 8, 8)),
        "pile_hulls": scenes.random_pile(11, n=200, hull_frac=0.5),
        "pile_batched": scenes.random_pile(12, n=40, worlds=16, hull_frac=0.5),
        "c2_small": scenes.c2(dims=(16, 8, 16)),
    }


SCENES = list(_scenes().keys())


@pytest.fixture(scope="module")
def scene_cache():
    return _scenes()


@pytest.mark.parametrize("name", SCENES)
def test_one_step_matches_oracle(ctx, scene_cache, name):
    sc = scene_cache[name]
    w, o = make_pair(ctx, sc, flags=GS)
    w.stepSimulation(3)
    pos, quat, lin, ang = w.read_state()
    o.set_state_f32(pos, quat, lin, ang)
    w.stepSimulation(1)
    o.step(1)
    # the colouring: bit-exact
    gb, ob = w.gs_batches(), o.gs_batches()
    assert len(gb) == len(ob) > 0
    assert np.array_equal(gb, ob), f"{int((gb != ob).any(axis=1).sum())} manifolds differ in cell or batch"
    # the impulses and the state
    gi = w.gs_constraints()
    oi = o.gs_applied()
    scale = max(1.0, float(np.abs(oi).max()))
    assert np.abs(gi["applied"] - oi[:, :4]).max() <= 1e-4 * scale
    assert np.abs(gi["fApplied"] - oi[:, 4:]).max() <= 1e-4 * scale
    gp, gq, gl, ga = w.read_state()
    op, oq, ol, oa = o.state()
    assert np.abs(gp[:, :3] - op[:, :3]).max() <= POS_TOL
    assert np.abs(gl[:, :3] - ol[:, :3]).max() <= VEL_TOL
    assert np.abs(ga[:, :3] - oa[:, :3]).max() <= VEL_TOL
    assert np.abs(gq - oq).max() <= 1e-5
    assert w.counters()["timeouts"] == 0


def test_device_colouring_is_valid_and_greedy(ctx, scene_cache):
    sc = scene_cache["c2_small"]
    w, _ = make_pair(ctx, sc, flags=GS)
    w.stepSimulation(4)
    o_batches = w.gs_batches()

    class View:
        def contacts(self):
            return w.contacts()

        def gs_batches(self):
            return o_batches

    nb = _check_colouring(View(), np.asarray(sc.mass) > 0)
    assert nb >= 2


def _world_inv_inertia(quat, local3):
    """R diag(local) R^T per body (FP64)."""
    x, y, z, w = (quat[:, k].astype(np.float64) for k in range(4))
    R = np.stack([np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
                  np.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], -1),
                  np.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1)], 1)
    return np.einsum("nik,nk,njk->nij", R, local3.astype(np.float64), R)


def test_constraints_follow_setconstraint4(ctx, scene_cache):
    """Constraint4 records of the device against setConstraint4 restated on
    the device's own contacts and the pre-solve state."""
    import oracle
    sc = scene_cache["pile_hulls"]
    w, o = make_pair(ctx, sc, flags=GS)
    w.stepSimulation(3)
    w.stage("aabbs")  # gravity enters the velocities here; positions do not move before the solve
    w.stage("broadphase")
    w.stage("narrowphase")
    pos, quat, lin, ang = w.read_state()
    w.stage("solve")
    c = w.contacts()
    g = w.gs_constraints()
    dyn = np.asarray(sc.mass) > 0
    inv_mass = np.where(dyn, 1.0 / np.where(dyn, np.asarray(sc.mass, np.float64), 1.0), 0.0)
    local = w.inertias()[:, :3]
    iw = _world_inv_inertia(quat, local)
    iw[~dyn] = 0.0
    dt = float(w.cfg.dt)
    assert len(c["normal"]) > 20
    for k in range(len(c["normal"])):
        A, B = abs(int(c["bodyA"][k])), abs(int(c["bodyB"][k]))
        jc, bb, center, fj = oracle.gs_constraint(c["pos"][k], c["normal"][k], pos[A, :3], pos[B, :3],
                                                  inv_mass[A], inv_mass[B], iw[A], iw[B], dt)
        n = int(c["normal"][k][3])
        np.testing.assert_allclose(g["jacCoeffInv"][k][:n], jc[:n], rtol=1e-5, atol=1e-7)
        np.testing.assert_allclose(g["b"][k][:n], bb[:n], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(g["center"][k][:3], center, atol=1e-5)
        np.testing.assert_allclose(g["fJacCoeffInv"][k], fj, rtol=1e-5, atol=1e-7)
        assert g["bodyA"][k] == A and g["bodyB"][k] == B


def test_graph_replay_is_bitwise_deterministic(ctx):
    sc = scenes.random_pile(21, n=300, hull_frac=0.5)
    states = []
    for _ in range(2):
        w, _ = make_pair(ctx, sc, flags=GS)
        w.stepSimulation(8)
        states.append(w.read_state())
        w.close()
    for a, b in zip(*states):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("name", ["pile_hulls", "c2_small"])
def test_grid_widths_agree_bitwise(ctx, scene_cache, name):
    """The two cooperative grid widths of the solve (solverMode 0 and 1) run
    the same batches in the same order: the same bits."""
    sc = scene_cache[name]
    states = []
    for mode in (0, 1):
        w, _ = make_pair(ctx, sc, flags=GS)
        t = w.tuning()
        t[6] = mode
        w.set_tuning(t)
        w.stepSimulation(6)
        states.append(w.read_state())
        assert w.counters()["timeouts"] == 0
        w.close()
    for a, b in zip(*states):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_adjoint_form_refuses_the_batched_solver(ctx, scene_cache):
    from experiments_b200 import b3
    w, _ = make_pair(ctx, scene_cache["column"], flags=GS)
    with pytest.raises(b3.B3Error):
        b3.Adjoint(w, 2, 1)
