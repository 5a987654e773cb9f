"""Stage-by-stage parity of the CUDA step with the oracle.

Bit-exact: world AABBs, sorted cell keys and permutation, pair sets (from
the same FP32 state). Contacts: points within 1e-5 m, normals within 1e-4.
One step: positions within 1e-5 m, velocities within 1e-4 m/s."""
import numpy as np
import pytest

from experiments_b200 import scenes

from helpers import make_pair, pair_set

pytestmark = pytest.mark.gpu

POS_TOL = 1e-5
NRM_TOL = 1e-4
VEL_TOL = 1e-4


def _scenes():
    return {
        "c1_8": scenes.c1(dims=(8, 8, 8)),
        "c1_full": scenes.c1(),
        "pile_hulls": scenes.random_pile(11, n=200, hull_frac=0.5),
        "pile_batched": scenes.random_pile(12, n=40, worlds=16, hull_frac=0.5),
        "c2_small": scenes.c2(dims=(16, 8, 16)),
    }


SCENES = list(_scenes().keys())


@pytest.fixture(scope="module")
def scene_cache():
    return _scenes()


def _run_broadphase(w, o):
    w.stage("aabbs")
    w.stage("broadphase")
    o.stage("aabbs")
    o.stage("broadphase")


@pytest.mark.parametrize("name", SCENES)
def test_aabbs_keys_pairs_bit_exact(ctx, scene_cache, name):
    sc = scene_cache[name]
    w, o = make_pair(ctx, sc)
    _run_broadphase(w, o)
    ga, oa = w.aabbs(), o.aabbs()
    assert np.array_equal(ga.view(np.uint32), oa.view(np.uint32)), "AABBs differ"
    gk, gv = w.sorted_hash()
    ok, ov = o.sorted_hash()
    assert np.array_equal(gk, ok), "sorted keys differ"
    assert np.array_equal(gv, ov), "sort permutation differs"
    gp, op = w.pairs(), o.pairs()
    assert len(gp) == len(op)
    assert pair_set(gp) == pair_set(op)
    c = w.counters()
    po, co = o.overflow()
    assert c["pairOverflow"] == po and c["cellOverflow"] == co
    assert c["timeouts"] == 0


def _match_contacts(gc, oc):
    gi = {int(p): k for k, p in enumerate(gc["pairIndex"])}
    oi = {int(p): k for k, p in enumerate(oc["pairIndex"])}
    assert set(gi) == set(oi), f"manifold sets differ: {len(set(gi) ^ set(oi))}"
    worst_p = worst_n = 0.0
    for p, kg in gi.items():
        ko = oi[p]
        n = int(gc["normal"][kg][3])
        assert n == int(oc["normal"][ko][3])
        assert gc["bodyA"][kg] == oc["bodyA"][ko] and gc["bodyB"][kg] == oc["bodyB"][ko]
        worst_n = max(worst_n, float(np.abs(gc["normal"][kg][:3] - oc["normal"][ko][:3]).max()))
        worst_p = max(worst_p, float(np.abs(gc["pos"][kg][:n] - oc["pos"][ko][:n]).max()))
    return worst_p, worst_n


@pytest.mark.parametrize("name", SCENES)
def test_contacts_match_oracle(ctx, scene_cache, name):
    sc = scene_cache[name]
    w, o = make_pair(ctx, sc)
    # advance both a few steps of free fall so piles settle into contact, then
    # hand the device state to the oracle so both narrowphases see one state
    w.stepSimulation(2 if name.startswith("pile") else 1)
    pos, quat, lin, ang = w.read_state()
    o.set_state_f32(pos, quat, lin, ang)
    w.stage("aabbs")
    w.stage("broadphase")
    w.stage("narrowphase")
    o.stage("aabbs")
    o.set_pairs(w.pairs())
    o.stage("narrowphase")
    gc, oc = w.contacts(), o.contacts()
    assert len(gc["normal"]) > 0
    wp, wn = _match_contacts(gc, oc)
    assert wp <= POS_TOL, f"contact point error {wp}"
    assert wn <= NRM_TOL, f"normal error {wn}"


@pytest.mark.parametrize("name", SCENES)
def test_one_step_matches_oracle(ctx, scene_cache, name):
    sc = scene_cache[name]
    w, o = make_pair(ctx, sc)
    w.stepSimulation(3)
    pos, quat, lin, ang = w.read_state()
    o.set_state_f32(pos, quat, lin, ang)
    w.stepSimulation(1)
    o.step(1)
    gp, gq, gl, ga = w.read_state()
    op, oq, ol, oa = o.state()
    assert np.abs(gp[:, :3] - op[:, :3]).max() <= POS_TOL
    assert np.abs(gl[:, :3] - ol[:, :3]).max() <= VEL_TOL
    assert np.abs(ga[:, :3] - oa[:, :3]).max() <= VEL_TOL
    assert np.abs(gq - oq).max() <= 1e-5


def test_graph_replay_is_bitwise_deterministic(ctx):
    sc = scenes.random_pile(21, n=300, hull_frac=0.5)
    a = scenes.build_world(ctx, sc)
    b = scenes.build_world(ctx, sc, useGraph=1)
    a.stepSimulation(20)
    b.stepSimulation(20)
    sa, sb = a.read_state(), b.read_state()
    for x, y in zip(sa, sb):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


def test_long_run_aggregates(ctx):
    """Stacking chaos makes trajectories diverge; compare aggregates."""
    sc = scenes.c1(dims=(6, 6, 6))
    w, o = make_pair(ctx, sc)
    steps = 240
    w.stepSimulation(steps)
    o.step(steps)
    gp, _, gl, _ = w.read_state()
    op, _, ol, _ = o.state()
    dyn = sc.mass > 0
    ke_g = 0.5 * np.sum(sc.mass[dyn] * np.sum(gl[dyn, :3] ** 2, 1))
    ke_o = 0.5 * np.sum(sc.mass[dyn] * np.sum(ol[dyn, :3] ** 2, 1))
    h_g, h_o = gp[dyn, 1].mean(), op[dyn, 1].mean()
    # mean height within 5 cm, kinetic energies of the same order
    assert abs(h_g - h_o) < 0.05
    assert np.isfinite(ke_g) and np.isfinite(ke_o)
    assert ke_g < 3.0 * ke_o + 5.0 and ke_o < 3.0 * ke_g + 5.0
    # maximum penetration into the ground (bottom face below y = 0)
    pen_g = 0.5 - gp[dyn, 1].min()
    pen_o = 0.5 - op[dyn, 1].min()
    assert abs(pen_g - pen_o) < 0.05
    # bodies rest on the ground, none fell through
    assert gp[dyn, 1].min() > 0.3 and op[dyn, 1].min() > 0.3


@pytest.mark.gpu
def test_autotune_keeps_state_and_results(ctx):
    """The autotuner restores the body state it started from, and the
    chosen launch shapes do not change the results (bit for bit)."""
    sc = scenes.random_pile(41, n=64, worlds=8, hull_frac=0.5)
    a = scenes.build_world(ctx, sc, useGraph=1)
    b = scenes.build_world(ctx, sc, useGraph=1)
    a.stepSimulation(5)
    b.stepSimulation(5)
    before = a.read_state()
    a.autotune(2)
    after = a.read_state()
    for x, y in zip(before, after):
        assert np.array_equal(x, y)
    t = a.tuning()
    # trials: 3 narrowphase CTA sizes, 2 clip forms, 2 pair search forms,
    # then the Jacobi shapes jointly (grid mode: 3 CTA sizes x 4 caps x 2
    # gathers; per-world mode: 3 x 2)
    assert t[5] == 3 + 2 + 2 + 24 + 6
    assert t[0] in (1, 2, 4) and t[6] in (0, 1) and t[2] in (64, 128, 256) and t[4] in (1, 2, 4, 8)
    assert t[7] in (0, 1) and t[8] in (0, 1) and t[9] in (0, 1)
    a.stepSimulation(10)
    b.stepSimulation(10)
    for x, y in zip(a.read_state(), b.read_state()):
        assert np.array_equal(x, y)
    a.close()
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
def test_gathered_averages_match_one_at_a_time(ctx, mode):
    """The Jacobi variant that gathers each body's copies four loads at a
    time gives the one-at-a-time results bit for bit, in both solver
    modes."""
    sc = scenes.random_pile(47, n=48, worlds=6, hull_frac=0.5)
    a = scenes.build_world(ctx, sc, useGraph=1)
    b = scenes.build_world(ctx, sc, useGraph=1)
    t = a.tuning()
    a.set_tuning([t[0], t[1], t[2], t[3], t[4], t[5], mode, 0])
    b.set_tuning([t[0], t[1], t[2], t[3], t[4], t[5], mode, 1])
    a.stepSimulation(30)
    b.stepSimulation(30)
    for x, y in zip(a.read_state(), b.read_state()):
        assert np.array_equal(x, y)
    a.close()
    b.close()


@pytest.mark.gpu
def test_per_world_solver_matches_grid_solver(ctx):
    """The batched solver variant (one block per world, block barriers) gives
    the grid-barrier solver's results bit for bit."""
    sc = scenes.random_pile(43, n=48, worlds=12, hull_frac=0.5)
    a = scenes.build_world(ctx, sc, useGraph=1)
    b = scenes.build_world(ctx, sc, useGraph=1)
    t = a.tuning()
    a.set_tuning([t[0], t[1], t[2], t[3], t[4], t[5], 0])
    b.set_tuning([t[0], t[1], t[2], t[3], t[4], t[5], 1])
    a.stepSimulation(30)
    b.stepSimulation(30)
    for x, y in zip(a.read_state(), b.read_state()):
        assert np.array_equal(x, y)
    a.close()
    b.close()
