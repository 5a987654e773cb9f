"""The two forms of the grid pair search give the same output bit for bit.

Form 0 runs one thread per body over its 27 neighbour cells; form 1 runs one
warp per body with a lane per cell and rebuilds the sequential per-body cap
(maxPairsPerBody - 1 pairs, one overflow count per cell that has more,
G3/bt3dGridBroadphaseOCL.cl:129-131, 159-162) from a warp scan of the cell
counts. Both must give the same pair list in the same order, the same pair
count and the same overflow counters, and the oracle's pair set; whole steps
then give the same bits. Cases: the parity scenes, small caps on a dense
pile, a world with 41 large bodies (two 32-wide ballots in the large-body
pass, with and without the per-body cap reached there) and the full
131,072-body mixed-hull scene after it has landed.
"""
import numpy as np
import pytest

from experiments_b200 import scenes

from helpers import make_pair, pair_set

pytestmark = pytest.mark.gpu


def _large_slab_pile():
    """A 300-body pile whose first 40 dynamic bodies are 20 m x 1 m x 20 m
    slabs (large proxies: half-diagonal above maxSmallProxySize / 2)."""
    sc = scenes.random_pile(73, n=300, hull_frac=0.5)
    sc.shape = sc.shape.copy()
    sc.shape[1:41] = 0
    return sc


CASES = {
    # name: (scene factory, steps before the search, world config overrides,
    #        pair overflow expected, cell overflow expected)
    "c1_8": (lambda: scenes.c1(dims=(8, 8, 8)), 40, {}, False, False),
    "pile_hulls": (lambda: scenes.random_pile(11, n=200, hull_frac=0.5), 30, {}, False, False),
    "pile_batched": (lambda: scenes.random_pile(12, n=40, worlds=16, hull_frac=0.5), 30, {}, False, False),
    "c2_small": (lambda: scenes.c2(dims=(16, 8, 16)), 60, {}, False, False),
    "caps_4_2": (lambda: scenes.random_pile(71, n=300, hull_frac=0.5), 30,
                 dict(maxPairsPerBody=4, maxBodiesPerCell=2), True, True),
    "caps_3_64": (lambda: scenes.random_pile(71, n=300, hull_frac=0.5), 30,
                  dict(maxPairsPerBody=3, maxBodiesPerCell=64), True, False),
    "caps_32_2": (lambda: scenes.random_pile(71, n=300, hull_frac=0.5), 30,
                  dict(maxPairsPerBody=32, maxBodiesPerCell=2), False, True),
    "large_slabs_cap_64": (_large_slab_pile, 0, dict(maxPairsPerBody=64, maxPairs=400000), False, False),
    "large_slabs_cap_8": (_large_slab_pile, 0, dict(maxPairsPerBody=8, maxPairs=400000), True, False),
}


def _with_form(w, form):
    t = w.tuning()
    t[8] = form
    w.set_tuning(t)


@pytest.mark.parametrize("name", list(CASES))
def test_pair_search_forms_agree_and_match_oracle(ctx, name):
    make, steps, over, pair_ovf, cell_ovf = CASES[name]
    sc = make()
    out = []
    for form in (0, 1):
        w, o = make_pair(ctx, sc, **over)
        _with_form(w, form)
        w.stepSimulation(steps)
        pos, quat, lin, ang = w.read_state()
        o.set_state_f32(pos, quat, lin, ang)
        for s in ("aabbs", "broadphase"):
            w.stage(s)
            o.stage(s)
        gp = np.asarray(w.pairs())
        c = w.counters()
        op = o.pairs()
        po, co = o.overflow()
        assert len(gp) == len(op) and pair_set(gp) == pair_set(op)
        assert c["pairOverflow"] == po and c["cellOverflow"] == co
        assert c["timeouts"] == 0
        out.append((gp, c, (pos, quat, lin, ang)))
        w.close()
    (p0, c0, s0), (p1, c1, s1) = out
    assert np.array_equal(p0, p1), "pair lists differ in content or order"
    for k in ("numPairs", "pairOverflow", "cellOverflow"):
        assert c0[k] == c1[k], k
    for a, b in zip(s0, s1):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    if pair_ovf:
        assert c0["pairOverflow"] > 0
    if cell_ovf:
        assert c0["cellOverflow"] > 0


def test_pair_search_forms_agree_on_the_full_mixed_hull_scene(ctx):
    sc = scenes.c2()
    states, pairs = [], []
    for form in (0, 1):
        w = scenes.build_world(ctx, sc, useGraph=1)
        _with_form(w, form)
        w.stepSimulation(120)
        states.append(w.read_state())
        w.stage("aabbs")
        w.stage("broadphase")
        pairs.append(np.asarray(w.pairs()))
        c = w.counters()
        assert c["timeouts"] == 0 and c["numPairs"] > 100000
        w.close()
    assert np.array_equal(pairs[0], pairs[1])
    for a, b in zip(*states):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
