"""The narrowphase stages by eight-lane groups give the warp kernels' results bit for bit.

k_np_clip_groups runs face selection, Sutherland-Hodgman clipping, the
depth filter, the contact reduction and the Contact4 write of four pairs per
warp, eight lanes each, with the arithmetic of k_np_clip (warp per pair);
pairs whose faces or clipped polygon exceed its 16-vertex tables are passed
to k_np_clip. k_np_refine_groups and k_np_exact_groups do the same for the
float-float ranking of up to 8 near-tied axes and for the float-float clip
of pairs whose FP32 clip was in doubt, passing the rest to k_np_refine and
k_np_exact. The two forms (b3_set_tuning index 9) must give the same
state bits step after step, on the parity scenes, on the compound and mesh
sub-pairs, and on prism columns built to reach the hand-over: 20-gon caps
resting on 20-gon caps (faces of 20 vertices) and 12-gon caps turned by 15
degrees against each other (clipped polygons of up to 24 vertices), also
with coincident cap edges. The contacts of the columns without coincident
edges also match the oracle.
"""
import numpy as np
import pytest

from experiments_b200 import scenes

from helpers import make_pair

pytestmark = pytest.mark.gpu

POS_TOL = 1e-5
NRM_TOL = 1e-4


def _prism(m, r, h):
    a = 2.0 * np.pi * np.arange(m) / m
    top = np.stack([r * np.cos(a), np.full(m, h), r * np.sin(a)], 1)
    bot = top.copy()
    bot[:, 1] = -h
    return np.concatenate([top, bot]).astype(np.float32)


def _prism_columns(aligned=False):
    """Six columns of four prisms resting cap on cap: 20-gon caps (faces
    past the groups' 16-vertex tables) and 12-gon caps turned by 15 degrees
    against each other (clipped polygons of up to 24 vertices). Unless
    aligned, the 20-gon levels turn by 9 degrees against each other and every
    level shifts by a few millimetres, so no edge of one cap lies on a side
    plane of the other; aligned, the 20-gon caps coincide, where the clip's
    inside / outside decisions are exact ties."""
    shapes = [scenes.box_vertices(10.0, 0.5, 10.0), _prism(20, 0.5, 0.25), _prism(12, 0.5, 0.25)]
    shape, pos, yaw = [], [], []
    for col in range(6):
        for level in range(4):
            shape.append(1 if col < 3 else 2)
            shift = 0.0 if aligned else 0.003 * level
            # caps 1 mm into each other, so the first step has contacts
            pos.append([(col - 2.5) * 1.5 + shift, 0.25 + level * 0.499, -0.5 * shift])
            step = np.pi / 12 if col >= 3 else (0.0 if aligned else np.pi / 20)
            yaw.append((level % 2) * step)
    n = len(shape)
    parts = [scenes.ground(),
             scenes._bodies(shape, np.ones(n), pos, scenes.yaw_quat(np.asarray(yaw)), np.full(n, 0.6), np.zeros(n))]
    return scenes.Scene(name="prism_columns", shapes=shapes, num_worlds=1, config={}, steps=1,
                        **scenes._concat(parts))


CASES = {
    # name: (scene factory, steps)
    "c1_8": (lambda: scenes.c1(dims=(8, 8, 8)), 60),
    "pile_hulls": (lambda: scenes.random_pile(11, n=200, hull_frac=0.5), 40),
    "pile_batched": (lambda: scenes.random_pile(12, n=40, worlds=16, hull_frac=0.5), 40),
    "c2_small": (lambda: scenes.c2(dims=(16, 8, 16)), 80),
    "compound_pile": (lambda: scenes.compound_pile(), 60),
    "mesh_terrain": (lambda: scenes.mesh_terrain(), 60),
    "prism_columns": (_prism_columns, 30),
    "prism_columns_aligned": (lambda: _prism_columns(aligned=True), 30),
    # resting, nearly aligned cubes: the float-float ranking and clip stages
    # carry many pairs
    "cube_lattice": (lambda: scenes.c5(dims=(24, 8, 24), steps=24), 24),
}


def _with_clip_form(w, form):
    t = w.tuning()
    t[9] = form
    w.set_tuning(t)


@pytest.mark.parametrize("name", list(CASES))
def test_clip_forms_agree_bitwise(ctx, name):
    make, steps = CASES[name]
    sc = make()
    out = []
    for form in (0, 1):
        w = scenes.build_world(ctx, sc, useGraph=1)
        _with_clip_form(w, form)
        w.stepSimulation(steps)
        c = w.counters()
        assert c["timeouts"] == 0 and c["numManifolds"] > 0
        out.append((w.read_state(), {k: c[k] for k in ("numManifolds", "numContactPoints", "refinedAxes",
                                                        "refinedClips", "clipOverflow")}))
        w.close()
    (s0, c0), (s1, c1) = out
    assert c0 == c1
    for a, b in zip(s0, s1):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    if name == "cube_lattice":
        assert c0["refinedAxes"] > 100 and c0["refinedClips"] > 100


def test_prism_contacts_match_oracle_in_both_forms(ctx):
    sc = _prism_columns()
    for form in (0, 1):
        w, o = make_pair(ctx, sc)
        _with_clip_form(w, form)
        for s in ("aabbs", "broadphase", "narrowphase"):
            w.stage(s)
        o.stage("aabbs")
        o.set_pairs(w.pairs())
        o.stage("narrowphase")
        gc, oc = w.contacts(), o.contacts()
        gi = {int(p): k for k, p in enumerate(gc["pairIndex"])}
        oi = {int(p): k for k, p in enumerate(oc["pairIndex"])}
        assert set(gi) == set(oi) and len(gi) >= 20  # every cap on cap, every prism on the ground
        for p, kg in gi.items():
            ko = oi[p]
            n = int(gc["normal"][kg][3])
            assert n == int(oc["normal"][ko][3])
            assert np.abs(gc["normal"][kg][:3] - oc["normal"][ko][:3]).max() <= NRM_TOL
            assert np.abs(gc["pos"][kg][:n] - oc["pos"][ko][:n]).max() <= POS_TOL
        w.close()
