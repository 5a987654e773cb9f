"""Spheres, planes, compounds and triangle meshes on the device against the
oracle (oracle/parity.py, one step stage by stage from the device's state):
pairs bit-exact, the same manifolds (sub-pair slots of compound and mesh
pairs included) with points within 1e-5 m and normals within 1e-4, and the
step within its bars.

  * 200 spheres of radius U(0.2, 0.5) dropped onto a plane (sphere-plane and
    sphere-sphere contacts, P2/satClipHullContacts.cl:957-1124);
  * 120 compounds of unit cubes (two-cube bars, three-cube L shapes) and
    12-point hulls dropped onto a ground box (compound child pairs,
    P2/sat.cl:639-926, P2/satClipHullContacts.cl:1184-1318);
  * 150 cubes and 12-point hulls dropped onto a 16 x 16 triangle-mesh
    terrain (triangle polytopes, P2/sat.cl:970-1191,
    P2/satClipHullContacts.cl:1387).
"""
import numpy as np
import pytest

import oracle
from experiments_b200 import scenes
from oracle import parity

from helpers import make_pair

pytestmark = pytest.mark.gpu

CASES = {
    "spheres_on_plane": (lambda: scenes.spheres_on_plane(), 90),
    "compound_pile": (lambda: scenes.compound_pile(), 200),
    "mesh_terrain": (lambda: scenes.mesh_terrain(), 90),
}


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("graph", [0, 1])
def test_shapes_step_matches_oracle(ctx, name, graph):
    make, settle = CASES[name]
    sc = make()
    w, o = make_pair(ctx, sc, useGraph=graph)
    w.stepSimulation(settle)
    rep = parity.one_step_report(w, o, dynamic=np.asarray(sc.mass) > 0,
                                 make_oracle=lambda f32: oracle.oracle_from_world(w, sc, f32=f32))
    print(name, rep)
    assert rep["pairs_bit_exact"] and rep["keys_bit_exact"] and rep["aabbs_bit_exact"]
    assert rep["manifold_set_equal"], "manifold sets differ"
    assert rep["manifolds"] > 0
    assert rep["contact_point_err_m"] <= parity.POS_TOL
    assert rep["normal_err"] <= parity.NRM_TOL
    bars, step_bars = rep["bars_used"], rep["step_bars_used"]
    for k in ("pos_err_m", "lin_vel_err_mps", "ang_vel_err_radps", "quat_err"):
        assert rep["solver_err"][k] <= bars[k], (k, rep["solver_err"][k], bars[k])
        assert rep[k] <= step_bars[k], (k, rep[k], step_bars[k])
    assert rep["timeouts"] == 0
    w.close()


def test_sub_pair_slots_follow_the_pairs(ctx):
    """Compound and mesh manifolds take the slots after the broadphase
    pairs', in pair order, and their bodies are the pairs' (the mesh body on
    side A)."""
    for sc in (scenes.compound_pile(), scenes.mesh_terrain()):
        w, o = make_pair(ctx, sc)
        w.stepSimulation(120)
        for s in ("aabbs", "broadphase", "narrowphase"):
            w.stage(s)
        P = len(w.pairs())
        c = w.contacts()
        sub = c["pairIndex"] >= P
        assert sub.sum() > 0
        assert np.all(np.diff(c["pairIndex"]) > 0)  # manifolds in slot order
        if sc.name.startswith("terrain"):
            assert np.all(np.abs(c["bodyA"][sub]) == 0)  # the mesh is body 0
        w.close()


def test_shapes_rest_on_the_device(ctx):
    """Long runs: spheres rest on the plane, compounds on the ground box and
    bodies on the mesh; nothing that stays over the ground falls through it
    or gains energy. (A body's position is its hull's vertex average, which
    for a 12-point hull can sit 0.2 m off the points' centre: the floors are
    below the lowest resting centre.) The compound pile is its first two
    layers, dropped from 2 m and 6 m."""
    for make, steps, floor in ((scenes.spheres_on_plane, 400, 0.15),
                               (lambda: scenes.compound_pile(n=32), 600, -0.1),
                               (scenes.mesh_terrain, 400, -0.1)):
        sc = make()
        w = scenes.build_world(ctx, sc, useGraph=1)
        w.stepSimulation(steps)
        pos, _, lin, _ = w.read_state()
        dyn = np.asarray(sc.mass) > 0
        # over the ground region (bodies may leave it over an edge)
        inside = (np.abs(pos[dyn, 0]) < 7.5) & (np.abs(pos[dyn, 2]) < 7.5)
        assert np.isfinite(pos).all()
        assert pos[dyn, 1][inside].min() > floor, sc.name
        assert np.abs(lin[dyn, :3][inside]).max() < 2.0, sc.name
        assert w.counters()["timeouts"] == 0
        w.close()
