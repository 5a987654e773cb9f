"""Parity at the benchmarked sizes, in the contact-rich part of each run.

The device steps the full workload scene to the window the benchmark times,
then the oracle takes the device's FP32 state and both run one step, stage
by stage (oracle/parity.py): AABBs, sorted cell keys, the sort permutation
and the pair set bit-exact; the same manifolds with contact points within
1e-5 m and normals within 1e-4; positions within 1e-5 m and velocities
within 1e-4 m/s. Where the step's Jacobi solve amplifies rounding (a densely
coupled, penetrating pile: the FP32 build of the oracle itself then
departs from the FP64 oracle by more than those bars), the solve is checked
on its own from the device's contacts against twice that FP32 envelope,
measured on the same state in the same test; the whole step's bar adds the
solve's sensitivity to the contact differences (the FP64 solve from the
device's contacts against the FP64 solve from the oracle's).

  * 131,072 mixed hulls (1/2 cubes, 1/4 12-point hulls, 1/4 42-vertex
    icospheres) on a 64x32x64 lattice, after 300 steps: every layer has
    landed and the pile is in contact.
  * 4,096 batched worlds of log-uniform[8, 512] piles, after 300 steps.
  * 1,048,576 unit cubes (128x64x128 lattice), after 24 of its 32 steps:
    the bottom layer is on the ground and the yawed neighbours touch.
"""
import numpy as np
import pytest

from experiments_b200 import scenes
import oracle
from oracle import parity

from helpers import make_pair

pytestmark = pytest.mark.gpu

CASES = {
    # name: (scene factory, device steps before the checked step)
    "c2_131k_settled": (lambda: scenes.c2(), 300),
    "c3_4096_worlds_settled": (lambda: scenes.c3(), 300),
    "c5_1m_cubes": (lambda: scenes.c5(), 24),
}


@pytest.mark.parametrize("name", list(CASES))
def test_full_size_step_matches_oracle(ctx, name):
    make, settle = CASES[name]
    sc = make()
    w, o = make_pair(ctx, sc, useGraph=1)
    w.stepSimulation(settle)
    rep = parity.one_step_report(w, o, dynamic=np.asarray(sc.mass) > 0,
                                 make_oracle=lambda f32: oracle.oracle_from_world(w, sc, f32=f32))
    print(name, {k: v for k, v in rep.items()})
    assert rep["aabbs_bit_exact"], "AABBs differ"
    assert rep["keys_bit_exact"], "sorted keys differ"
    assert rep["permutation_bit_exact"], "sort permutation differs"
    assert rep["pairs_bit_exact"], "pair sets differ"
    assert rep["overflow_match"]
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
