"""Failure paths of the device step, made to happen without faulting the GPU.

* A bounded wait that runs out: the persistent Jacobi solve's grid barrier
  gets a short poll limit, and block 0 arrives at its first barrier late (a
  bounded sleep, b3_set_wait_limits). The waiting blocks give up, the
  launch ends, and the host learns of it: b3_get_counters and b3_read_state
  return B3_ERR_TIMEOUT with counters.timeouts > 0. After b3_reset_counters
  and default limits the world steps normally again.
* The grid broadphase's capacity caps, which are part of the reference's
  semantics (maxPairsPerBody - 1 pairs kept per body, the first
  maxBodiesPerCell entries of a cell searched: G3/bt3dGridBroadphaseOCL.cl:
  129-131, 159-162): a dense pile with both caps small gives the oracle's
  truncated pair set bit for bit, with the same nonzero overflow counts.
"""
import numpy as np
import pytest

from experiments_b200 import b3, scenes

from helpers import make_pair, pair_set

pytestmark = pytest.mark.gpu

B3_ERR_TIMEOUT = 6


def test_jacobi_barrier_wait_runs_out_and_is_reported(ctx):
    sc = scenes.c1(dims=(8, 8, 8))
    w = scenes.build_world(ctx, sc, useGraph=0)
    t = w.tuning()
    w.set_tuning([t[0], t[1], 128, t[3], 4, t[5], 0, 0])  # grid-barrier Jacobi, many blocks
    w.stepSimulation(40)  # on the ground: the solve has manifolds
    rc, c = w.counters_status()
    assert rc == 0 and c["timeouts"] == 0 and c["numManifolds"] > 0
    w.set_wait_limits(spin_limit=32, hold_micros=20000)
    w.stepSimulation(1)
    rc, c = w.counters_status()
    assert rc == B3_ERR_TIMEOUT
    assert c["timeouts"] > 0
    with pytest.raises(b3.B3Error):
        w.read_state()
    # the context stays usable: default limits, errors cleared, steps resume
    w.set_wait_limits()
    w.reset_counters()
    w.stepSimulation(5)
    rc, c = w.counters_status()
    assert rc == 0 and c["timeouts"] == 0
    pos, _, lin, _ = w.read_state()
    assert np.isfinite(pos).all() and np.isfinite(lin).all()
    w.close()


@pytest.mark.parametrize("caps", [(4, 2), (3, 64), (32, 2)])
def test_broadphase_caps_truncate_like_the_oracle(ctx, caps):
    per_body, per_cell = caps
    sc = scenes.random_pile(71, n=300, hull_frac=0.5)
    w, o = make_pair(ctx, sc, maxPairsPerBody=per_body, maxBodiesPerCell=per_cell)
    w.stepSimulation(30)
    pos, quat, lin, ang = w.read_state()
    o.set_state_f32(pos, quat, lin, ang)
    for s in ("aabbs", "broadphase"):
        w.stage(s)
        o.stage(s)
    gk, gv = w.sorted_hash()
    ok, ov = o.sorted_hash()
    assert np.array_equal(gk, ok) and np.array_equal(gv, ov)
    gp, op = w.pairs(), o.pairs()
    assert len(gp) == len(op) and pair_set(gp) == pair_set(op)
    c = w.counters()
    po, co = o.overflow()
    assert c["pairOverflow"] == po and c["cellOverflow"] == co
    if per_body < 32:
        assert po > 0
    if per_cell < 64:
        assert co > 0
    w.close()
