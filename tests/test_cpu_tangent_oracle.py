"""The FP64 tangent-linear oracle (forward-mode dual numbers through the
whole step) against FP64 central differences of the FP64 oracle, on the
differentiable throw: it is the exact derivative the adjoint tests compare
the device gradients with."""
import numpy as np
import pytest

from adjoint_harness import oracle_run, oracle_state_at, oracle_tangent, random_seeds
from experiments_b200 import scenes


@pytest.mark.parametrize("t0,steps", [(10, 1), (30, 1), (10, 4)])
def test_tangent_matches_fp64_central_differences(host_ctx, t0, steps):
    sc = scenes.c4(worlds=4)
    rng = np.random.default_rng(5 + t0 + steps)
    st = oracle_state_at(host_ctx, sc, t0)
    seeds = random_seeds(sc, rng)
    dyn = np.asarray(sc.mass) > 0
    checked = 0
    for kind in ("lin", "ang", "mass", "friction"):
        comps = 3 if kind in ("lin", "ang") else 1
        d = rng.normal(size=(sc.n, comps)) * dyn[:, None]
        dd = d if comps == 3 else d[:, 0]
        tan, h0 = oracle_tangent(host_ctx, sc, st, steps, seeds, kind, dd)
        # two step sizes: the smaller has less truncation error, the larger
        # less cancellation; the tangent agrees with the better of the two
        rels, oks = [], []
        for eps in (1e-5, 1e-7):
            lp, hp = oracle_run(host_ctx, sc, st, steps, seeds, kind, dd, eps)
            lm, hm = oracle_run(host_ctx, sc, st, steps, seeds, kind, dd, -eps)
            fd = (lp - lm) / (2 * eps)
            rels.append(np.abs(tan - fd) / np.maximum(np.abs(fd), 1e-6))
            oks.append((hp == h0).all(1) & (hm == h0).all(1))
        same = oks[0] | oks[1]
        rel = np.where(oks[0] & oks[1], np.minimum(rels[0], rels[1]), np.where(oks[0], rels[0], rels[1]))
        assert same.sum() >= 2, kind
        assert np.all(rel[same] < 1e-5), (kind, rel, same)
        checked += int(same.sum())
    assert checked >= 8


def test_chained_one_step_tangents_equal_the_multi_step_tangent(host_ctx):
    """Carrying the tangent from step to step through the pose and velocity
    seeds reproduces the tangent of one multi-step run when the recorded
    trajectory is the oracle's own: the machinery that linearises the FP64
    step along another (the device's) trajectory."""
    from adjoint_harness import chained_tangent, make_oracle
    sc = scenes.c4(worlds=4)
    steps = 12
    st = oracle_state_at(host_ctx, sc, 20)
    o, _ = make_oracle(host_ctx, sc)
    o.set_state_f64(*st)
    traj = [[a.copy() for a in st]]
    for _ in range(steps):
        o.step(1)
        traj.append(o.state())
    o.close()
    rng = np.random.default_rng(17)
    seeds = random_seeds(sc, rng)
    dyn = np.asarray(sc.mass) > 0
    for kind in ("lin", "ang", "mass", "friction"):
        comps = 3 if kind in ("lin", "ang") else 1
        d = rng.normal(size=(sc.n, comps)) * dyn[:, None]
        dd = d if comps == 3 else d[:, 0]
        whole, _ = oracle_tangent(host_ctx, sc, st, steps, seeds, kind, dd)
        chained, dev_pos, dev_vel = chained_tangent(host_ctx, sc, traj, seeds, kind, dd)
        assert dev_pos.max() == 0 and dev_vel.max() == 0
        assert np.allclose(chained, whole, rtol=1e-10, atol=1e-12 * np.abs(whole).max()), (kind, chained, whole)
