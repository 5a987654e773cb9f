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
