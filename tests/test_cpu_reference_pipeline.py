"""The reference's CPU rigid-body pipeline (bullet2 btDiscreteDynamicsWorld,
compiled from the reference sources into oracle/_ref/libb3bullet.so), the
CPU baseline bench.py times: it loads, builds the workload scenes and
settles a cube stack on its ground."""
import numpy as np
import pytest

import oracle
from experiments_b200 import scenes

pytestmark = pytest.mark.skipif(oracle.bullet_lib() is None, reason="oracle/_ref/libb3bullet.so not built")


def test_cube_stack_settles_on_the_ground():
    sc = scenes.c1(dims=(4, 4, 4))
    w = oracle.ReferenceCpuWorld(sc)
    w.step(180)
    p = w.positions()
    dyn = np.asarray(sc.mass) > 0
    assert p[dyn, 1].min() > 0.45          # resting on the ground (top at y = 0)
    assert p[dyn, 1].max() < 4 * 1.05 + 1.5
    w.close()


def test_batched_worlds_are_independent():
    sc = scenes.random_pile(3, n=24, worlds=3)
    w = oracle.ReferenceCpuWorld(sc)
    w.step(30)
    p = w.positions()
    one = scenes.select_worlds(sc, [1])
    w1 = oracle.ReferenceCpuWorld(one)
    w1.step(30)
    assert np.array_equal(p[np.asarray(sc.world) == 1], w1.positions())
