"""The sweep-and-prune restatement (gpu_rigidbody_pipeline2's default
broadphase) against brute-force AABB overlap, on the reference's own
recorded kernel input (tests/golden/sap_kernel_args.npz) and on workload
scenes. A sweep over proxies sorted by min x must find exactly the
overlapping pairs, each oriented by sorted order; large (static) proxies
pair with every small proxy they overlap."""
import os

import numpy as np
import pytest

import oracle
from experiments_b200 import scenes
from helpers import host_oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _overlap(a, b):
    """Inclusive AABB overlap of records a (k x 8) against b (m x 8)."""
    return ((a[:, None, 0] <= b[None, :, 4]) & (b[None, :, 0] <= a[:, None, 4]) &
            (a[:, None, 1] <= b[None, :, 5]) & (b[None, :, 1] <= a[:, None, 5]) &
            (a[:, None, 2] <= b[None, :, 6]) & (b[None, :, 2] <= a[:, None, 6]))


def _brute_sorted(s):
    """Pairs (id_i, id_j), i < j in sorted order, of overlapping records."""
    ids = s[:, 3].view(np.int32)
    out = []
    for c0 in range(0, len(s), 512):
        blk = _overlap(s[c0:c0 + 512], s)
        ii, jj = np.nonzero(blk)
        ii = ii + c0
        keep = jj > ii
        out.append(np.stack([ids[ii[keep]], ids[jj[keep]]], 1))
    return np.concatenate(out) if out else np.zeros((0, 2), np.int32)


def test_reference_vector_pairs_are_the_overlapping_pairs():
    g = np.load(os.path.join(GOLDEN, "sap_kernel_args.npz"))
    s = g["sorted_aabbs"]
    assert len(s) == int(g["numObjects"]) and int(g["axis"]) == 0
    assert np.all(np.diff(s[:, 0]) >= 0)  # the recorded array is sorted by min x
    p = oracle.sap_sorted_pairs(s, 0)
    assert len(p) > 0 and len(p) < int(g["maxPairs"])
    assert set(map(tuple, p.tolist())) == set(map(tuple, _brute_sorted(s).tolist()))
    assert len(set(map(tuple, p.tolist()))) == len(p)  # no duplicates


@pytest.mark.parametrize("name", ["c1_8", "pile"])
def test_world_pairs_are_the_overlapping_pairs(host_ctx, name):
    sc = scenes.c1(dims=(8, 8, 8)) if name == "c1_8" else scenes.random_pile(31, n=120, hull_frac=0.5)
    w, o = host_oracle(host_ctx, sc, flags=1)
    o.step(3)
    o.stage("aabbs")
    o.stage("broadphase")
    pairs = o.pairs()
    a = o.aabbs()
    dyn = np.asarray(sc.mass) > 0
    keys, vals = o.sorted_hash()
    assert np.array_equal(np.sort(vals), np.where(dyn)[0])
    order = {int(b): k for k, b in enumerate(vals)}
    # small-small: every overlapping pair once, earlier sorted proxy first
    small = a[vals]
    exp = set(map(tuple, _brute_sorted(small).tolist()))
    # large-small: (static id, dynamic id)
    lg = np.where(~dyn)[0]
    ov = _overlap(a[lg], a[vals])
    li, sj = np.nonzero(ov)
    exp |= set(zip(lg[li].tolist(), vals[sj].astype(np.int64).tolist()))
    got = list(map(tuple, pairs.tolist()))
    assert set(got) == exp and len(got) == len(exp)
    # pair list order: by the sorted small proxy (second id of a large pair,
    # first id of a small pair)
    key = [order[b] if not dyn[a_] else order[a_] for a_, b in got]
    assert key == sorted(key)
    w.close()
    o.close()


def test_sap_flag_rules(host_ctx):
    """The SAP broadphase takes one world; unknown flag bits are refused."""
    from experiments_b200 import b3
    sc = scenes.random_pile(5, n=20, worlds=2)
    with pytest.raises(b3.B3Error):
        b3.PhysicsWorld(host_ctx, scenes.world_config(sc, flags=1))
    with pytest.raises(b3.B3Error):
        b3.PhysicsWorld(host_ctx, scenes.world_config(scenes.random_pile(5, n=20), flags=4))
    for flags in (1, 2, 3):  # SAP, batched Gauss-Seidel, both
        w = b3.PhysicsWorld(host_ctx, scenes.world_config(scenes.random_pile(5, n=20), flags=flags))
        w.close()
