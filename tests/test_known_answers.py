"""Analytic known-answer contacts for two unit cubes, on the oracle (CPU)
and on the product (GPU). They pin the SAT axis choice and the clipping of
P2/sat.cl:497-635 and P2/satClipHullContacts.cl:556-611, for which the
reference ships no host port: face-face stacked, face-face offset (clipped),
face-face yawed 45 degrees (octagon, reduced to 4 points) and edge-edge
crossed (single point, cross-product normal)."""
import numpy as np
import pytest

from experiments_b200 import scenes
from helpers import host_oracle

H = 0.5
S2 = np.sqrt(2.0) / 2.0


def _scene(pos_upper, q_lower, q_upper):
    shapes = [scenes.box_vertices(H, H, H)]
    return scenes.Scene("known_answer", shapes, np.array([0, 0]), np.array([1.0, 1.0], np.float32),
                        np.array([[0, 0, 0], pos_upper], np.float32),
                        np.array([q_lower, q_upper], np.float32), np.array([0.5, 0.5], np.float32),
                        np.zeros(2, np.int32), np.zeros((2, 3), np.float32), np.zeros((2, 3), np.float32),
                        config=dict(cellSize=1.0, gridDims=(16, 16, 16)))


ID = [0, 0, 0, 1]


def _yaw(a):
    return [0, np.sin(a / 2), 0, np.cos(a / 2)]


CASES = {
    # upper cube 0.1 into the lower one: B's top face corners, depth -0.1
    "stacked": (_scene([0, 0.9, 0], ID, ID),
                dict(normal=[0, -1, 0], depth=-0.1,
                     points=[[x, H, z] for x in (-H, H) for z in (-H, H)])),
    # shifted by half a cube: the top face clipped to x in [0, 0.5]
    "offset": (_scene([0.5, 0.95, 0], ID, ID),
               dict(normal=[0, -1, 0], depth=-0.05,
                    points=[[x, H, z] for x in (0.0, H) for z in (-H, H)])),
    # yawed 45 degrees: the overlap is the regular octagon with vertices at
    # (+-0.5, +-0.5 tan 22.5) and (+-0.5 tan 22.5, +-0.5); 4 of them are kept
    "yawed": (_scene([0, 0.9, 0], ID, _yaw(np.pi / 4)),
              dict(normal=[0, -1, 0], depth=-0.1, octagon=True)),
    # crossed edges: upper rotated 45 deg about z, lower 45 deg about x; the
    # axis is the cross product of the two edges (y), one point on the
    # lower cube's top edge
    "edge_edge": (_scene([0, 2 * S2 - 0.05, 0], [np.sin(np.pi / 8), 0, 0, np.cos(np.pi / 8)],
                         [0, 0, np.sin(np.pi / 8), np.cos(np.pi / 8)]),
                  dict(normal=[0, -1, 0], edge=True)),
}


def _check(name, normal, pts, n_pts):
    sc, exp = CASES[name]
    assert np.allclose(normal[:3], exp["normal"], atol=1e-6), (name, normal)
    p = np.asarray(pts)[:n_pts]
    if "points" in exp:
        assert n_pts == 4
        want = np.array(exp["points"])
        for q in p:
            assert np.min(np.max(np.abs(want - q[:3]), axis=1)) < 1e-5, (name, q)
        assert np.allclose(p[:, 3], exp["depth"], atol=1e-5)
    if exp.get("octagon"):
        t = H * np.tan(np.pi / 8)
        octo = [[sx * H, H, sz * t] for sx in (-1, 1) for sz in (-1, 1)] + \
               [[sx * t, H, sz * H] for sx in (-1, 1) for sz in (-1, 1)]
        octo = np.array(octo)
        assert n_pts == 4
        for q in p:
            assert np.min(np.max(np.abs(octo - q[:3]), axis=1)) < 1e-5, (name, q)
        assert np.allclose(p[:, 3], exp["depth"], atol=1e-5)
    if exp.get("edge"):
        assert n_pts == 1
        q = p[0]
        assert abs(q[1] - S2) < 1e-5 and abs(q[2]) < 1e-5 and abs(q[0]) <= 0.1, q
        assert q[3] < 0


@pytest.mark.parametrize("name", sorted(CASES))
def test_known_answer_oracle(host_ctx, name):
    sc, _ = CASES[name]
    w, o = host_oracle(host_ctx, sc)
    o.stage("aabbs")
    o.stage("broadphase")
    o.stage("narrowphase")
    c = o.contacts()
    assert len(c["normal"]) == 1
    _check(name, c["normal"][0], c["pos"][0], int(c["normal"][0][3]))
    w.close()
    o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_known_answer_gpu(ctx, name):
    sc, _ = CASES[name]
    w = scenes.build_world(ctx, sc, useGraph=0)
    w.stage("aabbs")
    w.stage("broadphase")
    w.stage("narrowphase")
    c = w.contacts()
    assert len(c["normal"]) == 1
    _check(name, c["normal"][0], c["pos"][0], int(c["normal"][0][3]))
    w.close()
