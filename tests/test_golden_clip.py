"""The reference's own recorded test vector for its clipping kernel
(testdata/clipFacesAndContactReductionKernel.7z, decoded into
tests/golden/clip_faces_k11.npz by tests/golden/make_golden.py): for each of
the 380 recorded pairs the oracle's restatement of
clipFacesAndContactReductionKernel (satClipHullContacts.cl:1845-1952) must
reproduce the kernel's output points, count and depths."""
import ctypes as C
import os

import numpy as np

import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "clip_faces_k11.npz")
D = C.POINTER(C.c_double)


def test_oracle_clip_reproduces_the_reference_test_vector():
    g = np.load(GOLDEN)
    L = oracle.lib()
    n = len(g["pairs"])
    assert n == 380
    worst = 0.0
    for k in range(n):
        nA, nB, nOut = int(g["numVertsA"][k]), int(g["numVertsB"][k]), int(g["numOut"][k])
        vA = np.ascontiguousarray(g["vertsA"][k][:nA].astype(np.float64))
        nrm = np.ascontiguousarray(g["normalA"][k].astype(np.float64))
        pB = np.ascontiguousarray(g["polyB"][k][:nB].astype(np.float64))
        out = np.zeros((64, 4))
        cnt = L.or_clip_face_world(vA.ctypes.data_as(D), nA, nrm.ctypes.data_as(D), pB.ctypes.data_as(D), nB,
                                   -1e30, 0.02, out.ctypes.data_as(D))
        assert cnt == nOut, (k, cnt, nOut)
        ref = g["points"][k][:nOut].astype(np.float64)
        # FP32 kernel vs FP64 restatement on FP32 inputs, world coordinates of a few metres
        err = np.max(np.abs(out[:cnt] - ref)) if cnt else 0.0
        assert err < 2e-6, (k, err)
        worst = max(worst, err)
    assert worst < 2e-6
