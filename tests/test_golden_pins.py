"""The reference pins of tests/test_cpu_pins.py replayed from committed
fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py from the
reference's own code), so they run where the reference sources and
oracle/_ref are absent:

* hull_pins.npz: btConvexUtility (P1/btConvexUtility.cpp:31-270) on every
  shape of the plain and batched workloads, against the product's hulls;
* jacobi_pins.npz: btPgsJacobiSolver::solveContacts
  (P2/btPgsJacobiSolver.cpp:171-189) on the manifolds of three settled
  piles, against the oracle's solver on the same inputs."""
import os

import numpy as np
import pytest

from experiments_b200 import b3, scenes
from helpers import host_oracle
import test_cpu_pins as pins

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_hulls_match_the_recorded_reference_tables(host_ctx):
    g = np.load(os.path.join(GOLDEN, "hull_pins.npz"))
    k = 0
    for sc in (scenes.c2(dims=(4, 2, 4)), scenes.c3(worlds=4)):
        w = b3.PhysicsWorld(host_ctx, scenes.world_config(sc))
        scenes.register_scene(w, sc)
        sh = w.shapes()
        for s, pts in enumerate(sc.shapes):
            assert np.array_equal(np.asarray(pts, np.float32), g[f"h{k}_points"])
            flat = g[f"h{k}_faces"]
            faces, i = [], 0
            while i < len(flat):
                faces.append(flat[i + 1:i + 1 + flat[i]])
                i += 1 + flat[i]
            assert pins.check_hull_against_reference(pts, sh, s, g[f"h{k}_verts"], g[f"h{k}_planes"], faces,
                                                     g[f"h{k}_edges"])
            k += 1
        w.close()
    assert k == int(g["count"])


@pytest.mark.parametrize("seed", [21, 22, 23])
def test_oracle_solver_matches_the_recorded_reference_solve(host_ctx, seed):
    g = np.load(os.path.join(GOLDEN, "jacobi_pins.npz"))
    sc = scenes.random_pile(seed, n=40, velocity=0.5)
    w, o = host_oracle(host_ctx, sc)
    body = g[f"s{seed}_body"].view(np.dtype([("pos", "<f4", 4), ("quat", "<f4", 4), ("lin", "<f4", 4),
                                            ("ang", "<f4", 4), ("shape", "<u4"), ("invMass", "<f4"),
                                            ("rest", "<f4"), ("fric", "<f4")]))
    c4 = g[f"s{seed}_contacts"].view(np.dtype([("pos", "<f4", (4, 4)), ("nrm", "<f4", 4), ("rest", "<u2"),
                                              ("fric", "<u2"), ("batch", "<i4"), ("a", "<i4"), ("b", "<i4")]))
    o.set_state_f32(body["pos"], body["quat"], body["lin"], body["ang"])
    # the inverse masses and local inverse inertias the reference solve was given
    inert = g[f"s{seed}_inertia"]
    o.set_params_f64(inv_mass=body["invMass"].astype(np.float64),
                     inv_inertia3=inert[:, [12, 17, 22]].astype(np.float64))
    o.set_contacts(dict(pos=c4["pos"].astype(np.float64), normal=c4["nrm"].astype(np.float64),
                        friction=(c4["fric"].astype(np.float32) / np.float32(65535.0)).astype(np.float64),
                        pairIndex=np.arange(len(c4)), bodyA=g[f"s{seed}_bodyA"], bodyB=g[f"s{seed}_bodyB"]))
    lin, ang = o.solve_velocities()
    dyn = np.asarray(sc.mass) > 0
    rl, ra = g[f"s{seed}_lin"], g[f"s{seed}_ang"]
    assert np.max(np.abs(lin[dyn, :3] - rl[dyn, :3]) / (1 + np.abs(rl[dyn, :3]))) < 5e-6
    assert np.max(np.abs(ang[dyn, :3] - ra[dyn, :3]) / (1 + np.abs(ra[dyn, :3]))) < 5e-6
    w.close()
    o.close()
