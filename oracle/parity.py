"""ORACLE — test infrastructure only.

One step of a device world checked stage by stage against the oracle from
the device's own FP32 state. tests/ assert on the report; bench.py puts it
beside the throughput it measured, so the error quoted with a number is the
error of the run that produced it.

The stages follow CLPhysicsDemo::stepSimulation
(opencl/gpu_rigidbody_pipeline2/CLPhysicsDemo.cpp:740-943): world AABBs,
cell hash + sort + pair search, narrowphase, solve, integrate. The checks
are the oracle contract: AABBs, sorted keys, the sort permutation and the
pair set bit-exact; contact points within 1e-5 m and normals within 1e-4;
positions within 1e-5 m and velocities within 1e-4 m/s after the step.
"""
import time

import numpy as np

POS_TOL = 1e-5
NRM_TOL = 1e-4
VEL_TOL = 1e-4
QUAT_TOL = 1e-5


def _contact_errors(gc, oc):
    """Manifolds matched by pair slot: (same manifold set, same point counts
    and bodies, worst point error, worst normal error)."""
    gi = {int(p): k for k, p in enumerate(gc["pairIndex"])}
    oi = {int(p): k for k, p in enumerate(oc["pairIndex"])}
    same_set = set(gi) == set(oi)
    same_counts = True
    worst_p = worst_n = 0.0
    if len(gi):
        common = np.array(sorted(set(gi) & set(oi)), np.int64)
        kg = np.array([gi[int(p)] for p in common], np.int64)
        ko = np.array([oi[int(p)] for p in common], np.int64)
        ng = gc["normal"][kg, 3].astype(np.int64)
        no = oc["normal"][ko, 3].astype(np.int64)
        same_counts = bool(np.array_equal(ng, no)) and bool(np.array_equal(gc["bodyA"][kg], oc["bodyA"][ko])) \
            and bool(np.array_equal(gc["bodyB"][kg], oc["bodyB"][ko]))
        worst_n = float(np.abs(gc["normal"][kg, :3] - oc["normal"][ko, :3]).max())
        # points beyond each manifold's count are unused slots
        mask = np.arange(4)[None, :] < np.minimum(ng, no)[:, None]
        # xyz and the depth in w
        d = np.abs(gc["pos"][kg][:, :, :4] - oc["pos"][ko][:, :, :4]).max(axis=2)
        worst_p = float(d[mask].max()) if mask.any() else 0.0
    return same_set, same_counts, worst_p, worst_n


def one_step_report(w, o, dynamic=None):
    """Hand the device world's current state to the oracle, run one step on
    both stage by stage, and report every comparison. `dynamic` (bool per
    body) restricts the state errors to dynamic bodies (static ones do not
    move). Leaves both worlds one step further on."""
    t0 = time.perf_counter()
    pos, quat, lin, ang = w.read_state()
    o.set_state_f32(pos, quat, lin, ang)
    rep = {}
    w.stage("aabbs")
    o.stage("aabbs")
    rep["aabbs_bit_exact"] = bool(np.array_equal(w.aabbs().view(np.uint32), o.aabbs().view(np.uint32)))
    w.stage("broadphase")
    o.stage("broadphase")
    gk, gv = w.sorted_hash()
    ok, ov = o.sorted_hash()
    rep["keys_bit_exact"] = bool(np.array_equal(gk, ok))
    rep["permutation_bit_exact"] = bool(np.array_equal(gv, ov))
    gp, op = np.asarray(w.pairs()).reshape(-1, 2), np.asarray(o.pairs()).reshape(-1, 2)
    rep["pairs"] = int(len(gp))
    rep["pairs_bit_exact"] = len(gp) == len(op) and \
        set(map(tuple, gp.tolist())) == set(map(tuple, op.tolist()))
    c = w.counters()
    po, co = o.overflow()
    rep["overflow_match"] = c["pairOverflow"] == po and c["cellOverflow"] == co
    w.stage("narrowphase")
    o.stage("narrowphase")
    gc, oc = w.contacts(), o.contacts()
    same_set, same_counts, wp, wn = _contact_errors(gc, oc)
    rep["manifolds"] = int(len(gc["normal"]))
    rep["manifold_set_equal"] = same_set and same_counts
    rep["contact_point_err_m"] = wp
    rep["normal_err"] = wn
    w.stage("solve")
    o.stage("solve")
    w.stage("integrate")
    o.stage("integrate")
    gp4, gq, gl, ga = w.read_state()
    op4, oq, ol, oa = o.state()
    sel = np.ones(len(gp4), bool) if dynamic is None else np.asarray(dynamic, bool)
    rep["pos_err_m"] = float(np.abs(gp4[sel, :3] - op4[sel, :3]).max())
    rep["lin_vel_err_mps"] = float(np.abs(gl[sel, :3] - ol[sel, :3]).max())
    rep["ang_vel_err_radps"] = float(np.abs(ga[sel, :3] - oa[sel, :3]).max())
    rep["quat_err"] = float(np.abs(gq[sel] - oq[sel]).max())
    c = w.counters()
    rep["timeouts"] = int(c["timeouts"])
    rep["within_bars"] = bool(rep["aabbs_bit_exact"] and rep["keys_bit_exact"] and rep["permutation_bit_exact"]
                              and rep["pairs_bit_exact"] and rep["manifold_set_equal"]
                              and wp <= POS_TOL and wn <= NRM_TOL and rep["pos_err_m"] <= POS_TOL
                              and rep["lin_vel_err_mps"] <= VEL_TOL and rep["ang_vel_err_radps"] <= VEL_TOL
                              and rep["quat_err"] <= QUAT_TOL and rep["timeouts"] == 0)
    rep["check_s"] = time.perf_counter() - t0
    return rep
