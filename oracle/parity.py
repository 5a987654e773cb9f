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


def manifold_differences(gc, oc, limit=20):
    """The manifolds (by pair slot) where the device and the oracle differ:
    present on one side only, other point counts or bodies, or points or
    normal beyond the bars. Each entry holds the slot, the kind and both
    records (bodies, normal with its count in w, points with depth in w)."""
    gi = {int(p): k for k, p in enumerate(gc["pairIndex"])}
    oi = {int(p): k for k, p in enumerate(oc["pairIndex"])}

    def rec(c, k):
        if k is None:
            return None
        n = int(c["normal"][k, 3])
        return {"bodies": [int(c["bodyA"][k]), int(c["bodyB"][k])], "normal": c["normal"][k].tolist(),
                "points": c["pos"][k][:n].tolist()}

    out = []
    for p in sorted(set(gi) | set(oi)):
        kg, ko = gi.get(p), oi.get(p)
        kind = None
        if kg is None:
            kind = "oracle only"
        elif ko is None:
            kind = "device only"
        else:
            ng, no = int(gc["normal"][kg, 3]), int(oc["normal"][ko, 3])
            if ng != no or gc["bodyA"][kg] != oc["bodyA"][ko] or gc["bodyB"][kg] != oc["bodyB"][ko]:
                kind = "counts or bodies"
            else:
                dp = float(np.abs(gc["pos"][kg][:ng] - oc["pos"][ko][:ng]).max()) if ng else 0.0
                dn = float(np.abs(gc["normal"][kg, :3] - oc["normal"][ko, :3]).max())
                if dp > POS_TOL or dn > NRM_TOL:
                    kind = "points %.3g m, normal %.3g" % (dp, dn)
        if kind:
            out.append({"slot": p, "kind": kind, "device": rec(gc, kg), "oracle": rec(oc, ko)})
            if len(out) >= limit:
                break
    return out


def _state_errors(a, b, sel):
    return {"pos_err_m": float(np.abs(a[0][sel, :3] - b[0][sel, :3]).max()),
            "lin_vel_err_mps": float(np.abs(a[2][sel, :3] - b[2][sel, :3]).max()),
            "ang_vel_err_radps": float(np.abs(a[3][sel, :3] - b[3][sel, :3]).max()),
            "quat_err": float(np.abs(a[1][sel] - b[1][sel]).max())}


def one_step_report(w, o, dynamic=None, make_oracle=None):
    """Hand the device world's current state to the oracle, run one step on
    both stage by stage, and report every comparison. `dynamic` (bool per
    body) restricts the state errors to dynamic bodies (static ones do not
    move). Leaves both worlds one step further on.

    With make_oracle (f32 -> a fresh oracle world of the same scene) the
    solve and integration are also checked on their own: the FP64 oracle
    and its FP32 build each solve from the device's contacts. The device
    against the FP64 oracle there is the solver's error; the FP32 build
    against the FP64 oracle is the envelope of the same algorithm evaluated
    in FP32 (a Jacobi solve of a densely coupled, penetrating system
    amplifies rounding over its iterations, in any FP32 implementation)."""
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
    rep["pair_overflow"] = int(po)
    w.stage("narrowphase")
    o.stage("narrowphase")
    gc, oc = w.contacts(), o.contacts()
    same_set, same_counts, wp, wn = _contact_errors(gc, oc)
    rep["manifolds"] = int(len(gc["normal"]))
    rep["manifold_set_equal"] = same_set and same_counts
    rep["manifold_differences"] = manifold_differences(gc, oc)
    rep["contact_point_err_m"] = wp
    rep["normal_err"] = wn
    w.stage("solve")
    o.stage("solve")
    w.stage("integrate")
    o.stage("integrate")
    gs = w.read_state()
    os_ = o.state()
    sel = np.ones(len(gs[0]), bool) if dynamic is None else np.asarray(dynamic, bool)
    rep.update(_state_errors(gs, os_, sel))
    c = w.counters()
    rep["timeouts"] = int(c["timeouts"])
    narrow_ok = bool(rep["aabbs_bit_exact"] and rep["keys_bit_exact"] and rep["permutation_bit_exact"]
                     and rep["pairs_bit_exact"] and rep["manifold_set_equal"] and wp <= POS_TOL and wn <= NRM_TOL)
    rep["narrowphase_within_bars"] = narrow_ok
    tol = {"pos_err_m": POS_TOL, "lin_vel_err_mps": VEL_TOL, "ang_vel_err_radps": VEL_TOL, "quat_err": QUAT_TOL}
    if make_oracle is not None:
        solved = []
        for f32 in (False, True):
            ox = make_oracle(f32)
            ox.set_state_f32(pos, quat, lin, ang)
            ox.stage("aabbs")
            ox.set_contacts(gc)
            ox.stage("solve")
            ox.stage("integrate")
            solved.append(ox.state())
            ox.close()
        solver = _state_errors(gs, solved[0], sel)
        env = _state_errors(solved[1], solved[0], sel)
        # how far the FP64 solve moves when given the device's contacts
        # instead of its own (both within the contact bars): the problem's
        # sensitivity to those differences, not an arithmetic error
        sens = _state_errors(solved[0], os_, sel)
        rep["solver_err"] = solver
        rep["fp32_envelope"] = env
        rep["contact_sensitivity"] = sens
        # the bars: the stated tolerance, or twice what FP32 arithmetic of the
        # same algorithm shows on this state, whichever is larger; the whole
        # step also carries the sensitivity to the contact differences
        bars = {k: max(tol[k], 2.0 * env[k]) for k in tol}
        step_bars = {k: max(tol[k], 2.0 * (env[k] + sens[k])) for k in tol}
        rep["bars_used"] = bars
        rep["step_bars_used"] = step_bars
        rep["solver_within_bars"] = all(solver[k] <= bars[k] for k in tol)
        rep["step_within_bars"] = all(rep[k] <= step_bars[k] for k in tol)
    else:
        rep["step_within_bars"] = all(rep[k] <= tol[k] for k in tol)
    rep["within_bars"] = bool(narrow_ok and rep["step_within_bars"] and rep.get("solver_within_bars", True)
                              and rep["timeouts"] == 0)
    rep["check_s"] = time.perf_counter() - t0
    return rep
