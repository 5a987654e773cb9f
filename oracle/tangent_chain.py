"""Test infrastructure (the checker, never the product): gradients of the
adjoint form against the FP64 tangent-linear oracle chained along a
recorded trajectory.

Over a long run of the differentiable throw the scene is chaotic: the
oracle's own FP64 trajectory leaves the device's FP32 one, and so does the
derivative along it. Chaining the exact FP64 one-step Jacobians at the
device's recorded states removes that sensitivity: the tangent is carried
from step to step through the pose and velocity seeds of the tangent-linear
build (`or_set_tangent` + `or_set_tangent_pose`), each step taken from the
recorded state. What differs from the device's reverse sweep is then the
adjoint's own arithmetic, plus any step whose discrete choices (contacts,
axes, clamp masks) the FP64 step makes differently from the device. Such
worlds are detected two ways: from the values of the same FP64 steps, and
from choices that flip when the recorded states are perturbed at the size of
the device's own one-step deviation from FP64.
"""
import numpy as np


def world_functional(scene, state, seeds):
    """Per-world linear functional sum <seed, state> over (pos, quat, lin, ang)."""
    wid = np.asarray(scene.world)
    out = np.zeros(scene.num_worlds)
    for k in range(4):
        cols = 4 if k == 1 else 3
        contrib = np.sum(seeds[k][:, :cols] * state[k][:, :cols], axis=1)
        np.add.at(out, wid, contrib)
    return out


def param_tangents(scene, inv_inertia3, kind, delta):
    """`set_tangent` keyword seeds of one body-parameter set along delta:
    "mass" (invMass = 1/m, and the inverse inertia is invMass times a shape
    factor) or "friction"; velocities are seeded as state."""
    m = np.asarray(scene.mass, np.float64)
    dyn = m > 0
    im = np.where(dyn, 1.0 / np.where(dyn, m, 1), 0.0)
    delta = np.asarray(delta, np.float64)
    if kind == "mass":
        dim = np.where(dyn, -delta / np.where(dyn, m, 1) ** 2, 0.0)
        return dict(inv_mass=dim, inv_inertia3=inv_inertia3 * np.where(dyn, dim / np.where(dyn, im, 1), 0.0)[:, None])
    if kind == "friction":
        return dict(friction=delta)
    return {}


def com_seeds(scene, final_pos):
    """Seeds of the throw's loss, the sum over worlds of the squared distance
    of the world's centre of mass (dynamic bodies, mass-weighted) from its
    target: d loss / d pos_i = 2 (com - target) m_i / M."""
    m = np.asarray(scene.mass, np.float64)
    wid = np.asarray(scene.world)
    seeds = [np.zeros((scene.n, 4)) for _ in range(4)]
    for k in range(scene.num_worlds):
        s = (wid == k) & (m > 0)
        com = (final_pos[s, :3] * m[s, None]).sum(0) / m[s].sum()
        seeds[0][s, :3] = 2 * (com - scene.extra["target"][k])[None, :] * (m[s, None] / m[s].sum())
    return seeds


def chained_tangent(o, inv_inertia3, scene, traj, seeds, kind, delta):
    """Directional derivative of the per-world functional of the last state
    of traj = [s_0, ..., s_T] (each (pos, quat, lin, ang), n x 4) along delta
    ("lin" / "ang": n x 3 initial velocities; "mass" / "friction": n), the
    FP64 tangent-linear step taken from each recorded state in turn.

    `o` is a tangent-linear OracleWorld of the scene. Returns (per-world
    derivatives, per-world largest position deviation and largest velocity
    deviation over the steps of the FP64 step from s_t against s_{t+1})."""
    n = scene.n
    params = param_tangents(scene, inv_inertia3, kind, delta)
    dpos, dquat, dlin, dang = [np.zeros((n, 4)) for _ in range(4)]
    if kind == "lin":
        dlin[:, :3] = delta
    elif kind == "ang":
        dang[:, :3] = delta
    wid = np.asarray(scene.world)
    dev_pos = np.zeros(scene.num_worlds)
    dev_vel = np.zeros(scene.num_worlds)
    for t in range(len(traj) - 1):
        o.set_state_f64(*[np.asarray(a, np.float64) for a in traj[t]])
        o.set_tangent(lin=dlin, ang=dang, **params)
        o.set_tangent_pose(dpos, dquat)
        o.step(1)
        dpos, dquat, dlin, dang = o.tangent()
        nxt = o.state()
        ep = np.abs(nxt[0][:, :3] - traj[t + 1][0][:, :3]).max(1)
        ev = np.maximum(np.abs(nxt[2][:, :3] - traj[t + 1][2][:, :3]).max(1),
                        np.abs(nxt[3][:, :3] - traj[t + 1][3][:, :3]).max(1))
        np.maximum.at(dev_pos, wid, ep)
        np.maximum.at(dev_vel, wid, ev)
    return world_functional(scene, (dpos, dquat, dlin, dang), seeds), dev_pos, dev_vel


# a world is stable when the FP64 step from every recorded state reproduces
# the next recorded state within ten times the one-step bars
STABLE_POS_M = 1e-4
STABLE_VEL_MPS = 1e-3
# and when the FP64 step's discrete choices at every recorded state stay the
# same under perturbations of the state at the size of the device's own
# one-step deviation from FP64 (positions 1e-6 m, velocities 1e-5 m/s,
# quaternions 1e-7): a choice that flips there is one the FP32 device may
# make the other way, and the derivative then follows another piece
PERTURB = (1e-6, 1e-7, 1e-5, 1e-5)


def active_signature(o, scene, traj, rng=None):
    """Per-world signatures (contact topology, active set) of the FP64
    steps from the recorded states (each optionally perturbed by PERTURB in
    uniform noise), accumulated over the trajectory. `o` is an FP64
    OracleWorld of the scene."""
    o.reset_active()
    dyn = (np.asarray(scene.mass) > 0)[:, None]
    for t in range(len(traj) - 1):
        st = [np.array(a, np.float64) for a in traj[t]]
        if rng is not None:
            for k in range(4):
                cols = 4 if k == 1 else 3
                st[k][:, :cols] += rng.uniform(-PERTURB[k], PERTURB[k], (scene.n, cols)) * dyn
        o.set_state_f64(*st)
        o.step(1)
    return o.active_hash()


def robust_worlds(o, scene, traj, perturbations=2, rng_seed=1):
    """Worlds whose FP64 discrete choices along the recorded trajectory are
    the same for the recorded states and for `perturbations` perturbed
    copies of them."""
    base = active_signature(o, scene, traj)
    rng = np.random.default_rng(rng_seed)
    ok = np.ones(scene.num_worlds, bool)
    for _ in range(perturbations):
        ok &= (active_signature(o, scene, traj, rng) == base).all(1)
    return ok


def gradient_errors(o, inv_inertia3, scene, traj, grads, seeds, directions=2, rng_seed=0, o_value=None):
    """Per parameter set ("lin", "ang", "mass", "friction") and world, the
    relative error (vector norm over `directions` random directions) of the
    device gradients' directional derivatives against the chained FP64
    tangent, and the per-world stability flags: the value criterion
    (STABLE_POS_M, STABLE_VEL_MPS) and, with an FP64 OracleWorld o_value,
    the robustness of the discrete choices (robust_worlds)."""
    rng = np.random.default_rng(rng_seed)
    dyn = np.asarray(scene.mass) > 0
    wid = np.asarray(scene.world)
    rel, stable = {}, np.ones(scene.num_worlds, bool)
    if o_value is not None:
        stable &= robust_worlds(o_value, scene, traj)
    for kind in ("lin", "ang", "mass", "friction"):
        comps = 3 if kind in ("lin", "ang") else 1
        ga = np.asarray(grads[kind], np.float64).reshape(scene.n, -1)
        ad, ref = [], []
        for _ in range(directions):
            d = rng.normal(size=(scene.n, comps)) * dyn[:, None]
            dd = d if comps == 3 else d[:, 0]
            t, dp, dv = chained_tangent(o, inv_inertia3, scene, traj, seeds, kind, dd)
            stable &= (dp <= STABLE_POS_M) & (dv <= STABLE_VEL_MPS)
            ad.append([np.sum(ga[wid == k] * d[wid == k]) for k in range(scene.num_worlds)])
            ref.append(t)
        ad, ref = np.array(ad), np.array(ref)
        rel[kind] = np.linalg.norm(ad - ref, axis=0) / np.maximum(np.linalg.norm(ref, axis=0), 1e-30)
    return rel, stable
