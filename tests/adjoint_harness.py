"""Test harness for the adjoint form: FP64 central differences on the oracle,
the product's reverse sweep, and a torch.autograd.Function over it (the
library itself does not depend on torch)."""
import copy

import numpy as np

import oracle
from experiments_b200 import b3, scenes
from oracle import tangent_chain
from oracle.tangent_chain import com_seeds, param_tangents, world_functional  # noqa: F401


def make_oracle(host_ctx, scene, dual=False):
    """Oracle world of a scene plus the per-body inverse inertia diagonal of
    the registration (FP64 copy); dual=True: the tangent-linear build."""
    w = b3.PhysicsWorld(host_ctx, scenes.world_config(scene))
    scenes.register_scene(w, scene)
    o = oracle.oracle_from_world(w, scene, dual=dual)
    ii = w.inertias()[:, :3].astype(np.float64)
    w.close()
    return o, ii


def oracle_state_at(host_ctx, scene, steps):
    """Oracle state after `steps` steps, rounded to FP32 (the state both sides
    start from)."""
    o, _ = make_oracle(host_ctx, scene)
    o.step(steps)
    st = [a.astype(np.float32).astype(np.float64) for a in o.state()]
    o.close()
    return st


def oracle_run(host_ctx, scene, state, steps, seeds, kind=None, delta=None, eps=0.0):
    """Run the oracle `steps` steps from `state` with one parameter set
    perturbed by eps * delta in FP64; returns the per-world functional and
    the per-world active-set signatures."""
    o, ii = make_oracle(host_ctx, scene)
    pos, quat, lin, ang = [a.copy() for a in state]
    m = np.asarray(scene.mass, np.float64)
    im = np.where(m > 0, 1.0 / np.where(m > 0, m, 1), 0.0)
    if kind == "lin":
        lin[:, :3] += eps * delta
    elif kind == "ang":
        ang[:, :3] += eps * delta
    elif kind == "mass":
        m2 = m + eps * delta
        im2 = np.where(m > 0, 1.0 / np.where(m > 0, m2, 1), 0.0)
        scale = np.where(im > 0, im2 / np.where(im > 0, im, 1), 0.0)
        o.set_params_f64(inv_mass=im2, inv_inertia3=ii * scale[:, None])
    elif kind == "friction":
        o.set_params_f64(friction=np.asarray(scene.friction, np.float64) + eps * delta)
    o.set_state_f64(pos, quat, lin, ang)
    o.reset_active()
    o.step(steps)
    st = o.state()
    h = o.active_hash()
    o.close()
    return world_functional(scene, st, seeds), h


def oracle_tangent(host_ctx, scene, state, steps, seeds, kind, delta):
    """Directional derivative of the per-world functional along delta (one
    parameter set: "lin" / "ang" n x 3, "mass" / "friction" n), from the
    FP64 tangent-linear oracle: exact derivatives of the FP64 step with its
    discrete choices held at the value path's. Returns the per-world
    derivatives and the per-world active-set signatures."""
    o, ii = make_oracle(host_ctx, scene, dual=True)
    o.set_state_f64(*[a.copy() for a in state])
    delta = np.asarray(delta, np.float64)
    if kind == "lin":
        o.set_tangent(lin=delta)
    elif kind == "ang":
        o.set_tangent(ang=delta)
    else:
        o.set_tangent(**param_tangents(scene, ii, kind, delta))
    o.reset_active()
    o.step(steps)
    d = o.tangent()
    h = o.active_hash()
    o.close()
    return world_functional(scene, d, seeds), h


def chained_tangent(host_ctx, scene, traj, seeds, kind, delta):
    """The FP64 tangent chained along a recorded trajectory
    (oracle.tangent_chain.chained_tangent) with a fresh tangent-linear
    oracle of the scene."""
    o, ii = make_oracle(host_ctx, scene, dual=True)
    out = tangent_chain.chained_tangent(o, ii, scene, traj, seeds, kind, delta)
    o.close()
    return out


def tangent_vectors(host_ctx, scene, state, steps, seeds, kind, per):
    """Whole FP64 gradient vectors of the per-world functional with respect
    to one parameter set, one tangent-linear run per body slot and
    component (worlds are independent, so a run seeds the same slot in
    every world). Returns (n x comps gradient, per-world signatures)."""
    dyn = np.asarray(scene.mass) > 0
    wid = np.asarray(scene.world)
    comps = 3 if kind in ("lin", "ang") else 1
    g = np.zeros((scene.n, comps))
    slots = np.where(dyn)[0].reshape(scene.num_worlds, per)
    h0 = None
    for j in range(per):
        bodies = slots[:, j]
        for c in range(comps):
            d = np.zeros((scene.n, comps))
            d[bodies, c] = 1.0
            t, h = oracle_tangent(host_ctx, scene, state, steps, seeds, kind, d if comps == 3 else d[:, 0])
            g[bodies, c] = t[wid[bodies]]
            h0 = h if h0 is None else h0
    return g, h0


def device_trajectory(ctx, scene, state, steps):
    """The device's states s_0 .. s_steps (FP32 values as FP64), one step
    at a time from `state`."""
    w = scenes.build_world(ctx, scene, useGraph=1)
    w.write_state(*[np.asarray(a, np.float32) for a in state])
    traj = [[a.astype(np.float64) for a in w.read_state()]]
    for _ in range(steps):
        w.stepSimulation(1)
        traj.append([a.astype(np.float64) for a in w.read_state()])
    w.close()
    return traj


def gpu_adjoint(ctx, scene, state, steps, seeds, checkpoint_every=16):
    """The product's gradients of the per-world functional."""
    w = scenes.build_world(ctx, scene, useGraph=1)
    w.write_state(*[np.asarray(a, np.float32) for a in state])
    adj = b3.Adjoint(w, steps, checkpoint_every)
    adj.forward()
    final = [a.astype(np.float64) for a in w.read_state()]
    adj.backward(*[np.asarray(s, np.float32) for s in seeds])
    g = adj.gradients()
    g["unclassified"] = adj.unclassified()
    g["final"] = final
    adj.close()
    w.close()
    return g


def random_seeds(scene, rng):
    dyn = (np.asarray(scene.mass) > 0).astype(np.float64)
    seeds = [rng.normal(size=(scene.n, 4)) * dyn[:, None] for _ in range(4)]
    for k in (0, 2, 3):
        seeds[k][:, 3] = 0.0
    return seeds


class Rollout:
    """torch.autograd.Function over a batched world: (initial linear and
    angular velocities, masses, friction) -> final positions."""

    @staticmethod
    def make(ctx, scene, steps, checkpoint_every=16):
        import torch

        class _F(torch.autograd.Function):
            @staticmethod
            def forward(fctx, lin0, ang0, mass, friction):
                sc = copy.copy(scene)
                sc.lin = lin0.detach().cpu().numpy().astype(np.float64)
                sc.ang = ang0.detach().cpu().numpy().astype(np.float64)
                sc.mass = mass.detach().cpu().numpy().astype(np.float64)
                sc.friction = friction.detach().cpu().numpy().astype(np.float64)
                w = scenes.build_world(ctx, sc, useGraph=1)
                w.write_velocities(sc.lin, sc.ang)
                adj = b3.Adjoint(w, steps, checkpoint_every)
                adj.forward()
                pos = torch.from_numpy(w.read_state()[0][:, :3].astype(np.float64))
                fctx.adj, fctx.world = adj, w
                return pos

            @staticmethod
            def backward(fctx, gpos):
                adj = fctx.adj
                adj.backward(d_pos=gpos.detach().cpu().numpy())
                g = adj.gradients()
                adj.close()
                fctx.world.close()
                return (torch.from_numpy(g["lin"].astype(np.float64)), torch.from_numpy(g["ang"].astype(np.float64)),
                        torch.from_numpy(g["mass"].astype(np.float64)),
                        torch.from_numpy(g["friction"].astype(np.float64)))

        return _F
