"""Shared helpers for the parity tests (scene -> product world + oracle)."""
import numpy as np

import oracle
from experiments_b200 import b3, scenes


def make_pair(ctx, scene, **over):
    """Product world on ctx and an oracle world for the same scene."""
    w = scenes.build_world(ctx, scene, **over) if ctx is not None else None
    return w, oracle.oracle_from_world(w, scene)


def host_oracle(host_ctx, scene, **over):
    w = b3.PhysicsWorld(host_ctx, scenes.world_config(scene, **over))
    scenes.register_scene(w, scene)
    return w, oracle.oracle_from_world(w, scene)


def pair_set(p):
    p = np.asarray(p).reshape(-1, 2)
    return set(map(tuple, p.tolist()))


def state4(scene):
    n = scene.n
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = scene.pos
    lin = np.zeros((n, 4), np.float32)
    lin[:, :3] = scene.lin
    ang = np.zeros((n, 4), np.float32)
    ang[:, :3] = scene.ang
    return pos, scene.quat.astype(np.float32), lin, ang
