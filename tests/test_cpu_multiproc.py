"""Multi-process path of the batched form on CPU: two `gloo` ranks each take
a body-balanced range of worlds (experiments_b200.sharding), step their
shard with the oracle, and reduce the per-world results with the only
collective the path has (a final gather of scalars). The gathered result
must equal one process stepping every world: worlds are independent, so
sharding changes nothing."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from experiments_b200 import sharding, scenes

STEPS = 6


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _world_com(scene, pos):
    m = np.asarray(scene.mass, np.float64)
    out = np.zeros((scene.num_worlds, 3))
    for w in range(scene.num_worlds):
        k = (np.asarray(scene.world) == w) & (m > 0)
        out[w] = (pos[k, :3] * m[k, None]).sum(0) / m[k].sum()
    return out


def _run_oracle(scene):
    import oracle
    from experiments_b200 import b3
    hc = b3.Context(-1)
    w = b3.PhysicsWorld(hc, scenes.world_config(scene))
    scenes.register_scene(w, scene)
    o = oracle.oracle_from_world(w, scene)
    o.step(STEPS)
    pos = o.state()[0]
    o.close()
    w.close()
    hc.close()
    return _world_com(scene, pos)


def _rank(rank, world_size, port, out_path):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size)
    full = scenes.c3(worlds=12, nmax=48)
    shard, (lo, hi) = sharding.shard_scene(full, rank, world_size)
    com = torch.from_numpy(_run_oracle(shard))
    # the one collective: gather per-world scalars to every rank
    sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world_size)]
    dist.all_gather(sizes, torch.tensor([com.shape[0]], dtype=torch.int64))
    maxn = int(max(s.item() for s in sizes))
    pad = torch.zeros(maxn, 3, dtype=torch.float64)
    pad[:com.shape[0]] = com
    bufs = [torch.zeros(maxn, 3, dtype=torch.float64) for _ in range(world_size)]
    dist.all_gather(bufs, pad)
    if rank == 0:
        allc = torch.cat([b[:int(s.item())] for b, s in zip(bufs, sizes)]).numpy()
        np.save(out_path, allc)
    dist.barrier()
    dist.destroy_process_group()


def test_partition_is_body_balanced_and_contiguous():
    sc = scenes.c3(worlds=64)
    off = sharding.world_offsets(sc)
    for ws in (1, 2, 3, 8):
        parts = sharding.partition_worlds(off, ws)
        assert parts[0][0] == 0 and parts[-1][1] == 64
        assert all(parts[i][1] == parts[i + 1][0] for i in range(ws - 1))
        loads = [off[h] - off[l] for l, h in parts]
        assert sum(loads) == sc.n
        assert max(loads) - min(loads) <= 2 * 512  # within two of the largest worlds


def test_two_gloo_ranks_match_one_process(tmp_path):
    out = str(tmp_path / "com.npy")
    mp.spawn(_rank, args=(2, _free_port(), out), nprocs=2, join=True)
    sharded = np.load(out)
    full = _run_oracle(scenes.c3(worlds=12, nmax=48))
    assert sharded.shape == full.shape
    assert np.array_equal(sharded, full)
