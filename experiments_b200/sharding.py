"""Partition of batched worlds across GPUs.

Batched worlds are independent, so they shard with no exchange step: each
rank steps a contiguous range of worlds in its own batched world, and the
only collective is the final reduction of scalar metrics (losses, counts).
Ranges are cut on the body-count prefix sums (b3_batch_world_offsets) so
every rank holds about the same number of bodies.
"""
import numpy as np


def partition_worlds(offsets, world_size):
    """Contiguous world ranges [lo, hi) per rank from body-count prefix sums
    `offsets` (numWorlds + 1 entries): rank r takes the worlds whose first
    body falls in [r T / R, (r + 1) T / R), T the total body count."""
    offsets = np.asarray(offsets, np.int64)
    nw = len(offsets) - 1
    total = int(offsets[-1])
    cuts = [0]
    for r in range(1, world_size):
        target = total * r / world_size
        k = int(np.searchsorted(offsets[:-1], target, side="left"))
        cuts.append(min(max(k, cuts[-1]), nw))
    cuts.append(nw)
    return [(cuts[r], cuts[r + 1]) for r in range(world_size)]


def world_offsets(scene):
    """Body-count prefix sums of a scene's worlds (host-side twin of
    b3_batch_world_offsets)."""
    counts = np.bincount(np.asarray(scene.world, np.int64), minlength=int(scene.num_worlds))
    return np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)


def shard_scene(scene, rank, world_size):
    """The sub-scene of worlds owned by `rank` (worlds renumbered from 0)."""
    from . import scenes
    lo, hi = partition_worlds(world_offsets(scene), world_size)[rank]
    return scenes.select_worlds(scene, range(lo, hi)), (lo, hi)
