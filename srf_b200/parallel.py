"""Event-sharded reconstruction across GPUs (one process per GPU).

The reference's only multi-worker step is the master summing the workers' image
buffers (src/python/srf/graph/reconstruction/master.py:54-59, worker.py:58-63); its live
app runs one worker. Here each rank owns a shard of the events, the image is replicated,
projection needs no exchange, and the back-projected images are summed with one
all-reduce (NCCL over NVLink on GPUs; gloo for CPU ranks in tests) before every rank
applies the same update. Shards are contiguous index ranges of each axis group, so the
concatenation of all shards is the full list.
"""

import torch
import torch.distributed as dist

from .data import Image, ListModeData, ListModeDataSplit


def shard_range(n, rank, world):
    """[start, stop) of rank's contiguous shard of n items."""
    per = (n + world - 1) // world
    start = min(n, rank * per)
    return start, min(n, start + per)


def shard(data, rank, world):
    """This rank's shard of ListModeData / ListModeDataSplit (views, no copy)."""
    if isinstance(data, ListModeDataSplit):
        return ListModeDataSplit(*[shard(data[a], rank, world) for a in ("x", "y", "z")])
    a, b = shard_range(len(data), rank, world)
    return type(data)(data.lors[a:b], data.values[a:b])


def allreduce_image(img, group=None):
    """Sum an Image's data over ranks in place (the master sum)."""
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(img.data, op=dist.ReduceOp.SUM, group=group)
    return img


class ShardedMLEM:
    """MLEM over event shards: x <- x * effinv * sum_ranks A_r^T(1 / (A_r x)).

    ``project(model, image, data)`` and ``backproject(model, data, image)`` default to
    ``srf_b200.physics``; tests inject other implementations (for example the oracle on
    CPU ranks). ``update(x, effinv, bp)`` defaults to the elementwise product."""

    def __init__(self, model, data, effinv, x0, group=None, project=None, backproject=None,
                 update=None):
        from . import physics
        self.model = model
        self.data = data
        self.effinv = effinv
        self.x = Image(x0.data.clone(), x0.center, x0.size)
        self.group = group
        self.project = project or physics.projection
        self.backproject = backproject or physics.backprojection
        self.update = update or (lambda x, e, b: x * e * b)

    def step(self):
        proj = self.project(self.model, self.x, self.data)
        bp = self.backproject(self.model, proj, self.x)
        allreduce_image(bp, self.group)
        self.x = Image(self.update(self.x.data, self.effinv.data, bp.data), self.x.center,
                       self.x.size)
        return self.x
