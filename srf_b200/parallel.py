"""Sharded reconstruction across GPUs (one process per GPU).

The reference's only multi-worker step is the master summing the workers' image
buffers (src/python/srf/graph/reconstruction/master.py:54-59, worker.py:58-63); its live
app runs one worker. Here each rank owns a shard of the events, the image is replicated,
projection needs no exchange, and the back-projected images are summed with one
all-reduce (NCCL over NVLink on GPUs; gloo for CPU ranks in tests) before every rank
applies the same update. Shards are contiguous index ranges of each axis group, so the
concatenation of all shards is the full list.

* ``ShardedMLEM``: full-list MLEM, one all-reduce per iteration.
* ``ShardedOSEM``: ordered subsets, one all-reduce per subset (the master sum of the
  reference, taken per subset); rank r's part of subset k is the events i = k (mod S) of
  its shard, so the union over ranks is exactly ``recon.make_subsets``' subset k and the
  sharded reconstruction equals the single-process one (up to summation order).
* ``sharded_efficiency_map``: every rank maps its own chunks of the detector-pair
  source (chunk c on rank c mod W), one all-reduce of the map sum, then the same merge.
* ``shard_frames`` / ``ShardedBatchedOSEM``: batched frames split across ranks with no
  communication at all (rank r reconstructs frames r, r + W, ...).
"""

import torch
import torch.distributed as dist

from .data import Image, ListModeData, ListModeDataSplit


def rank_world(group=None):
    """(rank, world size) of this process in ``group`` ((0, 1) without a process group)."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


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


def subset_shard(data, k, n_subsets, rank, world):
    """Rank's part of subset k: the events i = k (mod n_subsets) of each axis group that
    lie in the rank's contiguous shard (views, no copy)."""
    if isinstance(data, ListModeDataSplit):
        return ListModeDataSplit(*[subset_shard(data[a], k, n_subsets, rank, world)
                                   for a in ("x", "y", "z")])
    a, b = shard_range(len(data), rank, world)
    first = a + ((k - a) % n_subsets)
    return type(data)(data.lors[first:b:n_subsets], data.values[first:b:n_subsets])


class ShardedOSEM:
    """OSEM over event shards: per subset, this rank's projection + back-projection, the
    all-reduce of the back-projected image, then the same multiplicative update on every
    rank (``recon.OSEM``'s arithmetic: S * effinv per subset).

    ``data``: the full list-mode data (every rank takes its own shard of each axis group;
    the shards are views). ``project_back(model, image, data) -> (proj, back)`` defaults
    to ``physics.projection_backprojection`` and ``update(x, effinv, bp)`` (in place) to
    the library's ``srf_mlem_update``; tests inject CPU implementations. With
    ``use_graph`` one iteration, collectives included, is captured in a CUDA graph (NCCL
    all-reduces are capturable; every rank captures the same sequence)."""

    def __init__(self, model, data, effinv, x0, n_subsets=1, group=None, order=True,
                 use_graph=False, project_back=None, update=None):
        from . import ops, physics
        self.model = model
        self.group = group
        self.rank, self.world = rank_world(group)
        self.n_subsets = int(n_subsets)
        self.subsets = [subset_shard(data, k, self.n_subsets, self.rank, self.world)
                        for k in range(self.n_subsets)]
        if order and project_back is None:
            from .recon import order_subset
            self.subsets = [order_subset(model, d, x0) for d in self.subsets]
        self.effinv = Image((effinv.data * float(self.n_subsets)).contiguous(), effinv.center,
                            effinv.size)
        self.x = Image(x0.data.clone().contiguous(), x0.center, x0.size)
        self.project_back = project_back or physics.projection_backprojection
        self.update = update or ops.mlem_update_
        self.use_graph = use_graph
        self._graph = None
        self.iteration = 0

    def _subset_update(self, k):
        _, back = self.project_back(self.model, self.x, self.subsets[k])
        allreduce_image(back, self.group)
        self.update(self.x.data, self.effinv.data, back.data.contiguous())

    def _iterate(self):
        for k in range(self.n_subsets):
            self._subset_update(k)

    def _capture(self):
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        backup = self.x.data.clone()
        with torch.cuda.stream(s):
            self._iterate()
        torch.cuda.current_stream().wait_stream(s)
        self.x.data.copy_(backup)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._iterate()
        self.x.data.copy_(backup)
        self._graph = g

    def step(self):
        if self.use_graph:
            if self._graph is None:
                self._capture()
            self._graph.replay()
        else:
            self._iterate()
        self.iteration += 1
        return self.x

    def release(self):
        """Drop the captured graph (before ``destroy_process_group``)."""
        self._graph = None


def sharded_map_sum(model, lors, grid, center, size, group=None, chunk=16_000_000,
                    order=True, map_chunk=None):
    """The map sum over every chunk of ``lors``, each rank mapping chunks c = rank (mod
    W) and one all-reduce adding the ranks' parts (``recon.map_sum``)."""
    from .recon import _chunk_reader, map_sum
    rank, world = rank_world(group)
    n, chunk, _, _ = _chunk_reader(lors, chunk)
    mine = range(rank, (n + chunk - 1) // chunk, world)
    total = map_sum(model, lors, grid, center, size, chunk, order, chunks=mine,
                    map_chunk=map_chunk)
    if world > 1:
        dist.all_reduce(total, op=dist.ReduceOp.SUM, group=group)
    return total


def sharded_efficiency_map(model, lors, grid, center, size, inner_radius, axial_length,
                           group=None, chunk=16_000_000, crop_ratio=0.95, threshold=1e-6,
                           zero_below=True, order=True, map_chunk=None):
    """``recon.efficiency_map`` with the chunks of the detector-pair source shared among
    the ranks; every rank returns the same (inverted map, map sum)."""
    from .preprocess import crop_mask, merge_effmap
    total = sharded_map_sum(model, lors, grid, center, size, group, chunk, order, map_chunk)
    keep = crop_mask(grid, center, size, inner_radius, axial_length, crop_ratio,
                     device=total.device)
    return Image(merge_effmap(total, keep, threshold, zero_below), center, size), total


def shard_frames(n_frames, rank, world):
    """Frame indices of rank's share of a batch: r, r + W, r + 2W, ... (frames vary in
    size, so interleaving balances the ranks better than contiguous blocks)."""
    return list(range(rank, n_frames, world))


class ShardedBatchedOSEM:
    """``batched.BatchedOSEM`` of this rank's frames (``shard_frames``); frames are
    independent reconstructions, so nothing is exchanged. ``frames``: every frame's
    recon_process output (only this rank's are touched); ``x0``: one [nx,ny,nz] image or
    an [F, nx, ny, nz] stack of all frames' initial images."""

    def __init__(self, model, frames, effinv, x0, n_subsets=1, group=None, use_graph=False,
                 order=True):
        from .batched import BatchedOSEM
        self.rank, self.world = rank_world(group)
        self.frame_ids = shard_frames(len(frames), self.rank, self.world)
        if x0.dim() == 4:
            x0 = x0[self.frame_ids]
        self.inner = BatchedOSEM(model, [frames[f] for f in self.frame_ids], effinv, x0,
                                 n_subsets=n_subsets, use_graph=use_graph, order=order) \
            if self.frame_ids else None

    def step(self):
        return self.inner.step() if self.inner else None

    def images(self):
        """{frame index: image} of this rank's frames."""
        if self.inner is None:
            return {}
        return {f: self.inner.x[i] for i, f in enumerate(self.frame_ids)}
