"""MLEM / OSEM reconstruction and the efficiency-map pass on the GPU.

Reference path (relative to the SRF project root):

* ``ReconStep.kernel`` (src/python/srf/model/recon_step.py:33-41): projection, the
  reference back-projection A^T(1/Ax), then ``mlem_update`` x <- x * effinv * bp
  (:48-49). The list-mode measurement y = 1 is implicit in the division.
* ``LocalReconstructionGraph.run`` (src/python/srf/graph/reconstruction/
  local_reconstruction.py:44-51): one update per iteration over the whole list, the
  image saved as ``{prefix}_{i}.npy`` after every iteration.
* The efficiency map: ``Maplors`` over detector-pair LORs, summed over the three axis
  groups (physics/split_lors.py:116-133), cropped, normalised and inverted
  (preprocess/merge_map.py:8-88).

Ordered subsets (the reference carries them only in unused graph classes,
graph/reconstruction/master.py:122-162): subset k holds events k, k+S, k+2S, ... of
every axis group, and its update uses S * effinv, i.e. the sensitivity split evenly
over subsets. With S = 1 this is exactly the reference's full-list MLEM.

One iteration (all subsets) can be captured in a CUDA graph: the library never
synchronises the host, so the whole sequence of projector launches, image
permutations and updates replays with one launch.
"""

import os

import numpy as np
import torch

from . import ops
from .data import Image, ListModeData, ListModeDataSplit
from .physics import (CompleteLoRsModel, SplitLoRsModel, map_generated, map_lors,
                      projection_backprojection)
from .preprocess import crop_mask, map_process, merge_effmap, split_listmode


def mlem_update(image_prev, image_succ, efficiency_map):
    """x * effinv * bp (recon_step.py:48-49) in place on a copy of ``image_prev``."""
    out = image_prev.data.clone()
    ops.mlem_update_(out, efficiency_map.data.contiguous(), image_succ.data.contiguous())
    return Image(out, image_prev.center, image_prev.size)


def mlem_update_normal(image_prev, image_succ, efficiency_map):
    """x / effmap * bp (recon_step.py:52-53), with the reference's operation order: the
    division first, then the product, so a voxel with zero efficiency gives inf or NaN
    exactly as the reference does (``mlem_update`` with an inverted map is the path the
    reconstruction uses; there zero-efficiency voxels carry effinv = 0)."""
    out = image_prev.data / efficiency_map.data * image_succ.data
    return Image(out, image_prev.center, image_prev.size)


class ReconStep:
    """projection -> back-projection -> update (recon_step.py:17-45)."""

    def __init__(self, model, update=mlem_update):
        self.model = model
        self.update = update

    def __call__(self, image, efficiency_map, projection_data):
        _, back = projection_backprojection(self.model, image, projection_data)
        return self.update(image, back, efficiency_map)


# ------------------------------------------------------------------------- subsets


def _take(t, k, s):
    return t[k::s].contiguous() if s > 1 else t


def make_subsets(data, n_subsets):
    """Interleaved subsets of list-mode data (split or complete)."""
    out = []
    for k in range(n_subsets):
        if isinstance(data, ListModeDataSplit):
            out.append(ListModeDataSplit(*[
                ListModeData(_take(data[a].lors, k, n_subsets),
                             _take(data[a].values, k, n_subsets)) for a in "xyz"]))
        else:
            out.append(ListModeData(_take(data.lors, k, n_subsets),
                                    _take(data.values, k, n_subsets)))
    return out


def order_subset(model, data, image):
    """One subset's records reordered for the kernels (TOR: by direction inside 4096-record
    blocks, ``preprocess.order_listmode``; Siddon: by walk length, ``preprocess.
    ray_length_order``); values follow their records."""
    if isinstance(model, SplitLoRsModel):
        from .preprocess import order_listmode
        return order_listmode(data)
    if isinstance(model, CompleteLoRsModel) and len(data) > 1:
        from .preprocess import ray_length_order
        _, g, c, s = model.kernel_geometry(image)
        perm = ray_length_order(data.lors, g, c, s)
        return type(data)(data.lors[perm].contiguous(), data.values[perm].contiguous())
    return data


# ---------------------------------------------------------------------- efficiency map


def _chunk_reader(lors, chunk):
    """(n, chunk, device, take(start, count)) of an [N, 6] tensor or a chunked source."""
    if callable(lors):
        return (len(lors), getattr(lors, "chunk", chunk),
                getattr(lors, "device", torch.device("cuda")), lors)
    return lors.shape[0], chunk, lors.device, (lambda s, c: lors[s:s + c])


def map_chunk_default(model, part, img, order=True):
    """Maplors of one chunk of [count, 6] detector-pair LORs into ``img``'s geometry
    (``map_process`` and the axis groups for the TOR model, the raw LORs for Siddon)."""
    if isinstance(model, SplitLoRsModel):
        groups = map_process(part)
        if order:
            from .preprocess import order_by_direction
            groups = order_by_direction(groups)
        data = split_listmode(groups, without_tof=True)
    else:
        from .data import ListModeDataWithoutTOF
        data = ListModeDataWithoutTOF(part, torch.ones(part.shape[0], device=part.device))
    return map_lors(model, data, img).data


def map_sum(model, lors, grid, center, size, chunk=16_000_000, order=True, chunks=None,
            map_chunk=None):
    """Sum of Maplors over the chunks of ``lors`` (before the crop / normalise / invert
    of ``merge_effmap``). ``chunks``: indices of the chunks to take (all by default; a
    rank of a sharded pass takes its own); ``map_chunk(model, part, img)`` maps one chunk
    (``map_chunk_default``)."""
    from .synthetic import GeneratedPairs
    n, chunk, dev, take = _chunk_reader(lors, chunk)
    total = torch.zeros(tuple(grid), dtype=torch.float32, device=dev)
    img = Image(total, center, size)
    fused = isinstance(lors, GeneratedPairs) and isinstance(model, SplitLoRsModel) \
        and map_chunk is None
    fn = map_chunk or (lambda m, part, im: map_chunk_default(m, part, im, order))
    n_chunks = (n + chunk - 1) // chunk
    for c in (range(n_chunks) if chunks is None else chunks):
        s = c * chunk
        if s >= n:
            continue
        if fused:  # the kernels make the LORs themselves: nothing is materialised
            total.add_(map_generated(model, lors, img, s, min(chunk, n - s)).data)
        else:
            total.add_(fn(model, take(s, min(chunk, n - s)), img))
    return total


def efficiency_map(model, lors, grid, center, size, inner_radius, axial_length,
                   chunk=16_000_000, crop_ratio=0.95, threshold=1e-6, zero_below=True,
                   order=True):
    """Inverted efficiency map from detector-pair LORs: Maplors summed over the axis
    groups (or Siddon map), cropped, normalised to max 1 and inverted
    (merge_map.py:37-41). ``lors`` is an [N, 6] CUDA tensor, or a source with ``len()``
    and ``source(start, count)`` returning [count, 6] CUDA chunks (for example
    ``synthetic.RandomLorSource``), so that N LORs never exist at once; its chunk size
    then sets ``chunk``. A ``synthetic.GeneratedPairs`` source with the TOR model is
    mapped by kernels that make each LOR from its number: no LOR array at all. With ``order`` (TOR model) each chunk's map records are
    reordered by direction inside 4096-record blocks (``preprocess.order_by_direction``)
    before Maplors: the map is the same sum taken in another order, and the slab kernels
    walk fewer voxel slots for LORs of mixed directions (random detector pairs)."""
    total = map_sum(model, lors, grid, center, size, chunk, order)
    keep = crop_mask(grid, center, size, inner_radius, axial_length, crop_ratio,
                     device=total.device)
    return Image(merge_effmap(total, keep, threshold, zero_below), center, size), total


# ---------------------------------------------------------------------- OSEM driver


class OSEM:
    """Ordered-subsets EM with optional CUDA-graph capture of each iteration.

    ``data``: ListModeDataSplit (TOR) or ListModeData (Siddon) with values of one.
    ``effinv``: inverted efficiency map (Image). ``x0``: initial image (Image).
    ``order``: reorder each subset's records once (``order_subset``) so that every
    iteration's kernels waste fewer lanes; subset membership follows the caller's event
    order, so the image is the same sums taken in another order."""

    def __init__(self, model, data, effinv, x0, n_subsets=1, use_graph=False, order=True):
        self.model = model
        self.n_subsets = int(n_subsets)
        self.subsets = make_subsets(data, self.n_subsets)
        if order:  # inside each subset: the subsets hold the caller's events k, k+S, ...
            self.subsets = [order_subset(model, d, x0) for d in self.subsets]
        self.effinv = Image((effinv.data * float(self.n_subsets)).contiguous(), effinv.center,
                            effinv.size)
        self.x = Image(x0.data.clone().contiguous(), x0.center, x0.size)
        self.use_graph = use_graph
        self._graph = None
        self.iteration = 0

    def _subset_update(self, k):
        _, back = projection_backprojection(self.model, self.x, self.subsets[k])
        ops.mlem_update_(self.x.data, self.effinv.data, back.data)

    def _iterate(self):
        for k in range(self.n_subsets):
            self._subset_update(k)

    def _capture(self):
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        backup = self.x.data.clone()
        with torch.cuda.stream(s):
            self._iterate()  # warm-up outside the graph (allocator, lazy init)
        torch.cuda.current_stream().wait_stream(s)
        self.x.data.copy_(backup)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._iterate()
        self.x.data.copy_(backup)
        self._graph = g

    def step(self):
        """One full iteration over all subsets."""
        if self.use_graph:
            if self._graph is None:
                self._capture()
            self._graph.replay()
        else:
            self._iterate()
        self.iteration += 1
        return self.x

    def run(self, n_iterations, prefix=None, callback=None):
        for _ in range(n_iterations):
            self.step()
            if prefix is not None:
                save_checkpoint(prefix, self.iteration - 1, self.x)
            if callback is not None:
                callback(self.iteration, self.x)
        return self.x


# ----------------------------------------------------------------- checkpoint/resume


def save_checkpoint(prefix, iteration, image, seed=None):
    """``{prefix}_{i}.npy`` as the reference writes (local_reconstruction.py:50-51),
    plus ``{prefix}_{i}.meta.npz`` with the iteration, center, size and seed."""
    arr = image.data.detach().cpu().numpy()
    np.save(f"{prefix}_{iteration}.npy", arr)
    np.savez(f"{prefix}_{iteration}.meta.npz", iteration=iteration,
             center=np.array(image.center), size=np.array(image.size),
             seed=np.array(-1 if seed is None else seed))


def latest_checkpoint(prefix):
    """(iteration, path) of the newest ``{prefix}_{i}.npy``, or (None, None)."""
    d = os.path.dirname(prefix) or "."
    base = os.path.basename(prefix) + "_"
    best = None
    for f in os.listdir(d):
        if f.startswith(base) and f.endswith(".npy"):
            mid = f[len(base):-4]
            if mid.isdigit() and (best is None or int(mid) > best[0]):
                best = (int(mid), os.path.join(d, f))
    return best if best else (None, None)


def resume(prefix, center, size, device):
    """Image and next iteration index from the newest checkpoint (or (None, 0))."""
    it, path = latest_checkpoint(prefix)
    if it is None:
        return None, 0
    arr = np.load(path)
    return Image(torch.as_tensor(arr, device=device), center, size), it + 1
