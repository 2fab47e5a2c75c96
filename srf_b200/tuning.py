"""Kernel tuning for the TOR ops and a small autotuner.

``set_tuning(path, slab_slices, grid_mult)`` sets the library's process-wide knobs
(``srf_tor_set_tuning``): the kernel family (0 automatic, 1 shared-memory slabs with a
lane per (LOR, slab) segment, 2 LOR-centric, 3 shared-memory slabs with a segment's
slices spread over lanes), the number of slices per shared-memory slab (0 = as many as fit) and
the grid multiplier of the persistent slab kernel (0 = automatic). ``set_tuning()``
restores the library's defaults (all automatic).

``Autotuner`` times a caller-supplied step (for example one OSEM sub-iteration on a
representative subset) under each candidate setting with CUDA events and keeps the
fastest per key (geometry, patch size, problem size bucket); results can be saved to and
loaded from a JSON file so a reconstruction tunes once per configuration.
"""

import json
import math
import os

import torch

from . import _lib

DEFAULT = (0, 0, 0)


def set_tuning(path=0, slab_slices=0, grid_mult=0):
    _lib.call("srf_tor_set_tuning", int(path), int(slab_slices), int(grid_mult))
    return (path, slab_slices, grid_mult)


def set_siddon_tuning(path=0):
    """Siddon kernel family (``srf_siddon_set_tuning``): 0 automatic (the scatter ops
    reduce four consecutive voxels at a time where the image allows), 1 one per voxel."""
    _lib.call("srf_siddon_set_tuning", int(path))
    return path


def set_scratch_limit(nbytes=0):
    """Bound the per-call scratch of the slab kernels (``srf_tor_set_scratch_limit``);
    larger calls run in chunks of LORs. 0 restores the default (4 GiB)."""
    _lib.call("srf_tor_set_scratch_limit", int(nbytes))


def candidates(max_slab_slices):
    """Settings worth trying: full and half-depth slabs, each with the library's automatic
    grid multiplier (0: chosen per op and call size) and with multipliers 1 and 2 fixed,
    the spread-items slab kernel and the LOR-centric kernels. The automatic choice comes
    first, so a tie keeps it."""
    out = [(1, 0, 0), (1, 0, 1), (1, 0, 2)]
    half = max(1, max_slab_slices // 2)
    if half < max_slab_slices:
        out += [(1, half, 0), (1, half, 1), (1, half, 2)]
    out += [(3, 0, 1), (2, 0, 1)]
    return out


def key_for(grid, patch, n_lors, n_frames=1):
    bucket = int(math.log2(max(1, n_lors)))
    return f"g{grid[0]}x{grid[1]}x{grid[2]}_p{patch}_n2^{bucket}_f{n_frames}"


def cuda_event_time(step, warmup, reps):
    """Mean milliseconds of ``step()`` over ``reps`` runs after ``warmup`` untimed runs,
    with CUDA events on the current stream."""
    for _ in range(warmup):
        step()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    s.record()
    for _ in range(reps):
        step()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps


class Autotuner:
    """``timer(step, warmup, reps) -> ms`` measures one candidate (default: CUDA events)."""

    def __init__(self, cache_path=None, timer=None):
        self.cache_path = cache_path
        self.timer = timer or cuda_event_time
        self.table = {}
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                self.table = {k: tuple(v) for k, v in json.load(f).items()}

    def tune(self, key, step, cands, warmup=1, reps=3):
        """Time ``step()`` under each setting of ``cands``; apply and return the best."""
        if key in self.table:
            set_tuning(*self.table[key])
            return self.table[key], None
        timings = {}
        for c in cands:
            set_tuning(*c)
            timings[c] = self.timer(step, warmup, reps)
        best = min(timings, key=timings.get)
        self.table[key] = best
        set_tuning(*best)
        if self.cache_path:
            with open(self.cache_path, "w") as f:
                json.dump({k: list(v) for k, v in self.table.items()}, f, indent=1)
        return best, timings
