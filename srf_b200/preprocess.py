"""LOR preprocessing on the GPU: ``recon_process`` / ``map_process`` of
``src/python/srf/preprocess/function/on_tor_lors.py:243-262`` and the effmap merge of
``src/python/srf/preprocess/merge_map.py``.

``recon_process(events, tof_res)`` and ``map_process(lors)`` return a dict
``{'x': ..., 'y': ..., 'z': ...}`` of row-major CUDA tensors ([N_a, 10] / [N_a, 7]),
views into one buffer, exactly the reference's dict of numpy arrays but resident on
the device. The group sizes are read back to the host (one small copy).
"""

import numpy as np
import torch

from . import _lib
from .data import ListModeData, ListModeDataSplit, ListModeDataSplitWithoutTOF, as_cuda_f32

AXES = ("x", "y", "z")


def _stream(dev):
    return torch.cuda.current_stream(dev).cuda_stream


def _run(fn, events, ncols_in, ncols_out, *extra):
    ev = as_cuda_f32(events)
    if ev.dim() != 2 or ev.shape[1] < ncols_in:
        raise ValueError(f"expected [N, >={ncols_in}] events, got {tuple(ev.shape)}")
    if ev.stride(1) != 1:
        ev = ev.contiguous()
    n = ev.shape[0]
    dev = ev.device
    lib = _lib.load()
    ws_bytes = int(lib.srf_preprocess_workspace_size(n))
    ws = torch.empty(max(ws_bytes, 256), dtype=torch.uint8, device=dev)
    out = torch.empty((n, ncols_out), dtype=torch.float32, device=dev)
    counts = torch.zeros(3, dtype=torch.int64, device=dev)
    with torch.cuda.device(dev):
        _lib.call(fn, ev.data_ptr(), n, ev.stride(0), *extra, out.data_ptr(), counts.data_ptr(),
                  ws.data_ptr(), ws.numel(), _stream(dev))
    c = counts.cpu().tolist()
    groups, start = {}, 0
    for a, k in zip(AXES, c):
        groups[a] = out[start:start + k]
        start += k
    return groups


def recon_process(events, tof_res):
    """[N, 7] (x1,y1,z1,x2,y2,z2,tof) -> {'x','y','z'}: [N_a, 10]."""
    return _run("srf_recon_process", events, 7, 10, float(tof_res))


def map_process(lors):
    """[N, 6] (x1..z2) -> {'x','y','z'}: [N_a, 7]."""
    return _run("srf_map_process", lors, 6, 7)


def split_listmode(groups, values=None, without_tof=False):
    """Wrap recon/map_process output as the reference's loader does
    (``SplitWorkerLoader.load``, src/python/srf/data/loader.py:96-119): values of one."""
    parts = []
    for a in AXES:
        g = groups[a]
        v = values[a] if values is not None else torch.ones(g.shape[0], dtype=torch.float32,
                                                           device=g.device)
        parts.append(ListModeData(g, v))
    cls = ListModeDataSplitWithoutTOF if without_tof else ListModeDataSplit
    return cls(*parts)


# ------------------------------------------------------------------- effmap merge


def crop_mask(grid, center, size, inner_radius, axial_length, crop_ratio=0.95, device=None):
    """Keep-mask of ``crop_image`` (merge_map.py:47-65) over the [nx,ny,nz] image. The
    reference pairs the mesh list of ``RingBlock.get_meshes`` (np.meshgrid 'xy' order:
    iy, ix, iz) with the image flattened as (ix, iy, iz); the mask keeps that pairing.
    With ``device`` the mask is built there as a torch bool tensor (the same float64
    operations, so the same mask) instead of as a numpy array on the host."""
    grid = np.asarray(grid)
    center = np.asarray(center, dtype=np.float64)
    size = np.asarray(size, dtype=np.float64)
    interval = size / grid
    p0 = center - (size - interval) / 2
    p1 = center + (size - interval) / 2
    r = [np.linspace(p0[i], p1[i], grid[i]) for i in range(3)]
    if device is not None:
        return _crop_mask_torch(grid, r, inner_radius, axial_length, crop_ratio, device)
    m = np.array(np.meshgrid(r[0], r[1], r[2])).reshape((3, -1)).T
    keep = np.ones(m.shape[0], bool)
    keep[np.sqrt(m[:, 0] ** 2 + m[:, 1] ** 2) > crop_ratio * inner_radius] = False
    keep[np.abs(m[:, 2]) >= axial_length / 2] = False
    return keep.reshape(tuple(grid))


def _crop_mask_torch(grid, r, inner_radius, axial_length, crop_ratio, device):
    nx, ny, nz = (int(g) for g in grid)
    f = torch.arange(nx * ny * nz, dtype=torch.int64, device=device)
    # flat index f of the image walks the mesh list in meshgrid 'xy' order (iy, ix, iz)
    j, i, k = f // (nx * nz), (f // nz) % nx, f % nz
    x = torch.as_tensor(r[0], dtype=torch.float64, device=device)[i]
    y = torch.as_tensor(r[1], dtype=torch.float64, device=device)[j]
    z = torch.as_tensor(r[2], dtype=torch.float64, device=device)[k]
    keep = torch.sqrt(x * x + y * y) <= crop_ratio * inner_radius
    keep &= torch.abs(z) < axial_length / 2
    return keep.reshape(nx, ny, nz)


def merge_effmap(total, keep, threshold=1e-6, zero_below=True):
    """Crop, normalise to max 1 and invert a summed map (merge_map.py:37-41; with
    ``threshold=1e-7, zero_below=False`` the ``merge_effmap_full`` variant :85-87).
    ``total`` and ``keep`` are tensors on the same device; returns float32."""
    m = torch.where(keep, total, torch.zeros_like(total)).to(torch.float64)
    m = m / m.max()
    hi = m > threshold
    out = torch.where(hi, 1.0 / torch.where(hi, m, torch.ones_like(m)),
                      torch.zeros_like(m) if zero_below else m)
    return out.to(torch.float32)


def initial_image(grid, center, size, inner_radius, axial_length, device, crop_ratio=0.95):
    """``MasterLoader.create_image`` (src/python/srf/data/loader.py:28-37): ones,
    cropped like the effmap."""
    keep = crop_mask(grid, center, size, inner_radius, axial_length, crop_ratio, device=device)
    return keep.to(torch.float32)


def order_by_direction(groups):
    """Reorder each axis group's [N, C] records (C >= 6, x1..z2 first) by the shape of their
    tube's section, inside blocks of 4096 consecutive records (``srf_order_by_direction``).

    A LOR's section box spans sqrt((1 - uy^2) / q) by sqrt((1 - ux^2) / q) (q = 1 - ux^2 -
    uy^2, (ux, uy) its in-slice direction in the kernel frame), so records of similar
    direction walk boxes of the same size. The slab kernels give a warp 32 consecutive
    LORs of a slab and walk the largest box among them; grouping similar directions makes
    that box smaller, while sorting only inside blocks keeps every stretch of the per-slab
    lists a mix of directions (equal shares of the persistent grid stay equal work).
    List-mode events form an unordered set, and projection values follow their records,
    so a reconstruction over the reordered groups is the same sum taken in another order.
    Returns new groups (same device)."""
    out = {}
    for a, g in groups.items():
        if g.shape[0] < 2:
            out[a] = g
            continue
        src = g.to(torch.float32).contiguous()
        dst = torch.empty_like(src)
        dev = src.device
        with torch.cuda.device(dev):
            _lib.call("srf_order_by_direction", src.data_ptr(), src.shape[0], src.shape[1],
                      src.stride(0), dst.data_ptr(), _stream(dev))
        out[a] = dst
    return out


def order_listmode(data):
    """``order_by_direction`` for a ListModeDataSplit: each group's records reordered with
    their values (the values travel as an extra column)."""
    out = []
    for a in ("x", "y", "z"):
        d = data[a]
        rec = torch.cat([d.lors.to(torch.float32), d.values.to(torch.float32).reshape(-1, 1)], 1)
        o = order_by_direction({a: rec})[a]
        out.append(type(d)(o[:, :-1].contiguous(), o[:, -1].contiguous()))
    return type(data)(*out)


def ray_length_order(events, grid, center, size, block=4096):
    """Permutation that sorts [N, >=6] ray records by the number of voxels their Siddon walk
    visits (``srf_siddon_count_samples``), inside blocks of ``block`` consecutive records,
    so that the rays a warp walks together finish together. The geometry is the Siddon
    op's kernel order (grid, center, size, x fastest)."""
    from .ops import siddon_count_samples
    ev = events.to(torch.float32).contiguous()
    n = ev.shape[0]
    if n < 2:
        return torch.arange(n, device=ev.device)
    visits = siddon_count_samples(ev, grid, center, size, layout="nc").to(torch.int64)
    blk = torch.arange(n, device=ev.device, dtype=torch.int64) // int(block)
    return torch.argsort(blk * (1 << 24) + visits, stable=True)


def order_rays_by_length(events, grid, center, size, block=4096):
    """Siddon counterpart of ``order_by_direction``: the records reordered by
    ``ray_length_order`` (a reconstruction over them is the same sum in another order)."""
    perm = ray_length_order(events, grid, center, size, block)
    return events.to(torch.float32)[perm].contiguous()
