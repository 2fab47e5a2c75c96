"""Tensor-level projector ops with the reference TF ops' argument lists.

Each function mirrors one TF op of the reference and calls the matching C entry point:

==========================  ======================================================
``tor_projection``          TOR ``Projection``      (src/cpp/tf_custom_ops/tor.cc:14-28)
``tor_backprojection``      TOR ``Backprojection``  (tor.cc:30-47)
``tor_maplors``             TOR ``Maplors``         (tor.cc:49-64)
``siddon_projection``       Siddon ``Projection``   (siddon.cc:14-26)
``siddon_backprojection``   Siddon ``Backprojection`` (siddon.cc:28-43)
``siddon_maplors``          Siddon ``Maplors``      (siddon.cc:45-57)
``*_backproject_adjoint``   no reference counterpart: the plain transpose A^T v
==========================  ======================================================

``lors`` is a CUDA float32 tensor in the reference's ``[C, N]`` layout (one row per
field, as the reference passes ``transpose(lors)``) or in the row-major ``[N, C]``
layout that ``recon_process`` produces; ``layout`` says which ("auto" picks ``[C,N]``
when the first dimension equals C, like the reference). ``image`` is in the kernel's
layout ``[grid[2], grid[1], grid[0]]``; ``grid``/``center``/``size`` are three numbers
each in kernel order (the reference passes ``image.grid[::-1]``). As in the reference,
``image`` given to a back-projection or map op only provides the output's shape.

There is no CPU path: every op requires CUDA tensors and the compiled library.
"""

import torch

from . import _lib, profiling

TOR_COLS = 10
TOR_MAP_COLS = 7
SIDDON_COLS = 7


def _stream(device):
    return torch.cuda.current_stream(device).cuda_stream


def _call(dev, name, *args):
    if profiling._ACTIVE:
        with profiling.timed_call(name, torch.cuda.current_stream(dev)):
            return _lib.call(name, *args)
    return _lib.call(name, *args)


def _check_cuda(*tensors):
    dev = None
    for t in tensors:
        if t is None:
            continue
        if not isinstance(t, torch.Tensor) or not t.is_cuda:
            raise TypeError("srf_b200 ops need CUDA tensors (there is no CPU path)")
        if t.dtype != torch.float32:
            raise TypeError(f"expected float32, got {t.dtype}")
        if dev is None:
            dev = t.device
        elif t.device != dev:
            raise ValueError("all tensors must be on the same device")
    return dev


def _columns(lors, ncols, layout="auto", min_cols=None):
    """Column pointers + event stride for a [C,N] or [N,C] LOR tensor."""
    if lors.dim() != 2:
        raise ValueError(f"lors must be 2-D, got shape {tuple(lors.shape)}")
    need = ncols if min_cols is None else min_cols
    if layout == "auto":
        layout = "cn" if lors.shape[0] in range(need, ncols + 1) else "nc"
    if layout == "cn":
        if lors.shape[0] < need:
            raise ValueError(f"lors [C,N] needs {need} rows, got {lors.shape[0]}")
        t = lors if lors.stride(1) == 1 else lors.contiguous()
        n = t.shape[1]
        base = t.data_ptr()
        cols = [base + 4 * k * t.stride(0) for k in range(t.shape[0])]
        return t, cols, n, 1
    if layout == "nc":
        if lors.shape[1] < need:
            raise ValueError(f"lors [N,C] needs {need} columns, got {lors.shape[1]}")
        t = lors if lors.stride(1) == 1 else lors.contiguous()
        n = t.shape[0]
        base = t.data_ptr()
        cols = [base + 4 * k for k in range(t.shape[1])]
        return t, cols, n, t.stride(0)
    raise ValueError(f"unknown layout {layout!r}")


def _geom(grid, center, size):
    import ctypes as C
    g = [int(v) for v in (grid.tolist() if torch.is_tensor(grid) else grid)]
    c = [float(v) for v in (center.tolist() if torch.is_tensor(center) else center)]
    s = [float(v) for v in (size.tolist() if torch.is_tensor(size) else size)]
    if len(g) != 3 or len(c) != 3 or len(s) != 3:
        raise ValueError("grid, center and size need three values each")
    ga = (C.c_int * 3)(*g)
    ca = (C.c_float * 3)(*c)
    sa = (C.c_float * 3)(*s)
    return g, ga, ca, sa


def _image_shape(g):
    return (g[2], g[1], g[0])


def _as_image(image, g):
    shape = _image_shape(g)
    if image.numel() != shape[0] * shape[1] * shape[2]:
        raise ValueError(f"image has {image.numel()} voxels, grid {g} needs "
                         f"{shape[0] * shape[1] * shape[2]}")
    return image.contiguous()


def _values(v, n):
    if v.numel() != n:
        raise ValueError(f"lors_value has {v.numel()} entries for {n} LORs")
    return v.reshape(-1).contiguous()


def _out_image(out, g, like):
    shape = _image_shape(g)
    if out is None:
        return torch.empty(shape, dtype=torch.float32, device=like.device), False
    if tuple(out.shape) != shape and out.numel() != shape[0] * shape[1] * shape[2]:
        raise ValueError("out has the wrong size")
    if not out.is_contiguous():
        raise ValueError("out must be contiguous")
    return out, True


# ----------------------------------------------------------------------------- TOR


def tor_projection(lors, image, grid, center, size, kernel_width, geo_sigma2_flag=False,
                   tof_bin=1.0e4, tof_sigma2=1.0e4, layout="auto", out=None):
    dev = _check_cuda(lors, image, out)
    t, cols, n, stride = _columns(lors, TOR_COLS, layout)
    g, ga, ca, sa = _geom(grid, center, size)
    img = _as_image(image, g)
    if out is None:
        out = torch.empty(n, dtype=torch.float32, device=dev)
    elif out.numel() != n or not out.is_contiguous():
        raise ValueError("out must be a contiguous tensor with one entry per LOR")
    with torch.cuda.device(dev):
        _call(dev, "srf_tor_projection", *cols[:10], int(bool(geo_sigma2_flag)), out.data_ptr(),
                  ga, ca, sa, float(kernel_width), float(tof_bin), float(tof_sigma2),
                  img.data_ptr(), n, stride, _stream(dev))
    return out


def _tor_scatter(fn, lors, values, image, grid, center, size, kernel_width, geo_sigma2_flag,
                 tof_bin, tof_sigma2, layout, out, accumulate):
    dev = _check_cuda(lors, values, image, out)
    t, cols, n, stride = _columns(lors, TOR_COLS, layout)
    g, ga, ca, sa = _geom(grid, center, size)
    v = _values(values, n)
    res, _ = _out_image(out, g, lors)
    with torch.cuda.device(dev):
        _call(dev, fn, *cols[:10], int(bool(geo_sigma2_flag)), v.data_ptr(), ga, ca, sa,
                  float(kernel_width), float(tof_bin), float(tof_sigma2), res.data_ptr(), n,
                  stride, int(bool(accumulate) and out is not None), _stream(dev))
    return res


def tor_backprojection(image, lors, lors_value, grid, center, size, kernel_width,
                       geo_sigma2_flag=False, tof_bin=1.0e4, tof_sigma2=1.0e4, layout="auto",
                       out=None, accumulate=False):
    """image + sum_i w_i / lors_value[i] over LORs with lors_value > 1e-7 (the
    reference's ``Backprojection``; ``image`` only gives the shape)."""
    return _tor_scatter("srf_tor_backprojection", lors, lors_value, image, grid, center, size,
                        kernel_width, geo_sigma2_flag, tof_bin, tof_sigma2, layout, out,
                        accumulate)


def tor_projection_backprojection(lors, image, grid, center, size, kernel_width,
                                  geo_sigma2_flag=False, tof_bin=1.0e4, tof_sigma2=1.0e4,
                                  layout="auto", out_values=None, out=None, accumulate=False):
    """``tor_projection`` then ``tor_backprojection`` of its values in one call (both
    kernels share one set of per-slab LOR lists). Returns (values, back image)."""
    dev = _check_cuda(lors, image, out_values, out)
    t, cols, n, stride = _columns(lors, TOR_COLS, layout)
    g, ga, ca, sa = _geom(grid, center, size)
    img = _as_image(image, g)
    if out_values is None:
        out_values = torch.empty(n, dtype=torch.float32, device=dev)
    elif out_values.numel() != n or not out_values.is_contiguous():
        raise ValueError("out_values must be a contiguous tensor with one entry per LOR")
    res, _ = _out_image(out, g, lors)
    if res.data_ptr() == img.data_ptr():
        raise ValueError("the back-projection must not overwrite the projected image")
    with torch.cuda.device(dev):
        _call(dev, "srf_tor_projection_backprojection", *cols[:10], int(bool(geo_sigma2_flag)),
              out_values.data_ptr(), ga, ca, sa, float(kernel_width), float(tof_bin),
              float(tof_sigma2), img.data_ptr(), res.data_ptr(), n, stride,
              int(bool(accumulate) and out is not None), _stream(dev))
    return out_values, res


def tor_backproject_adjoint(values, lors, grid, center, size, kernel_width,
                            geo_sigma2_flag=False, tof_bin=1.0e4, tof_sigma2=1.0e4,
                            layout="auto", out=None, accumulate=False):
    """A^T values: the exact transpose of ``tor_projection``."""
    return _tor_scatter("srf_tor_backproject_adjoint", lors, values, None, grid, center, size,
                        kernel_width, geo_sigma2_flag, tof_bin, tof_sigma2, layout, out,
                        accumulate)


def tor_maplors(image, grid, center, size, lors, lors_value, kernel_width,
                geo_sigma2_flag=False, layout="auto", out=None, accumulate=False):
    """The reference's ``Maplors``: lors [7,N] (x1..z2, sigma2_factor), geometric
    weight only, image += w / lors_value with no threshold."""
    dev = _check_cuda(lors, lors_value, image, out)
    t, cols, n, stride = _columns(lors, TOR_MAP_COLS, layout)
    g, ga, ca, sa = _geom(grid, center, size)
    v = _values(lors_value, n)
    res, _ = _out_image(out, g, lors)
    with torch.cuda.device(dev):
        _call(dev, "srf_tor_maplors", *cols[:7], int(bool(geo_sigma2_flag)), v.data_ptr(), ga, ca,
                  sa, float(kernel_width), res.data_ptr(), n, stride,
                  int(bool(accumulate) and out is not None), _stream(dev))
    return res



def tor_maplors_generated(kind, crystals, n_rings, n_blocks, n_per_block, seed, first, count,
                          axis, grid, center, size, kernel_width, geo_sigma2_flag=False,
                          out=None, accumulate=False):
    """Maplors of generated detector-pair LORs ``first .. first+count-1`` of dominant-axis
    group ``axis`` (0, 1, 2) into an image in that group's kernel layout
    (``srf_tor_maplors_generated``: kind 0 random crystal pairs, kind 1 the scanner's
    block-pair enumeration). ``crystals``: CUDA float32 [n_crystals, 3]."""
    dev = _check_cuda(crystals, out)
    if crystals.dtype != torch.float32 or not crystals.is_contiguous() or crystals.dim() != 2 \
            or crystals.shape[1] != 3:
        raise ValueError("crystals must be a contiguous float32 [n, 3] CUDA tensor")
    g, ga, ca, sa = _geom(grid, center, size)
    res, _ = _out_image(out, g, crystals)
    with torch.cuda.device(dev):
        _call(dev, "srf_tor_maplors_generated", int(kind), crystals.data_ptr(), int(n_rings),
              int(n_blocks), int(n_per_block), int(seed) & ((1 << 64) - 1), int(first),
              int(count), int(axis), int(bool(geo_sigma2_flag)), ga, ca, sa,
              float(kernel_width), res.data_ptr(),
              int(bool(accumulate) and out is not None), _stream(dev))
    return res

def tor_count_samples(lors, grid, center, size, kernel_width, geo_sigma2_flag=False,
                      layout="auto"):
    """Per-LOR (non-zero-weight voxels, window voxels visited) as int32 [2, N]: the
    TOR operator's work, independent of the TOF setting."""
    dev = _check_cuda(lors)
    t, cols, n, stride = _columns(lors, TOR_COLS, layout, min_cols=TOR_MAP_COLS)
    g, ga, ca, sa = _geom(grid, center, size)
    counts = torch.empty((2, n), dtype=torch.int32, device=dev)
    fcol = cols[9] if len(cols) >= 10 else cols[6]
    with torch.cuda.device(dev):
        _call(dev, "srf_tor_count_samples", *cols[:6], fcol, int(bool(geo_sigma2_flag)), ga, ca,
                  sa, float(kernel_width), counts.data_ptr(), n, stride, _stream(dev))
    return counts


# -------------------------------------------------------------------------- Siddon


def siddon_count_samples(lors, grid, center, size, layout="auto"):
    """Per-ray voxels visited by the Siddon walk (int32 [N]): the operator's work."""
    dev = _check_cuda(lors)
    t, cols, n, stride = _columns(lors, SIDDON_COLS, layout, min_cols=6)
    g, ga, ca, sa = _geom(grid, center, size)
    counts = torch.empty(n, dtype=torch.int32, device=dev)
    with torch.cuda.device(dev):
        _call(dev, "srf_siddon_count_samples", *cols[:6], ga, ca, sa, counts.data_ptr(), n,
              stride, _stream(dev))
    return counts


def siddon_projection(lors, image, grid, center, size, tof_bin=1.0e4, tof_sigma2=1.0e4,
                      layout="auto", out=None):
    dev = _check_cuda(lors, image, out)
    t, cols, n, stride = _columns(lors, SIDDON_COLS, layout)
    g, ga, ca, sa = _geom(grid, center, size)
    img = _as_image(image, g)
    if out is None:
        out = torch.empty(n, dtype=torch.float32, device=dev)
    elif out.numel() != n or not out.is_contiguous():
        raise ValueError("out must be a contiguous tensor with one entry per LOR")
    with torch.cuda.device(dev):
        _call(dev, "srf_siddon_projection", *cols[:7], out.data_ptr(), ga, ca, sa,
                  float(tof_bin), float(tof_sigma2), img.data_ptr(), n, stride, _stream(dev))
    return out


def _siddon_scatter(fn, lors, values, image, grid, center, size, tof_bin, tof_sigma2, layout,
                    out, accumulate):
    dev = _check_cuda(lors, values, image, out)
    t, cols, n, stride = _columns(lors, SIDDON_COLS, layout)
    g, ga, ca, sa = _geom(grid, center, size)
    v = _values(values, n)
    res, _ = _out_image(out, g, lors)
    with torch.cuda.device(dev):
        _call(dev, fn, *cols[:7], v.data_ptr(), ga, ca, sa, float(tof_bin), float(tof_sigma2),
                  res.data_ptr(), n, stride, int(bool(accumulate) and out is not None),
                  _stream(dev))
    return res


def siddon_backprojection(image, lors, lors_value, grid, center, size, tof_bin=1.0e4,
                          tof_sigma2=1.0e4, layout="auto", out=None, accumulate=False):
    return _siddon_scatter("srf_siddon_backprojection", lors, lors_value, image, grid, center,
                           size, tof_bin, tof_sigma2, layout, out, accumulate)


def siddon_backproject_adjoint(values, lors, grid, center, size, tof_bin=1.0e4,
                               tof_sigma2=1.0e4, layout="auto", out=None, accumulate=False):
    return _siddon_scatter("srf_siddon_backproject_adjoint", lors, values, None, grid, center,
                           size, tof_bin, tof_sigma2, layout, out, accumulate)


def siddon_maplors(image, grid, center, size, lors, lors_value, layout="auto", out=None,
                   accumulate=False):
    """The reference's Siddon ``Maplors``: only x1..z2 of ``lors`` are read."""
    dev = _check_cuda(lors, lors_value, image, out)
    t, cols, n, stride = _columns(lors, SIDDON_COLS, layout, min_cols=6)
    g, ga, ca, sa = _geom(grid, center, size)
    v = _values(lors_value, n)
    res, _ = _out_image(out, g, lors)
    with torch.cuda.device(dev):
        _call(dev, "srf_siddon_maplors", *cols[:6], v.data_ptr(), ga, ca, sa, res.data_ptr(), n,
                  stride, int(bool(accumulate) and out is not None), _stream(dev))
    return res


# --------------------------------------------------------------------- image algebra


def mlem_update_(image, effinv, bp):
    """In place: image *= effinv * bp (``mlem_update``, model/recon_step.py:48-49)."""
    dev = _check_cuda(image, effinv, bp)
    if not (image.is_contiguous() and effinv.is_contiguous() and bp.is_contiguous()):
        raise ValueError("mlem_update_ needs contiguous tensors")
    if not (image.numel() == effinv.numel() == bp.numel()):
        raise ValueError("image, effinv and bp must have the same number of voxels")
    with torch.cuda.device(dev):
        _call(dev, "srf_mlem_update", image.data_ptr(), effinv.data_ptr(), bp.data_ptr(),
                  image.numel(), _stream(dev))
    return image


# ------------------------------------------------------------------ batched frames


def _frame_args(frame, n_frames, images_numel, g):
    if frame is None or frame.dtype != torch.int32 or not frame.is_cuda:
        raise TypeError("frame must be a CUDA int32 tensor")
    nvox = g[0] * g[1] * g[2]
    if images_numel != n_frames * nvox:
        raise ValueError(f"images hold {images_numel} voxels, {n_frames} frames need "
                         f"{n_frames * nvox}")
    return frame.contiguous(), nvox


def tor_projection_batched(lors, frame, images, n_frames, grid, center, size, kernel_width,
                           geo_sigma2_flag=False, tof_bin=1.0e4, tof_sigma2=1.0e4,
                           layout="auto", out=None):
    """Projection of LOR i through image images[frame[i]]; images [F, g2, g1, g0]."""
    dev = _check_cuda(lors, images, out)
    t, cols, n, stride = _columns(lors, TOR_COLS, layout)
    g, ga, ca, sa = _geom(grid, center, size)
    fr, nvox = _frame_args(frame, n_frames, images.numel(), g)
    if fr.numel() != n:
        raise ValueError("frame needs one entry per LOR")
    imgs = images.contiguous()
    if out is None:
        out = torch.empty(n, dtype=torch.float32, device=dev)
    with torch.cuda.device(dev):
        _call(dev, "srf_tor_projection_batched", *cols[:10], int(bool(geo_sigma2_flag)),
              fr.data_ptr(), int(n_frames), nvox, out.data_ptr(), ga, ca, sa,
              float(kernel_width), float(tof_bin), float(tof_sigma2), imgs.data_ptr(), n, stride,
              _stream(dev))
    return out


def tor_projection_backprojection_batched(lors, frame, images, n_frames, grid, center, size,
                                          kernel_width, geo_sigma2_flag=False, tof_bin=1.0e4,
                                          tof_sigma2=1.0e4, layout="auto", out_values=None,
                                          out=None, accumulate=False):
    """``tor_projection_batched`` then ``tor_backprojection_batched`` of its values in one
    call (one set of per-slab LOR lists for both). Returns (values, back images)."""
    dev = _check_cuda(lors, images, out_values, out)
    t, cols, n, stride = _columns(lors, TOR_COLS, layout)
    g, ga, ca, sa = _geom(grid, center, size)
    fr, nvox = _frame_args(frame, n_frames, images.numel(), g)
    if fr.numel() != n:
        raise ValueError("frame needs one entry per LOR")
    imgs = images.contiguous()
    if out_values is None:
        out_values = torch.empty(n, dtype=torch.float32, device=dev)
    elif out_values.numel() != n or not out_values.is_contiguous():
        raise ValueError("out_values must be a contiguous tensor with one entry per LOR")
    if out is None:
        out = torch.empty((n_frames, g[2], g[1], g[0]), dtype=torch.float32, device=dev)
        accumulate = False
    elif out.numel() != n_frames * nvox or not out.is_contiguous():
        raise ValueError("out must be a contiguous stack of n_frames images")
    if out.data_ptr() == imgs.data_ptr():
        raise ValueError("the back-projection must not overwrite the projected images")
    with torch.cuda.device(dev):
        _call(dev, "srf_tor_projection_backprojection_batched", *cols[:10],
              int(bool(geo_sigma2_flag)), fr.data_ptr(), int(n_frames), nvox,
              out_values.data_ptr(), ga, ca, sa, float(kernel_width), float(tof_bin),
              float(tof_sigma2), imgs.data_ptr(), out.data_ptr(), n, stride,
              int(bool(accumulate)), _stream(dev))
    return out_values, out


def tor_projection_backprojection_batched_strided(lors, frame, images, back, grid, center,
                                                  size, kernel_width, geo_sigma2_flag=False,
                                                  tof_bin=1.0e4, tof_sigma2=1.0e4,
                                                  layout="auto", out_values=None,
                                                  accumulate=True):
    """``tor_projection_backprojection_batched`` on image stacks in any axis order:
    ``images`` and ``back`` are [F, gz, gy, gx] views (the kernel's axes, e.g. a permuted
    view of an [F, nx, ny, nz] stack) with the same strides; ``back`` += the
    back-projection (unless ``accumulate``, all F x stride(0) floats from its base are
    zeroed first). Returns the projected values."""
    dev = _check_cuda(lors, images, back, out_values)
    t, cols, n, stride = _columns(lors, TOR_COLS, layout)
    g, ga, ca, sa = _geom(grid, center, size)
    if images.dim() != 4 or tuple(images.shape[1:]) != (g[2], g[1], g[0]):
        raise ValueError("images must be an [F, gz, gy, gx] view")
    if back.shape != images.shape or back.stride() != images.stride():
        raise ValueError("back must be a view of the same shape and strides as images")
    if images.dtype != torch.float32 or back.dtype != torch.float32:
        raise TypeError("images must be float32")
    import ctypes as C
    n_frames = int(images.shape[0])
    fs = int(images.stride(0))
    fr, _ = _frame_args(frame, n_frames, images.numel(), g)
    if fr.numel() != n:
        raise ValueError("frame needs one entry per LOR")
    if back.data_ptr() == images.data_ptr():
        raise ValueError("the back-projection must not overwrite the projected images")
    if out_values is None:
        out_values = torch.empty(n, dtype=torch.float32, device=dev)
    elif out_values.numel() != n or not out_values.is_contiguous():
        raise ValueError("out_values must be a contiguous tensor with one entry per LOR")
    st = (C.c_int64 * 3)(int(images.stride(3)), int(images.stride(2)), int(images.stride(1)))
    with torch.cuda.device(dev):
        _call(dev, "srf_tor_projection_backprojection_batched_strided", *cols[:10],
              int(bool(geo_sigma2_flag)), fr.data_ptr(), n_frames, fs, out_values.data_ptr(),
              ga, ca, sa, float(kernel_width), float(tof_bin), float(tof_sigma2),
              images.data_ptr(), back.data_ptr(), st, n, stride, int(bool(accumulate)),
              _stream(dev))
    return out_values


def _tor_scatter_batched(fn, lors, frame, values, n_frames, grid, center, size, kernel_width,
                         geo_sigma2_flag, tof_bin, tof_sigma2, layout, out, accumulate):
    dev = _check_cuda(lors, values, out)
    t, cols, n, stride = _columns(lors, TOR_COLS, layout)
    g, ga, ca, sa = _geom(grid, center, size)
    nvox = g[0] * g[1] * g[2]
    if out is None:
        out = torch.empty((n_frames, g[2], g[1], g[0]), dtype=torch.float32, device=dev)
        accumulate = False
    fr, _ = _frame_args(frame, n_frames, out.numel(), g)
    v = _values(values, n)
    with torch.cuda.device(dev):
        _call(dev, fn, *cols[:10], int(bool(geo_sigma2_flag)), fr.data_ptr(), int(n_frames), nvox,
              v.data_ptr(), ga, ca, sa, float(kernel_width), float(tof_bin), float(tof_sigma2),
              out.data_ptr(), n, stride, int(bool(accumulate)), _stream(dev))
    return out


def tor_backprojection_batched(lors, frame, lors_value, n_frames, grid, center, size,
                               kernel_width, geo_sigma2_flag=False, tof_bin=1.0e4,
                               tof_sigma2=1.0e4, layout="auto", out=None, accumulate=False):
    """Reference back-projection A^T(1/v) of each LOR into its frame's image."""
    return _tor_scatter_batched("srf_tor_backprojection_batched", lors, frame, lors_value,
                                n_frames, grid, center, size, kernel_width, geo_sigma2_flag,
                                tof_bin, tof_sigma2, layout, out, accumulate)


def tor_backproject_adjoint_batched(values, lors, frame, n_frames, grid, center, size,
                                    kernel_width, geo_sigma2_flag=False, tof_bin=1.0e4,
                                    tof_sigma2=1.0e4, layout="auto", out=None,
                                    accumulate=False):
    """Plain adjoint A^T values per frame."""
    return _tor_scatter_batched("srf_tor_backproject_adjoint_batched", lors, frame, values,
                                n_frames, grid, center, size, kernel_width, geo_sigma2_flag,
                                tof_bin, tof_sigma2, layout, out, accumulate)
