"""List-mode files and streaming them onto the GPU.

Formats (the reference's, ``src/python/srf/io/listmode.py:8-32`` and
``src/python/srf/data/loader.py:96-145``):

* ``.npy``: float32 ``[N, 7]`` rows ``x1, y1, z1, x2, y2, z2, tof`` (or ``[N, 6]`` without
  TOF). Read memory-mapped, so a file larger than host memory streams in chunks.
* ``.h5``: group ``listmode_data`` with datasets ``fst`` [N,3], ``snd`` [N,3] and optional
  ``tof`` [N] and ``weight`` [N]. Needs h5py, which is optional here.

``stream_events`` moves a file (or any ``[N, C]`` array) to the GPU chunk by chunk through
two pinned staging buffers on a copy stream, so the upload of chunk k+1 overlaps the
caller's work on chunk k; ``load_split`` / ``load_complete`` build the model inputs the
reference's ``SplitWorkerLoader`` / ``CompleteWorkerLoader`` build.
"""

import os

import numpy as np
import torch

from .data import Image, ListModeData

H5_GROUP = "listmode_data"


def _h5py():
    try:
        import h5py
    except ImportError as exc:  # optional dependency
        raise ImportError("reading .h5 list-mode files needs h5py; convert the file to .npy "
                          "([N,7] float32: fst, snd, tof) or install h5py") from exc
    return h5py


def load_listmode(path, mmap=True):
    """Events of a list-mode file as a float32 numpy array [N, 7] (x1..z2, tof) or
    [N, 6] for an h5 file without ``tof``. ``.npy`` files are memory-mapped."""
    path = os.fspath(path)
    if path.endswith(".npy"):
        a = np.load(path, mmap_mode="r" if mmap else None)
        if a.ndim != 2 or a.shape[1] < 6:
            raise ValueError(f"{path}: expected an [N, 6] or [N, 7] array, got {a.shape}")
        if a.dtype != np.float32:
            a = np.asarray(a, dtype=np.float32)
        return a
    if path.endswith(".h5"):
        h5py = _h5py()
        with h5py.File(path, "r") as f:
            g = f[H5_GROUP]
            cols = [np.asarray(g["fst"], np.float32), np.asarray(g["snd"], np.float32)]
            if "tof" in g:
                cols.append(np.asarray(g["tof"], np.float32).reshape(-1, 1))
            return np.ascontiguousarray(np.hstack(cols))
    raise ValueError(f"{path}: unknown list-mode format (expected .npy or .h5)")


def save_listmode(path, events):
    """Write [N, 6|7] events as ``.npy`` (float32) or as the reference's h5 layout."""
    path = os.fspath(path)
    ev = np.ascontiguousarray(np.asarray(events, dtype=np.float32))
    if path.endswith(".npy"):
        np.save(path, ev)
        return
    if path.endswith(".h5"):
        h5py = _h5py()
        with h5py.File(path, "w") as f:
            g = f.create_group(H5_GROUP)
            g.create_dataset("fst", data=ev[:, 0:3], compression="gzip")
            g.create_dataset("snd", data=ev[:, 3:6], compression="gzip")
            if ev.shape[1] > 6:
                g.create_dataset("tof", data=ev[:, 6], compression="gzip")
        return
    raise ValueError(f"{path}: unknown list-mode format (expected .npy or .h5)")


def chunk_bounds(n, chunk):
    """[start, stop) ranges of consecutive chunks covering n rows."""
    if chunk < 1:
        raise ValueError("chunk must be positive")
    return [(s, min(n, s + chunk)) for s in range(0, n, chunk)]


def stream_events(source, chunk=16_000_000, device=None):
    """Yield the rows of ``source`` (a path or an [N, C] array) as contiguous float32 CUDA
    tensors of at most ``chunk`` rows, in order. Two pinned host buffers alternate: chunk
    k+1 is copied into one and uploaded on a separate stream while the caller works on
    chunk k (each yielded tensor is ready on the current stream). Three device buffers
    rotate, so a yielded tensor stays valid until the generator is advanced twice: the
    caller may hold chunk k while it works on chunk k+1 (neighbouring chunks in pairs).
    Clone a chunk to keep it longer (``list(stream_events(...))`` without cloning
    would hold aliases of the three buffers)."""
    arr = load_listmode(source) if isinstance(source, (str, os.PathLike)) else source
    if arr.ndim != 2:
        raise ValueError("source must be an [N, C] array")
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
    n, c = arr.shape
    if n == 0:
        return
    rows = min(chunk, n)
    pinned = [torch.empty((rows, c), dtype=torch.float32).pin_memory() for _ in range(2)]
    n_dev = min(3, (n + rows - 1) // rows)
    gpu = [torch.empty((rows, c), dtype=torch.float32, device=dev) for _ in range(n_dev)]
    copy = torch.cuda.Stream(device=dev)
    staged = [None, None]  # per pinned buffer: its last upload's event
    ready = [None] * n_dev  # per device buffer: the event of the upload it holds
    bounds = chunk_bounds(n, rows)

    def upload(k):
        s, e = bounds[k]
        h, d = k % 2, k % n_dev
        if staged[h] is not None:
            staged[h].synchronize()  # the pinned buffer's previous upload has finished
        pinned[h][: e - s].numpy()[:] = arr[s:e]
        with torch.cuda.stream(copy):
            # the caller's work queued so far (on chunks up to k-1) is done with gpu[d],
            # which last held chunk k-3
            copy.wait_stream(torch.cuda.current_stream(dev))
            gpu[d][: e - s].copy_(pinned[h][: e - s], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(copy)
        staged[h] = ready[d] = ev

    upload(0)
    for k in range(len(bounds)):
        if k + 1 < len(bounds):
            upload(k + 1)
        s, e = bounds[k]
        torch.cuda.current_stream(dev).wait_event(ready[k % n_dev])
        yield gpu[k % n_dev][: e - s]


def load_split(lors_path, tof_res, emap_path=None, center=None, size=None, chunk=16_000_000,
               device=None):
    """``SplitWorkerLoader.load``: events -> ``recon_process`` on the GPU chunk by chunk ->
    ListModeDataSplit with values of one (and the efficiency map as an Image). Each axis
    group holds the rows a single ``recon_process`` call gives, ordered chunk by chunk
    (the sums of projection and back-projection do not depend on the order)."""
    from .data import ListModeDataSplit
    from .preprocess import recon_process
    parts = {a: [] for a in "xyz"}
    for ev in stream_events(lors_path, chunk, device):
        groups = recon_process(ev, tof_res)
        for a in "xyz":
            parts[a].append(groups[a])
    groups = {a: (torch.cat(v) if v else torch.zeros((0, 10), device="cuda"))
              for a, v in parts.items()}
    data = ListModeDataSplit(*[ListModeData(groups[a], torch.ones(groups[a].shape[0],
                                                                  device=groups[a].device))
                               for a in "xyz"])
    out = {"projection_data": data}
    if emap_path is not None:
        out["efficiency_map"] = _load_image(emap_path, center, size, data.x.lors.device)
    return out


def load_complete(lors_path, emap_path=None, center=None, size=None, device=None):
    """``CompleteWorkerLoader.load``: [N, 7] events as ListModeData (values: the TOF
    column, as the reference's loader sets them) on the GPU."""
    arr = load_listmode(lors_path)
    if arr.shape[1] < 7:
        arr = np.hstack([arr[:, :6], np.ones((arr.shape[0], 1), np.float32)])
    # each chunk is copied out before the generator reuses its buffer
    ev = torch.cat([c.clone() for c in stream_events(np.ascontiguousarray(arr[:, :7]),
                                                      device=device)])
    out = {"projection_data": ListModeData(ev, ev[:, 6].contiguous())}
    if emap_path is not None:
        out["efficiency_map"] = _load_image(emap_path, center, size, ev.device)
    return out


def _load_image(path, center, size, device):
    if center is None or size is None:
        raise ValueError("an efficiency map needs the image center and size")
    a = np.load(os.fspath(path)).astype(np.float32)
    return Image(torch.as_tensor(a, device=device), center, size)
