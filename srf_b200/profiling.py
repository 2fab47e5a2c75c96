"""Per-launch device timing of library calls with CUDA events.

``with KernelTimer() as kt: ...`` records a start/end event pair on the launching
stream around every library entry point called inside the block (no host
synchronisation while recording); ``kt.summary()`` synchronises once and returns, per
entry point, the launch count and total/mean device milliseconds. NVTX ranges are
pushed per call as well, so an external profiler shows the same names.
"""

import collections
import contextlib

import torch

_ACTIVE = []


class KernelTimer:
    def __init__(self, enabled=True):
        self.enabled = enabled
        self.records = []  # (name, start_event, end_event)

    def __enter__(self):
        if self.enabled:
            _ACTIVE.append(self)
        return self

    def __exit__(self, *exc):
        if self.enabled and _ACTIVE and _ACTIVE[-1] is self:
            _ACTIVE.pop()
        return False

    def clear(self):
        self.records = []

    def summary(self):
        torch.cuda.synchronize()
        out = collections.OrderedDict()
        for name, s, e in self.records:
            ms = s.elapsed_time(e)
            d = out.setdefault(name, {"launches": 0, "total_ms": 0.0})
            d["launches"] += 1
            d["total_ms"] += ms
        for d in out.values():
            d["mean_ms"] = d["total_ms"] / d["launches"]
        return out


@contextlib.contextmanager
def timed_call(name, stream):
    """Used by the binding around each library call."""
    if not _ACTIVE:
        yield
        return
    t = _ACTIVE[-1]
    s = torch.cuda.Event(enable_timing=True)
    e = torch.cuda.Event(enable_timing=True)
    s.record(stream)
    torch.cuda.nvtx.range_push(name)
    try:
        yield
    finally:
        torch.cuda.nvtx.range_pop()
        e.record(stream)
        t.records.append((name, s, e))


def measure_peaks(device=None, l2_mib=48, l2_reps=20, ex2_iters=4096, smem_iters=8192,
                  atomic_iters=2048):
    """Measured L2 read bandwidth (GB/s), ex2 throughput (per second), shared-memory read
    bandwidth (GB/s) and shared-memory float atomicAdd rates (per second; lanes on
    distinct banks, and hashed addresses) of this GPU, from the library's probe kernels
    (``srf_probe_l2_read``, ``srf_probe_ex2``, ``srf_probe_smem_read``,
    ``srf_probe_smem_atomic``): one warm-up and one timed launch each, CUDA events on the
    current stream. The L2 buffer (default 48 MiB) stays resident in the 126 MB L2."""
    import ctypes

    from . import _lib
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
    with torch.cuda.device(dev):
        nt = ctypes.c_int64(0)
        _lib.call("srf_probe_threads", ctypes.byref(nt))
        sink = torch.empty(nt.value, dtype=torch.float32, device=dev)
        n = l2_mib * (1 << 20) // 4
        buf = torch.rand(n, dtype=torch.float32, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

        def timed(fn):
            fn()
            s.record()
            fn()
            e.record()
            torch.cuda.synchronize(dev)
            return s.elapsed_time(e) / 1e3

        t_l2 = timed(lambda: _lib.call("srf_probe_l2_read", buf.data_ptr(), n, l2_reps,
                                       sink.data_ptr(), stream))
        t_ex2 = timed(lambda: _lib.call("srf_probe_ex2", ex2_iters, sink.data_ptr(), stream))
        ns = ctypes.c_int64(0)
        _lib.call("srf_probe_smem_threads", ctypes.byref(ns))
        ssink = torch.empty(ns.value, dtype=torch.float32, device=dev)
        t_sm = timed(lambda: _lib.call("srf_probe_smem_read", smem_iters, ssink.data_ptr(),
                                       stream))
        t_at = timed(lambda: _lib.call("srf_probe_smem_atomic", atomic_iters, 0,
                                       ssink.data_ptr(), stream))
        t_ar = timed(lambda: _lib.call("srf_probe_smem_atomic", atomic_iters, 1,
                                       ssink.data_ptr(), stream))
    l2_bytes = l2_reps * (n // 4) * 16
    return {"l2_gbs": l2_bytes / t_l2 / 1e9, "ex2_per_s": nt.value * 8 * ex2_iters / t_ex2,
            "smem_gbs": ns.value * smem_iters * 16 / t_sm / 1e9,
            "smem_atomic_per_s": ns.value * atomic_iters / t_at,
            "smem_atomic_random_per_s": ns.value * atomic_iters / t_ar,
            "l2_buffer_mib": l2_mib,
            "method": "srf_probe_l2_read / srf_probe_ex2 / srf_probe_smem_read / "
                      "srf_probe_smem_atomic, CUDA events"}
