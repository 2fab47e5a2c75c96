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
