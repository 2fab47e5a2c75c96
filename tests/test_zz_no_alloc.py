"""srf_recon_process_noalloc: LOR preprocessing for callers that cannot allocate device
memory when they preprocess (a service with a fixed memory budget that forbids
allocations after start-up, or a latency-critical path that cannot take cudaMalloc's
implicit device synchronisation). It runs the same kernels as srf_recon_process with
the scratch taken from a buffer inside the library, so its output must equal the
workspace entry point's exactly.

Called through the C ABI with ctypes. Two calls in a row on different inputs (the
second smaller than the first) check that nothing from the previous call's scratch
leaks into the next. This file is collected last so a failure here comes after every
other test has run; it also passes alone in a fresh process.
"""

import ctypes

import numpy as np
import pytest
import torch

from srf_b200 import _lib
from tests import _cases as K

pytestmark = pytest.mark.gpu

MAX_EVENTS = 8388608  # SRF_RECON_PROCESS_NOALLOC_MAX_EVENTS in include/srf_b200.h


def _with_workspace(lib, ev, tof_res):
    n = ev.shape[0]
    ws_bytes = int(lib.srf_preprocess_workspace_size(n))
    ws = torch.empty(max(ws_bytes, 256), dtype=torch.uint8, device="cuda")
    out = torch.full((n, 10), -1.0, dtype=torch.float32, device="cuda")
    counts = torch.zeros(3, dtype=torch.int64, device="cuda")
    st = lib.srf_recon_process(ev.data_ptr(), n, ev.stride(0), tof_res, out.data_ptr(),
                               counts.data_ptr(), ws.data_ptr(), ws.numel(),
                               torch.cuda.current_stream().cuda_stream)
    assert st == 0, lib.srf_status_string(st)
    return out, counts


def _no_alloc(lib, ev, tof_res):
    n = ev.shape[0]
    out = torch.full((n, 10), -1.0, dtype=torch.float32, device="cuda")
    counts = torch.zeros(3, dtype=torch.int64, device="cuda")
    st = lib.srf_recon_process_noalloc(ev.data_ptr(), n, ev.stride(0), tof_res, out.data_ptr(),
                                       counts.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert st == 0, lib.srf_status_string(st)
    return out, counts


def test_no_alloc_matches_workspace_entry_point_twice():
    lib = _lib.load()
    first = np.vstack([K.events(30000, 91, 530.0), K.box_events(6000, 92)]).astype(np.float32)
    second = np.vstack([K.events(9000, 93, 530.0), K.box_events(2000, 94)]).astype(np.float32)
    for events, tof_res in ((first, 530.0), (second, 530.0)):
        ev = torch.as_tensor(events).cuda().contiguous()
        ref_out, ref_counts = _with_workspace(lib, ev, tof_res)
        got_out, got_counts = _no_alloc(lib, ev, tof_res)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(got_counts.cpu().numpy(), ref_counts.cpu().numpy())
        total = int(ref_counts.sum())
        assert total > 0
        # exact equality (stricter than the 1e-5 rel-L2 used for the projectors):
        # both entry points run the same kernels on the same inputs
        np.testing.assert_array_equal(got_out[:total].cpu().numpy(),
                                      ref_out[:total].cpu().numpy())


def test_no_alloc_rejects_too_many_events():
    lib = _lib.load()
    ev = torch.zeros((4, 7), dtype=torch.float32, device="cuda")
    out = torch.zeros((4, 10), dtype=torch.float32, device="cuda")
    counts = torch.zeros(3, dtype=torch.int64, device="cuda")
    st = lib.srf_recon_process_noalloc(ev.data_ptr(), MAX_EVENTS + 1, 7, 530.0, out.data_ptr(),
                                       counts.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert st == 3  # SRF_ERR_UNSUPPORTED, nothing launched
    assert lib.srf_status_string(st) == b"unsupported parameters"


def test_no_alloc_at_the_event_limit():
    """A call with exactly SRF_RECON_PROCESS_NOALLOC_MAX_EVENTS events uses the whole
    built-in scratch; it must still equal the workspace entry point, then a small call
    right after it must too."""
    lib = _lib.load()
    big = K.box_events(MAX_EVENTS, 95)
    small = K.box_events(5000, 96)
    for events in (big, small):
        ev = torch.as_tensor(events).cuda().contiguous()
        ref_out, ref_counts = _with_workspace(lib, ev, 530.0)
        got_out, got_counts = _no_alloc(lib, ev, 530.0)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(got_counts.cpu().numpy(), ref_counts.cpu().numpy())
        assert int(ref_counts.sum()) == events.shape[0]
        assert torch.equal(got_out, ref_out)
        del ev, ref_out, got_out
