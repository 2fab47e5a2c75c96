"""Timing of the reference's own CUDA projector kernels (src/cpp/tf_custom_ops/tor.cu.cc
built for sm_100a by oracle/Makefile) against this library on the same B200 and the
same LORs: the primary TOF-TOR configuration (128x128x64 at 3.2 mm, kernel_width
10.19 mm, 530 ps), one dominant-axis group of 1M events. Results (ms and the ratio) go
to SRF_PARITY_LOG. Skipped where oracle/_ref was not built."""

import math

import numpy as np
import pytest
import torch

from oracle import pyoracle as O
from srf_b200 import ops
from srf_b200 import preprocess as PP
from srf_b200 import synthetic as S
from srf_b200.physics import SplitLoRsModel
from srf_b200.scanner import tof_info
from tests.test_gpu_parity import record

pytestmark = pytest.mark.gpu


def _time(fn, reps=3):
    fn()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps


def test_reference_gpu_kernels_timing():
    if not O.ReferenceGPU.available():
        pytest.skip("reference GPU build not present")
    R = O.ReferenceGPU()
    wl = S.tor_128()
    tof_bin, tof_sigma2 = tof_info(wl.tof_res_ps, wl.tof_bin_ps)
    ph = S.standard_phantom(half_length=wl.scanner.axial_length / 2)
    ev = S.generate_events(1_000_000, wl.scanner, ph, seed=3,
                           tof_sigma_mm=math.sqrt(tof_sigma2), device="cuda")
    g = PP.recon_process(ev, wl.tof_res_ps)["x"]
    img = torch.as_tensor(ph.voxelize(wl.grid, wl.center, wl.size) + 0.05, device="cuda")
    model = SplitLoRsModel(wl.kernel_width, False, tof_sigma2=tof_sigma2, tof_bin=tof_bin)
    kimg = img.permute(*model.perm("x")).contiguous()
    grid = list(kimg.shape[::-1])
    c = [0.0, 0.0, 0.0]
    size = [wl.voxel * n for n in grid]
    soa = g.t().contiguous()  # the reference op's [10, N] columns
    n = g.shape[0]
    kw = float(np.float32(wl.kernel_width))

    ref_pv = R.tor_projection(soa, kimg, grid, c, size, kw, False, tof_bin, tof_sigma2)
    our_pv = ops.tor_projection(g, kimg, grid, c, size, kw, False, tof_bin, tof_sigma2,
                                layout="nc")
    err = float((our_pv.double() - ref_pv.double()).norm() / ref_pv.double().norm())
    assert err <= 1e-5

    ref_ms = _time(lambda: (R.tor_projection(soa, kimg, grid, c, size, kw, False, tof_bin,
                                             tof_sigma2),
                            R.tor_backprojection(soa, ref_pv, grid, c, size, kw, False, tof_bin,
                                                 tof_sigma2)), reps=2)
    our_ms = _time(lambda: (ops.tor_projection(g, kimg, grid, c, size, kw, False, tof_bin,
                                               tof_sigma2, layout="nc"),
                            ops.tor_backprojection(kimg, g, our_pv, grid, c, size, kw, False,
                                                   tof_bin, tof_sigma2, layout="nc")))
    record("reference_gpu_timing", lors=n, reference_ms=ref_ms, ours_ms=our_ms,
           speedup=ref_ms / our_ms, rel_l2_projection=err,
           workload="x group of 1M events, 128x128x64, kw 10.19, TOF 530 ps")
    assert our_ms < ref_ms


def test_reference_gpu_siddon_timing():
    """The reference's own Siddon kernels (siddon.cu.cc for sm_100a) against this library,
    plain non-TOF Siddon at 64x64x32 (3.4 mm): 1M seeded events from the cylinder
    phantom, tof_sigma2 = 1e6 (TOF off). Rays the oracle's walk does not visit (misses,
    and rays that would make the reference read outside the image) are left out of both."""
    if not O.ReferenceGPU.available():
        pytest.skip("reference GPU build not present")
    from srf_b200.physics import CompleteLoRsModel
    from srf_b200.data import Image
    R = O.ReferenceGPU()
    wl = S.siddon_64()
    ph = S.standard_phantom(half_length=wl.scanner.axial_length / 2)
    ev = S.generate_events(1_000_000, wl.scanner, ph, seed=wl.seed, device="cuda")
    img = torch.as_tensor(ph.voxelize(wl.grid, wl.center, wl.size) + np.float32(0.05),
                          device="cuda")
    model = CompleteLoRsModel(tof_sigma2=1.0e6, tof_bin=1.0e4)
    kimg, g, c, sz = model.kernel_geometry(Image(img, wl.center, wl.size))
    kimg = kimg.contiguous()
    ev_np = ev.cpu().numpy()
    visits, _ = O.siddon_counts(np.ascontiguousarray(ev_np.T), g, c, sz)
    sel = ev_np[visits > 0]
    rows = torch.as_tensor(np.ascontiguousarray(sel), device="cuda")
    soa = rows.t().contiguous()  # the reference op's [7, N] columns
    b, s2 = model.tof_bin, model.tof_sigma2

    ref_pv = R.siddon_projection(soa, kimg, g, c, sz, b, s2)
    our_pv = ops.siddon_projection(rows, kimg, g, c, sz, b, s2, layout="nc")
    err = float((our_pv.double() - ref_pv.double()).norm() / ref_pv.double().norm())
    assert err <= 1e-5
    ref_bp = R.siddon_backprojection(soa, ref_pv, g, c, sz, b, s2)
    our_bp = ops.siddon_backprojection(kimg, rows, ref_pv, g, c, sz, b, s2, layout="nc")
    err_b = float((our_bp.double() - ref_bp.double()).norm() / ref_bp.double().norm())
    assert err_b <= 1e-5

    ref_ms = _time(lambda: (R.siddon_projection(soa, kimg, g, c, sz, b, s2),
                            R.siddon_backprojection(soa, ref_pv, g, c, sz, b, s2)))
    our_ms = _time(lambda: (ops.siddon_projection(rows, kimg, g, c, sz, b, s2, layout="nc"),
                            ops.siddon_backprojection(kimg, rows, our_pv, g, c, sz, b, s2,
                                                      layout="nc")))
    record("reference_gpu_siddon_timing", rays=int(rows.shape[0]), reference_ms=ref_ms,
           ours_ms=our_ms, speedup=ref_ms / our_ms, rel_l2_projection=err,
           rel_l2_backprojection=err_b,
           workload="1M events (rays visiting the image), 64x64x32 at 3.4 mm, non-TOF")
    assert our_ms < ref_ms
