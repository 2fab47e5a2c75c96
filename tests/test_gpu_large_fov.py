"""GPU parity at the large axial FOV geometry: 256x256x128 image at 2.5 mm, ring scanner
R 390 mm with 600 crystals x 320 rings over 1 m, TOF 400 ps (tof_sigma2 649.21 mm^2),
TOR FWHM 4 mm (kernel_width 10.19 mm, window 7 x 7 at 2.5 mm). At 256-wide kernel slices
fewer than four padded slices fit in shared memory, so the default slab kernels run on
bands of rows (46 rows x 4 slices); every kernel family is checked here at that geometry:
projection, back-projection A^T(1/v), map and the combined call against the oracle's f32
mode (<= 1e-5 rel-L2) and its FP64 mode (the documented bound), against the reference's
own sm_100a kernels where they were built, a chunked run against one pass, and the
per-LOR work counts against the oracle's.
Reference: src/cpp/tf_custom_ops/tor.cu.cc:348-481 (launchers), :22-242 (operator)."""

import numpy as np
import pytest

from oracle import preprocess_ref as P
from oracle import pyoracle as O
from srf_b200 import ops
from tests import _cases as K
from tests.test_gpu_parity import FP64_TOL, TOL, TOR_PATHS, cu, host, record

pytestmark = pytest.mark.gpu

RES = 400.0


@pytest.fixture(scope="module")
def lcase():
    return K.large_case(n=6000, seed=71, n_box=1500, tof_res=RES)


@pytest.fixture(params=list(TOR_PATHS))
def tor_path(request):
    from srf_b200 import tuning
    tuning.set_tuning(*TOR_PATHS[request.param])
    yield request.param
    tuning.set_tuning()


def _params(geo):
    b, s2 = K.tof_params(RES)
    assert abs(s2 - 649.21) < 0.01
    return (4.0 if geo else K.KW_CONFIG), geo, b, s2


@pytest.mark.parametrize("geo", [False, True])
@pytest.mark.parametrize("axis", ["x", "y", "z"])
def test_large_fov_projection_backprojection(lcase, axis, geo, tor_path):
    kw, geo, b, s2 = _params(geo)
    lors, img, g, c, s = K.tor_axis(lcase, axis)
    assert lors.shape[1] > 200
    L, I = cu(lors), cu(img)
    pv = host(ops.tor_projection(L, I, g, c, s, kw, geo, b, s2, layout="cn"))
    ref = O.tor_projection(lors, img, g, c, s, kw, geo, b, s2, mode="f32", contract=True)
    r64 = O.tor_projection(lors, img, g, c, s, kw, geo, b, s2, mode="f64")
    assert np.count_nonzero(ref) > 100
    e, e64 = K.rel_l2(pv, ref), K.rel_l2(pv, r64)
    tol64 = FP64_TOL["tof530_kw4_geo" if geo else "default"]
    record("large_fov_projection", axis=axis, geo=geo, path=tor_path, rel_l2=e, rel_l2_fp64=e64)
    assert e <= TOL and e64 <= tol64, (e, e64)

    v = ref.copy()
    v[::11] = 0.0  # below the 1e-7 threshold: dropped by the reference
    bp = host(ops.tor_backprojection(I, L, cu(v), g, c, s, kw, geo, b, s2, layout="cn"))
    refb = O.tor_backprojection(lors, v, g, c, s, kw, geo, b, s2, mode="f32", contract=True)
    refb64 = O.tor_backprojection(lors, v, g, c, s, kw, geo, b, s2, mode="f64")
    eb, eb64 = K.rel_l2(bp, refb), K.rel_l2(bp, refb64)
    record("large_fov_backprojection", axis=axis, geo=geo, path=tor_path, rel_l2=eb,
           rel_l2_fp64=eb64)
    assert eb <= TOL and eb64 <= tol64, (eb, eb64)

    # the combined call: its projection, then the back-projection of its own values
    pv2, bp2 = ops.tor_projection_backprojection(L, I, g, c, s, kw, geo, b, s2, layout="cn")
    pv2, bp2 = host(pv2), host(bp2)
    refc = O.tor_backprojection(lors, ref, g, c, s, kw, geo, b, s2, mode="f32", contract=True)
    assert K.rel_l2(pv2, ref) <= TOL
    assert K.rel_l2(bp2, refc) <= TOL


@pytest.mark.parametrize("axis", ["x", "y", "z"])
def test_large_fov_map(axis, tor_path):
    from srf_b200.synthetic import random_lors
    lors6 = random_lors(6000, K.LARGE_SCANNER, 13).numpy()
    groups = P.map_process(lors6)
    grid, voxel = (256, 256, 128), 2.5
    size = [gg * voxel for gg in grid]
    lors7 = np.ascontiguousarray(groups[axis].T.astype(np.float32))
    _, g, c, s = P.axis_view(np.zeros(grid, np.float32), [0.0, 0.0, 0.0], size, axis)
    vals = (0.5 + np.random.default_rng(3).random(lors7.shape[1])).astype(np.float32)
    L = cu(lors7)
    got = host(ops.tor_maplors(L, g, c, s, L, cu(vals), K.KW_CONFIG, False, layout="cn"))
    ref = O.tor_maplors(lors7, vals, g, c, s, K.KW_CONFIG, False, mode="f32", contract=True)
    r64 = O.tor_maplors(lors7, vals, g, c, s, K.KW_CONFIG, False, mode="f64")
    assert np.count_nonzero(ref) > 0
    e, e64 = K.rel_l2(got, ref), K.rel_l2(got, r64)
    record("large_fov_map", axis=axis, path=tor_path, rel_l2=e, rel_l2_fp64=e64)
    assert e <= TOL and e64 <= FP64_TOL["default"], (e, e64)


def test_large_fov_against_reference_gpu(lcase):
    if not O.ReferenceGPU.available():
        pytest.skip("reference GPU build not present")
    R = O.ReferenceGPU()
    kw, geo, b, s2 = _params(False)
    for axis in "xyz":
        lors, img, g, c, s = K.tor_axis(lcase, axis)
        L, I = cu(lors), cu(img)
        ref = host(R.tor_projection(L, I, g, c, s, kw, geo, b, s2))
        got = host(ops.tor_projection(L, I, g, c, s, kw, geo, b, s2, layout="cn"))
        e = K.rel_l2(got, ref)
        refb = host(R.tor_backprojection(L, cu(ref), g, c, s, kw, geo, b, s2))
        gotb = host(ops.tor_backprojection(I, L, cu(ref), g, c, s, kw, geo, b, s2, layout="cn"))
        eb = K.rel_l2(gotb, refb)
        record("large_fov_vs_reference_gpu", axis=axis, rel_l2=e, rel_l2_bproj=eb)
        assert e <= TOL and eb <= TOL, (axis, e, eb)


def test_large_fov_chunked_equals_one_pass(lcase):
    """With the scratch budget forcing one 4096-LOR chunk per binning pass (the way a
    16M-event chunk of the full workload is split when its worst-case slab lists exceed
    the budget), every op gives the single-pass result."""
    from srf_b200 import tuning
    kw, geo, b, s2 = _params(False)
    lors = np.concatenate([K.tor_axis(lcase, "x")[0]] * 5, axis=1)
    _, img, g, c, s = K.tor_axis(lcase, "x")
    assert lors.shape[1] > 2 * 4096
    L, I = cu(lors), cu(img)
    M = cu(lors[[0, 1, 2, 3, 4, 5, 9]])  # map records: x1..z2, sigma2 factor

    def run():
        pv, bp = ops.tor_projection_backprojection(L, I, g, c, s, kw, geo, b, s2, layout="cn")
        m = ops.tor_maplors(I, g, c, s, M, pv + 1.0, kw, geo, layout="cn")
        return host(pv), host(bp), host(m)

    one = run()
    try:
        tuning.set_scratch_limit(4 * 4096 * 64)  # one tile of LORs per chunk
        chunked = run()
    finally:
        tuning.set_scratch_limit()
    for a, c_ in zip(one, chunked):
        assert np.count_nonzero(a) > 0
        assert K.rel_l2(c_, a) <= 1e-6


@pytest.mark.parametrize("geo", [False, True])
def test_large_fov_count_samples_match_oracle(lcase, geo):
    """The per-LOR work counts the bench's roofline uses (non-zero-weight voxels, window
    voxels visited) equal the oracle's at this geometry."""
    kw = 4.0 if geo else K.KW_CONFIG
    for axis in "xyz":
        lors, _, g, c, s = K.tor_axis(lcase, axis)
        slots, useful, _ = O.tor_counts(lors, g, c, s, kw, geo)
        got = host(ops.tor_count_samples(cu(lors), g, c, s, kw, geo, layout="cn"))
        assert useful.sum() > 0
        np.testing.assert_array_equal(got[0].astype(np.int64), useful)
        np.testing.assert_array_equal(got[1].astype(np.int64), slots)
