"""GPU parity of the CUDA projectors against the oracle and the reference's outputs.

Tolerance: relative L2 error <= 1e-5 in float32 (projection values per LOR, or the
back-projected image). The oracle's f32 mode with contract=1 reproduces the
reference's device arithmetic; its f64 mode is the exact-arithmetic statement of the
same operator. Set SRF_PARITY_LOG=<file> to append each measured error as JSON.
"""

import json
import math
import os

import numpy as np
import pytest
import torch

from oracle import preprocess_ref as P
from oracle import pyoracle as O
from srf_b200 import ops
from tests import _cases as K

pytestmark = pytest.mark.gpu
TOL = 1e-5  # against the reference's float arithmetic (oracle f32 mode / reference kernels)
# Against the FP64 oracle (the same discrete operator with exact arithmetic) the bound is
# the reference's own float error, measured on the CPU between the oracle's f32 and f64
# modes: <= 6e-6 for the primary TOR configuration; a narrow tube (kernel_width 4 with
# the geometric sigma factor, sigma^2 down to ~0.1 mm^2) loses ~1e-4 to the float
# cancellation in d^2 = |delta|^2 - (delta.u)^2 that the reference computes; the
# Siddon float walk accumulates next-boundary error (~1e-5 on back-projected images).
FP64_TOL = {"default": 1e-5, "tof530_kw4_geo": 3e-4, "siddon_image": 3e-5}
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_outputs.npz")


def record(name, **vals):
    path = os.environ.get("SRF_PARITY_LOG")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(dict(test=name, **vals)) + "\n")


def cu(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy()


TOR_PARAMS = {
    "tof530_kw10": (K.KW_CONFIG, 530.0, False),
    "tof530_kw4_geo": (4.0, 530.0, True),
    "tofdefault": (K.KW_CONFIG, 1.0e4, False),
    "notof": (K.KW_CONFIG, None, False),
}


def _tp(name):
    kw, res, geo = TOR_PARAMS[name]
    if res is None:
        b, s2 = K.tof_params(530.0)
        return kw, geo, b, 1.0e6
    b, s2 = K.tof_params(res)
    return kw, geo, b, s2


@pytest.fixture(scope="module")
def tcase():
    # The timed workload's geometry (128x128x64 at 3.2 mm), fewer events.
    return K.tor_case(n=3000, seed=31, grid=(128, 128, 64), voxel=3.2, n_box=600)


# Tuning of the TOR kernels, (path, slices per slab): shared-memory slabs with a lane per
# (LOR, slab) segment (1, the default), the same with 16 slices per slab, which splits
# every slice into bands of rows, slabs with a segment's slices spread over lanes (3), and
# LOR-centric kernels reading the image from L2 with global atomics (2, the fallback when
# nothing fits in shared memory).
TOR_PATHS = {"slab": (1, 0), "slab_grid2": (1, 0, 2), "slab_bands": (1, 16),
             "slab_spread": (3, 0), "global": (2, 0)}


@pytest.fixture(params=list(TOR_PATHS))
def tor_path(request):
    """Every TOR kernel family must agree with the oracle."""
    from srf_b200 import tuning
    tuning.set_tuning(*TOR_PATHS[request.param])
    yield request.param
    tuning.set_tuning()


@pytest.mark.parametrize("pname", list(TOR_PARAMS))
@pytest.mark.parametrize("axis", ["x", "y", "z"])
def test_tor_projection(tcase, pname, axis, tor_path):
    kw, geo, b, s2 = _tp(pname)
    lors, img, g, c, s = K.tor_axis(tcase, axis)
    gpu = host(ops.tor_projection(cu(lors), cu(img), g, c, s, kw, geo, b, s2, layout="cn"))
    f32 = O.tor_projection(lors, img, g, c, s, kw, geo, b, s2, mode="f32", contract=True)
    f64 = O.tor_projection(lors, img, g, c, s, kw, geo, b, s2, mode="f64")
    e32, e64 = K.rel_l2(gpu, f32), K.rel_l2(gpu, f64)
    record("tor_projection", params=pname, axis=axis, n=int(lors.shape[1]), rel_l2_f32=e32,
           rel_l2_f64=e64)
    assert np.count_nonzero(f32) > 0
    assert e32 <= TOL and e64 <= TOL, (e32, e64)
    # row-major [N,10] input gives the same result (up to float summation order: the
    # slab path adds per-slab partial sums atomically)
    gpu_nc = host(ops.tor_projection(cu(lors.T), cu(img), g, c, s, kw, geo, b, s2,
                                     layout="nc"))
    assert K.rel_l2(gpu_nc, gpu) <= 1e-6


@pytest.fixture(params=list(TOR_PATHS))
def scatter_kernel(request):
    """Back-projection / map / adjoint in every TOR kernel family against the oracle."""
    from srf_b200 import tuning
    tuning.set_tuning(*TOR_PATHS[request.param])
    yield request.param
    tuning.set_tuning()


@pytest.mark.parametrize("pname", ["tof530_kw10", "tof530_kw4_geo", "notof"])
@pytest.mark.parametrize("axis", ["x", "y", "z"])
def test_tor_backprojection(tcase, pname, axis, scatter_kernel):
    kw, geo, b, s2 = _tp(pname)
    lors, img, g, c, s = K.tor_axis(tcase, axis)
    pv = O.tor_projection(lors, img, g, c, s, kw, geo, b, s2, mode="f32")
    pv[::9] = 0.0  # LORs at or below the 1e-7 threshold contribute nothing
    pv[1::9] = 5e-8
    gpu = host(ops.tor_backprojection(cu(img), cu(lors), cu(pv), g, c, s, kw, geo, b, s2,
                                      layout="cn"))
    f32 = O.tor_backprojection(lors, pv, g, c, s, kw, geo, b, s2, mode="f32", contract=True)
    f64 = O.tor_backprojection(lors, pv, g, c, s, kw, geo, b, s2, mode="f64")
    e32, e64 = K.rel_l2(gpu, f32), K.rel_l2(gpu, f64)
    record("tor_backprojection", params=pname, axis=axis, rel_l2_f32=e32, rel_l2_f64=e64)
    assert np.count_nonzero(f32) > 0
    assert e32 <= TOL and e64 <= FP64_TOL.get(pname, FP64_TOL["default"]), (e32, e64)


@pytest.mark.parametrize("geo", [False, True])
def test_tor_maplors(geo, scatter_kernel):
    mc = K.map_case(n=4000, seed=7, grid=(128, 128, 64), voxel=3.2)
    for axis in "xyz":
        lors7 = np.ascontiguousarray(mc["groups"][axis].T.astype(np.float32))
        _, g, c, s = P.axis_view(np.zeros(mc["grid"], np.float32), mc["center"], mc["size"],
                                 axis)
        vals = (0.5 + np.random.default_rng(3).random(lors7.shape[1])).astype(np.float32)
        gpu = host(ops.tor_maplors(cu(np.zeros((g[2], g[1], g[0]), np.float32)), g, c, s,
                                   cu(lors7), cu(vals), K.KW_CONFIG, geo, layout="cn"))
        f32 = O.tor_maplors(lors7, vals, g, c, s, K.KW_CONFIG, geo, mode="f32", contract=True)
        f64 = O.tor_maplors(lors7, vals, g, c, s, K.KW_CONFIG, geo, mode="f64")
        e32, e64 = K.rel_l2(gpu, f32), K.rel_l2(gpu, f64)
        record("tor_maplors", geo=geo, axis=axis, rel_l2_f32=e32, rel_l2_f64=e64)
        assert e32 <= TOL and e64 <= TOL, (axis, e32, e64)


@pytest.mark.parametrize("pname", ["tof530_kw10", "notof"])
def test_tor_adjoint_identity(tcase, pname, scatter_kernel):
    """<A x, y> = <x, A^T y> for the plain adjoint, evaluated in float64 sums."""
    kw, geo, b, s2 = _tp(pname)
    rng = np.random.default_rng(17)
    for axis in "xyz":
        lors, img, g, c, s = K.tor_axis(tcase, axis)
        x = rng.random(img.shape, dtype=np.float32)
        y = rng.random(lors.shape[1], dtype=np.float32)
        ax = host(ops.tor_projection(cu(lors), cu(x), g, c, s, kw, geo, b, s2, layout="cn"))
        aty = host(ops.tor_backproject_adjoint(cu(y), cu(lors), g, c, s, kw, geo, b, s2,
                                               layout="cn"))
        lhs = float(np.dot(ax.astype(np.float64), y))
        rhs = float(np.dot(x.ravel().astype(np.float64), aty.ravel()))
        err = abs(lhs - rhs) / abs(lhs)
        record("tor_adjoint", params=pname, axis=axis, rel_err=err)
        assert err < 1e-5, (axis, lhs, rhs)


def test_tor_backprojection_equals_adjoint_of_reciprocal(tcase):
    """The reference's Backprojection is A^T(1/v) over v > 1e-7 (tor.cu.cc:203-205)."""
    kw, geo, b, s2 = _tp("tof530_kw10")
    lors, img, g, c, s = K.tor_axis(tcase, "y")
    pv = O.tor_projection(lors, img, g, c, s, kw, geo, b, s2, mode="f32")
    bp = host(ops.tor_backprojection(cu(img), cu(lors), cu(pv), g, c, s, kw, geo, b, s2,
                                     layout="cn"))
    inv = np.where(pv > 1e-7, 1.0 / np.maximum(pv, 1e-30), 0.0).astype(np.float32)
    adj = host(ops.tor_backproject_adjoint(cu(inv), cu(lors), g, c, s, kw, geo, b, s2,
                                           layout="cn"))
    assert K.rel_l2(bp, adj) < 1e-6


# -------------------------------------------------------------------------- Siddon


@pytest.fixture(scope="module")
def scase():
    sc = K.siddon_case(n=6000, seed=41, grid=(64, 64, 32), voxel=3.4)
    box = K.box_events(1500, 42, half=(180.0, 180.0, 90.0))
    sc["lors"] = np.ascontiguousarray(np.vstack([sc["events"], box]).T)
    return sc


SID_PARAMS = {"tof530": 530.0, "tofdefault": 1.0e4, "notof": None}


@pytest.fixture(params=[0, 1], ids=["quad", "scalar"])
def sid_path(request):
    """The Siddon kernel family: scatter ops reduce quads of voxels, or one per voxel."""
    from srf_b200 import tuning
    tuning.set_siddon_tuning(request.param)
    yield request.param
    tuning.set_siddon_tuning(0)


def _sp(name):
    b, s2 = K.tof_params(530.0 if SID_PARAMS[name] is None else SID_PARAMS[name])
    return b, (1.0e6 if SID_PARAMS[name] is None else s2)


@pytest.mark.parametrize("pname", list(SID_PARAMS))
def test_siddon_projection_backprojection(scase, pname, sid_path):
    b, s2 = _sp(pname)
    args = (scase["grid"], scase["center"], scase["size"])
    lors, img = scase["lors"], scase["kimage"]
    gpu = host(ops.siddon_projection(cu(lors), cu(img), *args, b, s2, layout="cn"))
    f32, bad = O.siddon_projection(lors, img, *args, b, s2, mode="f32", contract=True,
                                   return_bad=True)
    f64 = O.siddon_projection(lors, img, *args, b, s2, mode="f64")
    e32, e64 = K.rel_l2(gpu, f32), K.rel_l2(gpu, f64)
    record("siddon_projection", params=pname, rel_l2_f32=e32, rel_l2_f64=e64, bad=int(bad))
    assert e32 <= TOL and e64 <= TOL, (e32, e64)
    pv = f32.copy()
    pv[::11] = 0.0
    gb = host(ops.siddon_backprojection(cu(img), cu(lors), cu(pv), *args, b, s2, layout="cn"))
    b32 = O.siddon_backprojection(lors, pv, *args, b, s2, mode="f32", contract=True)
    b64 = O.siddon_backprojection(lors, pv, *args, b, s2, mode="f64")
    e32, e64 = K.rel_l2(gb, b32), K.rel_l2(gb, b64)
    record("siddon_backprojection", params=pname, rel_l2_f32=e32, rel_l2_f64=e64)
    assert e32 <= TOL and e64 <= FP64_TOL["siddon_image"], (e32, e64)


def test_siddon_maplors_and_adjoint(scase, sid_path):
    args = (scase["grid"], scase["center"], scase["size"])
    lors = scase["lors"]
    vals = (0.5 + np.random.default_rng(5).random(lors.shape[1])).astype(np.float32)
    gm = host(ops.siddon_maplors(cu(np.zeros(1, np.float32)), *args, cu(lors), cu(vals),
                                 layout="cn"))
    m32 = O.siddon_maplors(lors, vals, *args, mode="f32", contract=True)
    m64 = O.siddon_maplors(lors, vals, *args, mode="f64")
    record("siddon_maplors", rel_l2_f32=K.rel_l2(gm, m32), rel_l2_f64=K.rel_l2(gm, m64))
    assert K.rel_l2(gm, m32) <= TOL and K.rel_l2(gm, m64) <= FP64_TOL["siddon_image"]
    b, s2 = _sp("tof530")
    rng = np.random.default_rng(9)
    x = rng.random(scase["kimage"].shape, dtype=np.float32)
    y = rng.random(lors.shape[1], dtype=np.float32)
    ax = host(ops.siddon_projection(cu(lors), cu(x), *args, b, s2, layout="cn"))
    aty = host(ops.siddon_backproject_adjoint(cu(y), cu(lors), *args, b, s2, layout="cn"))
    lhs = float(np.dot(ax.astype(np.float64), y))
    rhs = float(np.dot(x.ravel().astype(np.float64), aty.ravel()))
    assert abs(lhs - rhs) / abs(lhs) < 1e-5


# --------------------------------------------------------------- preprocessing


def test_recon_process_gpu_bit_exact(tcase):
    from srf_b200 import preprocess as PP
    ev = tcase["events"]
    got = PP.recon_process(cu(ev), tcase["tof_res"])
    for a in "xyz":
        np.testing.assert_array_equal(host(got[a]), tcase["groups"][a].astype(np.float32))


def test_map_process_gpu_bit_exact():
    from srf_b200 import preprocess as PP
    mc = K.map_case(n=5000, seed=8)
    got = PP.map_process(cu(mc["lors"]))
    for a in "xyz":
        np.testing.assert_array_equal(host(got[a]), mc["groups"][a].astype(np.float32))


def test_preprocess_many_tiles():
    """More events than one 4096-event tile, TOF off (no cut), so the stable scatter's
    cross-tile offsets are exercised."""
    from srf_b200 import preprocess as PP
    ev = np.vstack([K.events(9000, 77, 1.0e4), K.box_events(3000, 78)]).astype(np.float32)
    ref = P.recon_process(ev, 1.0e4)
    got = PP.recon_process(cu(ev), 1.0e4)
    for a in "xyz":
        np.testing.assert_array_equal(host(got[a]), ref[a].astype(np.float32))


# ------------------------------------------------------------------- golden vectors


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN)


def test_golden_preprocessing_gpu(gold):
    from srf_b200 import preprocess as PP
    got = PP.recon_process(cu(gold["tor_events"]), float(gold["tor_params"][3]))
    for a in "xyz":
        np.testing.assert_array_equal(host(got[a]), gold[f"pre_{a}"])
    gm = PP.map_process(cu(gold["map_lors"]))
    for a in "xyz":
        np.testing.assert_array_equal(host(gm[a]), gold[f"map_pre_{a}"])


@pytest.mark.parametrize("axis", ["x", "y", "z"])
def test_golden_tor_gpu(gold, axis, tor_path):
    kw, b, s2, _ = [float(v) for v in gold["tor_params"]]
    img, g, c, s = P.axis_view(gold["tor_image"], gold["center"].tolist(), gold["size"].tolist(),
                               axis)
    lors = cu(gold[f"pre_{axis}"])
    pv = host(ops.tor_projection(lors, cu(img), g, c, s, kw, False, b, s2, layout="nc"))
    assert K.rel_l2(pv, gold[f"tor_proj_{axis}"]) <= TOL
    pvg = host(ops.tor_projection(lors, cu(img), g, c, s, kw, True, b, s2, layout="nc"))
    assert K.rel_l2(pvg, gold[f"tor_proj_geo_{axis}"]) <= TOL
    bp = host(ops.tor_backprojection(cu(img), lors, cu(gold[f"tor_bproj_in_{axis}"]), g, c, s,
                                     kw, False, b, s2, layout="nc"))
    assert K.rel_l2(bp, gold[f"tor_bproj_{axis}"]) <= TOL
    ml = cu(gold[f"map_pre_{axis}"])
    mp = host(ops.tor_maplors(cu(img), g, c, s, ml, cu(np.ones(ml.shape[0], np.float32)), kw,
                              False, layout="nc"))
    assert K.rel_l2(mp, gold[f"tor_map_{axis}"]) <= TOL


def test_golden_siddon_gpu(gold):
    kw, b, s2, _ = [float(v) for v in gold["tor_params"]]
    lors, img = cu(gold["sid_lors"]), cu(gold["sid_image"])
    g, c, s = gold["sid_grid"].tolist(), [0.0, 0.0, 0.0], gold["sid_size"].tolist()
    for tag, s2x in (("tof", s2), ("notof", 1.0e6)):
        pv = host(ops.siddon_projection(lors, img, g, c, s, b, s2x, layout="cn"))
        assert K.rel_l2(pv, gold[f"sid_proj_{tag}"]) <= TOL
        bp = host(ops.siddon_backprojection(img, lors, cu(gold[f"sid_proj_{tag}"]), g, c, s, b,
                                            s2x, layout="cn"))
        assert K.rel_l2(bp, gold[f"sid_bproj_{tag}"]) <= TOL
    mp = host(ops.siddon_maplors(img, g, c, s, lors, cu(np.ones(lors.shape[1], np.float32)),
                                 layout="cn"))
    assert K.rel_l2(mp, gold["sid_map"]) <= TOL


# --------------------------------------------------------------------- edge cases


def test_empty_inputs():
    g, c, s = [16, 16, 8], [0.0, 0.0, 0.0], [51.2, 51.2, 25.6]
    img = cu(np.ones((8, 16, 16), np.float32))
    e10 = torch.zeros((10, 0), device="cuda")
    assert ops.tor_projection(e10, img, g, c, s, 4.0, layout="cn").numel() == 0
    bp = host(ops.tor_backprojection(img, e10, torch.zeros(0, device="cuda"), g, c, s, 4.0,
                                     layout="cn"))
    assert bp.shape == (8, 16, 16) and not bp.any()
    pv, bp = ops.tor_projection_backprojection(e10, img, g, c, s, 4.0, layout="cn")
    assert pv.numel() == 0 and not host(bp).any()
    e7 = torch.zeros((7, 0), device="cuda")
    assert ops.siddon_projection(e7, img, g, c, s, layout="cn").numel() == 0


def test_degenerate_lors_give_zero_not_nan():
    g, c, s = [16, 16, 8], [0.0, 0.0, 0.0], [51.2, 51.2, 25.6]
    img = cu(np.ones((8, 16, 16), np.float32))
    rows = np.array([
        [0, 0, -50, 0, 0, -50, 0, 0, 0, 1],      # zero length
        [300, 300, -50, 310, 300, 50, 0, 0, 0, 1],  # misses the FOV
        [np.nan, 0, -50, 0, 0, 50, 0, 0, 0, 1],  # NaN endpoint
        [1, 2, -50, 3, -2, 50, 2, 0, 0, 0.5],    # ordinary
    ], np.float32)
    pv = host(ops.tor_projection(cu(rows), img, g, c, s, 4.0, False, 6.0, 1139.77, layout="nc"))
    assert np.all(np.isfinite(pv)) and pv[0] == 0 and pv[1] == 0 and pv[2] == 0 and pv[3] > 0
    sid = np.array([[0, 0, 0, 0, 0, 0, 0], [300, 300, 0, 310, 300, 1, 0],
                    [np.nan, 0, 0, 1, 1, 1, 0], [-100, 3, 1, 100, -2, -1, 5]], np.float32)
    sp = host(ops.siddon_projection(cu(sid), img, g, c, s, 6.0, 1139.77, layout="nc"))
    assert np.all(np.isfinite(sp)) and sp[:3].tolist() == [0, 0, 0] and sp[3] > 0


def test_accumulate_adds(tcase):
    kw, geo, b, s2 = _tp("tof530_kw10")
    lors, img, g, c, s = K.tor_axis(tcase, "x")
    pv = O.tor_projection(lors, img, g, c, s, kw, geo, b, s2, mode="f32")
    once = ops.tor_backprojection(cu(img), cu(lors), cu(pv), g, c, s, kw, geo, b, s2,
                                  layout="cn")
    out = once.clone()
    ops.tor_backprojection(cu(img), cu(lors), cu(pv), g, c, s, kw, geo, b, s2, layout="cn",
                           out=out, accumulate=True)
    assert K.rel_l2(host(out), 2 * host(once)) < 1e-6


def test_wider_records_and_strides(tcase):
    """[N,C] records with extra trailing columns use the event stride."""
    kw, geo, b, s2 = _tp("tof530_kw10")
    lors, img, g, c, s = K.tor_axis(tcase, "y")
    wide = np.hstack([lors.T, np.full((lors.shape[1], 3), 7.0, np.float32)])
    a = host(ops.tor_projection(cu(lors), cu(img), g, c, s, kw, geo, b, s2, layout="cn"))
    w = host(ops.tor_projection(cu(wide), cu(img), g, c, s, kw, geo, b, s2, layout="nc"))
    assert K.rel_l2(w, a) <= 1e-6


def test_cpu_tensors_are_rejected():
    with pytest.raises(TypeError):
        ops.tor_projection(torch.zeros(10, 4), torch.zeros(8, 16, 16), [16, 16, 8], [0, 0, 0],
                           [1, 1, 1], 4.0)


def test_tor_maplors_zero_divisor_matches_reference(scatter_kernel):
    """Maplors divides without a threshold (tor.cu.cc:239): a zero divisor puts inf on
    voxels with non-zero weight and NaN (0/0) on the other visited voxels."""
    mc = K.map_case(n=600, seed=12, grid=(64, 64, 32), voxel=6.4)
    lors7 = np.ascontiguousarray(mc["groups"]["x"].T.astype(np.float32))
    _, g, c, s = P.axis_view(np.zeros(mc["grid"], np.float32), mc["center"], mc["size"], "x")
    vals = np.ones(lors7.shape[1], np.float32)
    hits = O.tor_counts(np.ascontiguousarray(lors7), g, c, s, K.KW_CONFIG)[1]
    vals[int(np.argmax(hits))] = 0.0  # a LOR that does cross the image
    gpu = host(ops.tor_maplors(cu(np.zeros((g[2], g[1], g[0]), np.float32)), g, c, s,
                               cu(lors7), cu(vals), K.KW_CONFIG, False, layout="cn"))
    ref = O.tor_maplors(lors7, vals, g, c, s, K.KW_CONFIG, False, mode="f32", contract=True)
    np.testing.assert_array_equal(np.isnan(gpu), np.isnan(ref))
    np.testing.assert_array_equal(np.isinf(gpu), np.isinf(ref))
    fin = np.isfinite(ref)
    assert np.isnan(ref).any() and np.isinf(ref).any()
    assert K.rel_l2(gpu[fin], ref[fin]) <= TOL


def test_slab_chunks_equal_one_pass():
    """With the scratch budget forcing one 4096-LOR chunk at a time, every slab op gives
    the single-pass result (projection values, images)."""
    from srf_b200 import tuning
    big = K.tor_case(n=40000, seed=91, grid=(128, 128, 64), voxel=3.2, n_box=4000)
    kw, geo, b, s2 = _tp("tof530_kw10")
    lors, img, g, c, s = K.tor_axis(big, "x")
    assert lors.shape[1] > 3 * 4096
    L, I = cu(lors), cu(img)
    vals = cu(np.random.default_rng(3).random(lors.shape[1], dtype=np.float32) + 0.5)

    def run():
        pv = host(ops.tor_projection(L, I, g, c, s, kw, geo, b, s2, layout="cn"))
        bp = host(ops.tor_backprojection(I, L, vals, g, c, s, kw, geo, b, s2, layout="cn"))
        adj = host(ops.tor_backproject_adjoint(vals, L, g, c, s, kw, geo, b, s2, layout="cn"))
        L7 = torch.cat([L[:6], L[9:10]]).contiguous()  # x1..z2, sigma2_factor
        mp = host(ops.tor_maplors(I, g, c, s, L7, vals, kw, geo, layout="cn"))
        return pv, bp, adj, mp

    tuning.set_tuning(path=1)
    try:
        one = run()
        tuning.set_scratch_limit(1)
        try:
            chunked = run()
        finally:
            tuning.set_scratch_limit(0)
    finally:
        tuning.set_tuning()
    for a, b_ in zip(one, chunked):
        assert np.count_nonzero(a) > 0
        assert K.rel_l2(b_, a) <= 1e-6


@pytest.mark.parametrize("pname", ["tof530_kw10", "tof530_kw4_geo", "notof"])
@pytest.mark.parametrize("axis", ["x", "y", "z"])
def test_tor_projection_backprojection_combined(tcase, pname, axis, tor_path):
    """The combined call gives the separate calls' projection values and back-projected
    image in every kernel family, and both match the oracle."""
    kw, geo, b, s2 = _tp(pname)
    lors, img, g, c, s = K.tor_axis(tcase, axis)
    L, I = cu(lors), cu(img)
    pv_t, bp_t = ops.tor_projection_backprojection(L, I, g, c, s, kw, geo, b, s2, layout="cn")
    pv, bp = host(pv_t), host(bp_t)
    pv_sep = ops.tor_projection(L, I, g, c, s, kw, geo, b, s2, layout="cn")
    bp_sep = host(ops.tor_backprojection(I, L, pv_sep, g, c, s, kw, geo, b, s2, layout="cn"))
    assert K.rel_l2(pv, host(pv_sep)) <= 1e-6
    assert K.rel_l2(bp, bp_sep) <= 1e-6
    f32 = O.tor_projection(lors, img, g, c, s, kw, geo, b, s2, mode="f32", contract=True)
    back = O.tor_backprojection(lors, f32, g, c, s, kw, geo, b, s2, mode="f32", contract=True)
    e_p, e_b = K.rel_l2(pv, f32), K.rel_l2(bp, back)
    record("tor_projection_backprojection", params=pname, axis=axis, rel_l2_proj=e_p,
           rel_l2_back=e_b)
    assert np.count_nonzero(back) > 0
    assert e_p <= TOL and e_b <= TOL, (e_p, e_b)
    # accumulate adds onto the given image; the image must not be overwritten in place
    acc = cu(np.full(img.shape, 2.0, np.float32))
    ops.tor_projection_backprojection(L, I, g, c, s, kw, geo, b, s2, layout="cn", out=acc,
                                      accumulate=True)
    assert K.rel_l2(host(acc), bp + 2.0) <= 1e-6
    with pytest.raises(ValueError):
        ops.tor_projection_backprojection(L, I, g, c, s, kw, geo, b, s2, layout="cn", out=I)


def test_tor_projection_backprojection_chunked():
    """With one 4096-LOR chunk at a time the combined call still equals one pass."""
    from srf_b200 import tuning
    big = K.tor_case(n=40000, seed=91, grid=(128, 128, 64), voxel=3.2, n_box=4000)
    kw, geo, b, s2 = _tp("tof530_kw10")
    lors, img, g, c, s = K.tor_axis(big, "x")
    L, I = cu(lors), cu(img)
    tuning.set_tuning(path=1)
    try:
        one = [host(t) for t in ops.tor_projection_backprojection(L, I, g, c, s, kw, geo, b, s2,
                                                                  layout="cn")]
        tuning.set_scratch_limit(1)
        try:
            chunked = [host(t) for t in ops.tor_projection_backprojection(
                L, I, g, c, s, kw, geo, b, s2, layout="cn")]
        finally:
            tuning.set_scratch_limit(0)
    finally:
        tuning.set_tuning()
    for a, b_ in zip(one, chunked):
        assert np.count_nonzero(a) > 0
        assert K.rel_l2(b_, a) <= 1e-6


@pytest.mark.parametrize("pname", ["tof530_kw10", "tof530_kw4_geo"])
def test_tor_count_samples_match_oracle(tcase, pname):
    """Per-LOR TOR work (non-zero-weight voxels, in-grid window voxels: the numerator of
    the bench's roofline) equals the oracle's count for every axis group."""
    kw, geo, _, _ = _tp(pname)
    for axis in "xyz":
        lors, _, g, c, s = K.tor_axis(tcase, axis)
        slots, useful, _ = O.tor_counts(lors, g, c, s, kw, geo)
        got = host(ops.tor_count_samples(cu(lors), g, c, s, kw, geo, layout="cn"))
        assert useful.sum() > 0
        np.testing.assert_array_equal(got[0].astype(np.int64), useful)
        np.testing.assert_array_equal(got[1].astype(np.int64), slots)


def test_siddon_count_samples_match_oracle():
    """Per-ray voxel visits of the Siddon walk equal the oracle's count (rays that miss
    the image, or start off the grid, visit none)."""
    sc = K.siddon_case(n=20000, seed=67, grid=(64, 64, 32), voxel=3.4)
    args = (sc["grid"], sc["center"], sc["size"])
    visits, _ = O.siddon_counts(sc["lors"], *args)
    got = host(ops.siddon_count_samples(cu(sc["lors"]), *args, layout="cn"))
    assert visits.sum() > 0
    np.testing.assert_array_equal(got.astype(np.int64), visits)


# kernel widths whose window edge P = ceil((sqrt(2) kw + voxel_z) / voxel_x) covers every
# specialised slab / LOR-centric kernel (P = 2..8) and the generic kernel (P > 8), at 3.2 mm
KW_FOR_PATCH = {2: 2.0, 3: 4.0, 4: 6.0, 5: 8.0, 6: K.KW_CONFIG, 7: 12.5, 8: 15.0, 10: 20.0}


@pytest.fixture(scope="module")
def pcase():
    return K.tor_case(n=4000, seed=37, grid=(96, 96, 48), voxel=3.2, n_box=800)


@pytest.mark.parametrize("patch", list(KW_FOR_PATCH))
def test_tor_every_window_size(pcase, patch, scatter_kernel):
    """Projection and back-projection against the oracle for every window size."""
    kw = KW_FOR_PATCH[patch]
    assert math.ceil((math.sqrt(2) * np.float32(kw) + 3.2) / 3.2) == patch
    b, s2 = K.tof_params(530.0)
    for axis in "xz":
        lors, img, g, c, s = K.tor_axis(pcase, axis)
        pv = host(ops.tor_projection(cu(lors), cu(img), g, c, s, kw, False, b, s2, layout="cn"))
        ref = O.tor_projection(lors, img, g, c, s, kw, False, b, s2, mode="f32", contract=True)
        assert np.count_nonzero(ref) > 0
        assert K.rel_l2(pv, ref) <= TOL, (axis, "projection")
        bp = host(ops.tor_backprojection(cu(img), cu(lors), cu(ref), g, c, s, kw, False, b, s2,
                                         layout="cn"))
        refb = O.tor_backprojection(lors, ref, g, c, s, kw, False, b, s2, mode="f32",
                                    contract=True)
        assert K.rel_l2(bp, refb) <= TOL, (axis, "back-projection")
