"""Pin the oracle to the reference itself (CPU, no GPU needed).

The reference's own projector sources (src/cpp/tf_custom_ops/tor.cu.cc, siddon.cu.cc)
are compiled for the host through oracle/shim (oracle/Makefile, target ref-host). With
contract=0 the oracle's f32 mode rounds exactly as that build does, so the two must
agree BIT FOR BIT on every op. The f64 mode is then checked against f32 at float
accuracy. These tests skip where the reference checkout is absent.
"""

import numpy as np
import pytest

from oracle import pyoracle as O
from tests import _cases as K


@pytest.fixture(scope="module")
def tor_c():
    return K.tor_case(n=1500, seed=11)


@pytest.fixture(scope="module")
def sid_c():
    return K.siddon_case(n=2500, seed=21)


TOR_PARAMS = [
    (K.KW_CONFIG, 530.0, False),
    (4.0, 530.0, True),
    (K.KW_CONFIG, 1.0e4, False),  # the app's default "no TOF" scanner: TOF stays on
]


@pytest.mark.parametrize("kw,tof_res,geo", TOR_PARAMS)
@pytest.mark.parametrize("axis", ["x", "y", "z"])
def test_tor_projection_bit_exact(refhost, tor_c, kw, tof_res, geo, axis):
    b, s2 = K.tof_params(tof_res)
    lors, img, g, c, s = K.tor_axis(tor_c, axis)
    ref = refhost.tor_projection(lors, img, g, c, s, kw, geo, b, s2)
    orc = O.tor_projection(lors, img, g, c, s, kw, geo, b, s2, mode="f32", contract=False)
    assert ref.shape == orc.shape
    assert np.count_nonzero(ref) > 0
    np.testing.assert_array_equal(orc, ref)


@pytest.mark.parametrize("kw,tof_res,geo", TOR_PARAMS)
@pytest.mark.parametrize("axis", ["x", "y", "z"])
def test_tor_backprojection_bit_exact(refhost, tor_c, kw, tof_res, geo, axis):
    b, s2 = K.tof_params(tof_res)
    lors, img, g, c, s = K.tor_axis(tor_c, axis)
    pv = refhost.tor_projection(lors, img, g, c, s, kw, geo, b, s2)
    pv[::7] = 0.0  # exercise the `> 1e-7` threshold
    ref = refhost.tor_backprojection(lors, pv, g, c, s, kw, geo, b, s2)
    orc = O.tor_backprojection(lors, pv, g, c, s, kw, geo, b, s2, mode="f32", contract=False)
    assert np.count_nonzero(ref) > 0
    np.testing.assert_array_equal(orc, ref)


@pytest.mark.parametrize("geo", [False, True])
def test_tor_maplors_bit_exact(refhost, geo):
    mc = K.map_case(n=2000, seed=5)
    for axis in "xyz":
        lors7 = np.ascontiguousarray(mc["groups"][axis].T.astype(np.float32))
        _, g, c, s = (None,) + tuple(K.P.axis_view(np.zeros(mc["grid"], np.float32),
                                                   mc["center"], mc["size"], axis)[1:])
        ones = np.ones(lors7.shape[1], np.float32)
        ref = refhost.tor_maplors(lors7, ones, g, c, s, K.KW_CONFIG, geo)
        orc = O.tor_maplors(lors7, ones, g, c, s, K.KW_CONFIG, geo, mode="f32", contract=False)
        np.testing.assert_array_equal(orc, ref)


@pytest.mark.parametrize("tof_res", [530.0, 1.0e4, 1.0e6])
def test_siddon_projection_bit_exact(refhost, sid_c, tof_res):
    b, s2 = K.tof_params(tof_res)
    if tof_res >= 1.0e6:
        s2 = 1.0e6  # true non-TOF (>= 405758)
    ref = refhost.siddon_projection(sid_c["lors"], sid_c["kimage"], sid_c["grid"],
                                    sid_c["center"], sid_c["size"], b, s2)
    orc = O.siddon_projection(sid_c["lors"], sid_c["kimage"], sid_c["grid"], sid_c["center"],
                              sid_c["size"], b, s2, mode="f32", contract=False)
    assert np.count_nonzero(ref) > 0
    np.testing.assert_array_equal(orc, ref)


@pytest.mark.parametrize("tof_res", [530.0, 1.0e6])
def test_siddon_backprojection_and_map_bit_exact(refhost, sid_c, tof_res):
    b, s2 = K.tof_params(tof_res)
    if tof_res >= 1.0e6:
        s2 = 1.0e6
    args = (sid_c["grid"], sid_c["center"], sid_c["size"])
    pv = refhost.siddon_projection(sid_c["lors"], sid_c["kimage"], *args, b, s2)
    ref = refhost.siddon_backprojection(sid_c["lors"], pv, *args, b, s2)
    orc = O.siddon_backprojection(sid_c["lors"], pv, *args, b, s2, mode="f32", contract=False)
    np.testing.assert_array_equal(orc, ref)
    ones = np.ones(pv.shape, np.float32)
    refm = refhost.siddon_maplors(sid_c["lors"], ones, *args)
    orcm = O.siddon_maplors(sid_c["lors"], ones, *args, mode="f32", contract=False)
    np.testing.assert_array_equal(orcm, refm)


def test_reference_multithreaded_matches_serial(refhost, tor_c):
    """The CPU-baseline harness splits events over threads; results must not change
    beyond float summation order."""
    b, s2 = K.tof_params(530.0)
    lors, img, g, c, s = K.tor_axis(tor_c, "x")
    a = refhost.tor_projection(lors, img, g, c, s, K.KW_CONFIG, False, b, s2, nthreads=1)
    m = refhost.tor_projection(lors, img, g, c, s, K.KW_CONFIG, False, b, s2, nthreads=4)
    np.testing.assert_array_equal(a, m)
    bp1 = refhost.tor_backprojection(lors, a, g, c, s, K.KW_CONFIG, False, b, s2, nthreads=1)
    bp4 = refhost.tor_backprojection(lors, a, g, c, s, K.KW_CONFIG, False, b, s2, nthreads=4)
    assert K.rel_l2(bp4, bp1) < 1e-6


@pytest.mark.parametrize("axis", ["x", "z"])
def test_f64_oracle_close_to_f32(tor_c, axis):
    b, s2 = K.tof_params(530.0)
    lors, img, g, c, s = K.tor_axis(tor_c, axis)
    f32 = O.tor_projection(lors, img, g, c, s, K.KW_CONFIG, False, b, s2, mode="f32")
    f64 = O.tor_projection(lors, img, g, c, s, K.KW_CONFIG, False, b, s2, mode="f64")
    assert K.rel_l2(f32, f64) < 1e-5


def test_siddon_f64_close_to_f32(sid_c):
    b, s2 = K.tof_params(530.0)
    args = (sid_c["grid"], sid_c["center"], sid_c["size"])
    f32 = O.siddon_projection(sid_c["lors"], sid_c["kimage"], *args, b, s2, mode="f32")
    f64 = O.siddon_projection(sid_c["lors"], sid_c["kimage"], *args, b, s2, mode="f64")
    assert K.rel_l2(f32, f64) < 1e-5
