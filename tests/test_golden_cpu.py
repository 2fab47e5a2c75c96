"""Golden-vector checks of the oracle (CPU).

* ``test_on_lors_known_answers``: the six hand-written LORs of the reference's own
  test (tests/python/preprocess/test_on_lors.py:12-84) through the numpy restatement.
* The remaining tests compare the oracle with tests/golden/reference_outputs.npz,
  which tests/golden/make_golden.py produced by running the reference's own
  preprocessing code and its own projector sources (compiled for the host).
"""

import os

import numpy as np
import pytest

from oracle import preprocess_ref as P
from oracle import pyoracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_outputs.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN)


def dummy_lors():
    return np.array([
        [-5.0, -5.0, -5.0, 5.0, 5.0, 5.0],
        [-5.0, -5.0, 0.0, 5.0, 5.0, 0.0],
        [0.0, 5.0, 0.0, 0.0, -5.0, 0.0],
        [-5.0, 0.0, 0.0, 5.0, 0.0, 0.0],
        [0.0, -3.0, 5.0, 0.0, 3.0, -5.0],
        [102., 37., -15., 109., -5., -15.],
    ], dtype=np.float32)


def test_on_lors_known_answers():
    lors = dummy_lors()
    # Partition(Axis.x) (test_on_lors.py:51-59)
    np.testing.assert_array_equal(lors[P.dominant_index(lors, "x")], np.array([
        [-5.0, -5.0, -5.0, 5.0, 5.0, 5.0],
        [-5.0, -5.0, 0.0, 5.0, 5.0, 0.0],
        [-5.0, 0.0, 0.0, 5.0, 0.0, 0.0]], np.float32))
    # dominentBy on unit directions (test_on_lors.py:43-49)
    d = np.array([[0, 0, 0, 1, 0, 0], [0, 0, 0, 0, 1, 0], [0, 0, 0, 0, 0, 1]], np.float32)
    assert list(P.dominant_index(d, "z")) == [2]
    # map_process (test_on_lors.py:65-84)
    r = P.map_process(lors)
    np.testing.assert_array_equal(r["x"][:, 0:6], np.array([
        [-5.0, -5.0, -5.0, 5.0, 5.0, 5.0],
        [-5.0, 0.0, -5.0, 5.0, 0.0, 5.0],
        [0.0, 0.0, -5.0, 0.0, 0.0, 5.0]]))
    np.testing.assert_array_equal(r["y"][:, 0:6], np.array([
        [0.0, 0.0, -5.0, 0.0, 0.0, 5.0],
        [109., -15., -5., 102., -15., 37.]]))
    np.testing.assert_array_equal(r["z"][:, 0:6], np.array([[0.0, 3.0, -5.0, 0.0, -3.0, 5.0]]))


def test_recon_process_matches_reference_code(gold):
    r = P.recon_process(gold["tor_events"], float(gold["tor_params"][3]))
    for a in "xyz":
        np.testing.assert_array_equal(r[a].astype(np.float32), gold[f"pre_{a}"])


def test_map_process_matches_reference_code(gold):
    r = P.map_process(gold["map_lors"])
    for a in "xyz":
        np.testing.assert_array_equal(r[a].astype(np.float32), gold[f"map_pre_{a}"])


def _tor_geom(gold, axis):
    img, g, c, s = P.axis_view(gold["tor_image"], gold["center"].tolist(),
                               gold["size"].tolist(), axis)
    return img, g, c, s


@pytest.mark.parametrize("axis", ["x", "y", "z"])
def test_oracle_tor_matches_golden(gold, axis):
    kw, b, s2, _ = [float(v) for v in gold["tor_params"]]
    img, g, c, s = _tor_geom(gold, axis)
    lors = np.ascontiguousarray(gold[f"pre_{axis}"].T)
    pv = O.tor_projection(lors, img, g, c, s, kw, False, b, s2, mode="f32", contract=False)
    np.testing.assert_array_equal(pv, gold[f"tor_proj_{axis}"])
    pvg = O.tor_projection(lors, img, g, c, s, kw, True, b, s2, mode="f32", contract=False)
    np.testing.assert_array_equal(pvg, gold[f"tor_proj_geo_{axis}"])
    bp = O.tor_backprojection(lors, gold[f"tor_bproj_in_{axis}"], g, c, s, kw, False, b, s2,
                              mode="f32", contract=False)
    np.testing.assert_array_equal(bp, gold[f"tor_bproj_{axis}"])
    ml = np.ascontiguousarray(gold[f"map_pre_{axis}"].T)
    mp = O.tor_maplors(ml, np.ones(ml.shape[1], np.float32), g, c, s, kw, False, mode="f32",
                       contract=False)
    np.testing.assert_array_equal(mp, gold[f"tor_map_{axis}"])


def test_oracle_siddon_matches_golden(gold):
    kw, b, s2, _ = [float(v) for v in gold["tor_params"]]
    lors, img = gold["sid_lors"], gold["sid_image"]
    g, c, s = gold["sid_grid"].tolist(), [0.0, 0.0, 0.0], gold["sid_size"].tolist()
    for tag, s2x in (("tof", s2), ("notof", 1.0e6)):
        pv = O.siddon_projection(lors, img, g, c, s, b, s2x, mode="f32", contract=False)
        np.testing.assert_array_equal(pv, gold[f"sid_proj_{tag}"])
        bp = O.siddon_backprojection(lors, pv, g, c, s, b, s2x, mode="f32", contract=False)
        np.testing.assert_array_equal(bp, gold[f"sid_bproj_{tag}"])
    mp = O.siddon_maplors(lors, np.ones(lors.shape[1], np.float32), g, c, s, mode="f32",
                          contract=False)
    np.testing.assert_array_equal(mp, gold["sid_map"])
