"""Scanner geometry against the reference's own known answers
(tests/python/scanner/test_scanner.py:17-100 and tests/python/scanner/test_block.py:1-70 of
SRF): first-block centre of the mCT ring, block-pair order, a rotated block's crystal mesh,
and the LOR between two opposite one-crystal blocks."""

import math

import numpy as np

from srf_b200.scanner import CylindricalPET


def _mct():
    # mCT ring and block parameters of test_scanner.py:19-41
    return CylindricalPET(inner_radius=424.5, outer_radius=444.5, axial_length=220.0,
                          nb_rings=4, nb_blocks_per_ring=48, gap=4.0, block_grid=[1, 13, 13],
                          block_size=[20.0, 52.0, 52.0], tof_res=530, tof_bin=40, name="mCT")


def test_first_block_centre():
    sc = _mct()
    z = -(4.0 + 52.0) * (4 - 1) / 2  # test_scanner.py:56-59
    x = (424.5 + 444.5) / 2
    m = sc.block_meshes(0, 0)
    assert m.shape == (13 * 13, 3)
    np.testing.assert_allclose(m.mean(0), [x, 0.0, z], atol=1e-9)


def test_block_pair_order():
    # test_scanner.py:82-98 with rings [1, 2, 3]: blocks 1..3
    diff = [[i + 1, j + 1] for i, j in CylindricalPET.block_pairs(3, same_ring=False)]
    assert diff == [[1, 2], [1, 3], [2, 1], [2, 3], [3, 1], [3, 2]]
    same = [[i + 1, j + 1] for i, j in CylindricalPET.block_pairs(3, same_ring=True)]
    assert same == [[1, 2], [1, 3], [2, 3]]


def test_rotated_block_mesh():
    # test_block.py:14-20, 40-44: a one-crystal block centred at (1, 0, 0) rotated by pi/4
    sc = CylindricalPET(inner_radius=0.0, outer_radius=2.0, axial_length=1.0, nb_rings=1,
                        nb_blocks_per_ring=8, gap=0.0, block_grid=[1, 1, 1],
                        block_size=[6.0, 2.0, 1.0])
    np.testing.assert_allclose(sc.block_meshes(0, 1), [[math.sqrt(2) / 2, math.sqrt(2) / 2, 0.0]],
                               atol=1e-12)


def test_opposite_blocks_lor():
    # test_block.py:56-69: blocks at angles 0 and pi -> the LOR (1,0,0)-(-1,0,0)
    sc = CylindricalPET(inner_radius=0.0, outer_radius=2.0, axial_length=1.0, nb_rings=1,
                        nb_blocks_per_ring=2, gap=0.0, block_grid=[1, 1, 1],
                        block_size=[6.0, 2.0, 1.0])
    np.testing.assert_allclose(sc.make_ring_pairs_lors(0, 0), [[1.0, 0, 0, -1.0, 0, 0]],
                               atol=1e-12)


def test_tof_info_known_answers():
    """tof_info restates _get_tof_info (src/python/srf/api/app/srfapp_new.py:244-251): the
    3-sigma limit res * 0.15 / 2.35482005 * 3 mm, sigma^2 = limit^2 / 9, bin * 0.15 mm. The
    workloads' figures: 530 ps FWHM -> sigma 33.76 mm (sigma^2 1139.774), 400 ps -> 25.48 mm
    (649.213), 40 ps bins -> 6 mm."""
    import math
    from srf_b200.scanner import tof_info
    b, s2 = tof_info(530.0, 40.0)
    assert b == 6.0
    assert abs(s2 - 1139.7741617120942) < 1e-9
    assert abs(math.sqrt(s2) - 33.76) < 5e-3
    b, s2 = tof_info(400.0, 40.0)
    assert b == 6.0
    assert abs(s2 - 649.2127656601461) < 1e-9
    assert abs(math.sqrt(s2) - 25.48) < 5e-3
    # the same operations, in the reference's order
    limit = 530.0 * 0.15 / 2.35482005 * 3
    assert tof_info(530.0, 40.0)[1] == (limit ** 2) / 9
