"""Generated detector-pair LORs (the effmap source that never materialises its LORs): the
SplitMix64 host mirror against the published first outputs, the random pairs' range and
distinctness, the block-pair enumeration against the scanner's own ring-pair LORs in
the reference's order, and (GPU) the fused map kernels against the same LORs mapped
from memory and against the oracle."""

import numpy as np
import pytest
import torch

from srf_b200.scanner import CylindricalPET, RingScanner
from srf_b200.synthetic import GeneratedPairs, random_pair_indices, splitmix64


def small_pet():
    return CylindricalPET(inner_radius=99.0, outer_radius=119.0, axial_length=33.4,
                          nb_rings=3, nb_blocks_per_ring=8, gap=0.0, block_grid=[1, 4, 1],
                          block_size=[20.0, 40.0, 11.0])


def _splitmix64_stream(seed, n):
    """The generator as published: state += gamma, then the finaliser (Python ints)."""
    m = (1 << 64) - 1
    s, out = seed, []
    for _ in range(n):
        s = (s + 0x9E3779B97F4A7C15) & m
        z = ((s ^ (s >> 30)) * 0xBF58476D1CE4E5B9) & m
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
        out.append(z ^ (z >> 31))
    return out


def test_splitmix64_matches_the_published_stream():
    z = splitmix64(0, np.arange(2, dtype=np.uint64))
    assert [hex(int(v)) for v in z] == ["0xe220a8397b1dcdaf", "0x6e789e6aa1b965f4"]
    for seed in (0, 1, 12345, (1 << 64) - 7):
        got = [int(v) for v in splitmix64(seed, np.arange(64, dtype=np.uint64))]
        assert got == _splitmix64_stream(seed, 64)


def test_random_chords_in_range_uniform_and_grouped():
    nr, nc = 8, 50
    a, b = random_pair_indices(nr, nc, 9, 123, 400_000)
    assert a.min() >= 0 and b.min() >= 0 and a.max() < nr * nc and b.max() < nr * nc
    # chunks are independent of where a call starts
    a2, b2 = random_pair_indices(nr, nc, 9, 123 + 5000, 10)
    np.testing.assert_array_equal(a[5000:5010], a2)
    np.testing.assert_array_equal(b[5000:5010], b2)
    # every ordered pair equally likely: ring pairs and in-ring positions each uniform
    ra, rb, ka, kb = a // nc, b // nc, a % nc, b % nc
    h = np.bincount(ra * nr + rb, minlength=nr * nr)
    assert abs(h.std() / h.mean()) < 0.08
    hk = np.bincount(ka * nc + kb, minlength=nc * nc)
    assert abs(hk.std() / hk.mean()) < 0.25
    # a group of 256 numbers shares its chord class and ring offset
    g0 = (123 // 256 + 1) * 256 - 123
    grp = slice(g0, g0 + 256)
    assert len(np.unique((ka[grp] + kb[grp]) % nc)) == 1
    assert len(np.unique(rb[grp] - ra[grp])) == 1


def test_block_pair_enumeration_matches_the_scanner():
    pet = small_pet()
    src = GeneratedPairs.block_pairs(pet, device="cpu")
    ref = np.vstack([pet.make_ring_pairs_lors(i, j) for i in range(pet.nb_rings)
                     for j in range(pet.nb_rings)]).astype(np.float32)
    assert len(src) == ref.shape[0]
    np.testing.assert_array_equal(src.host_lors(0, len(src)), ref)
    np.testing.assert_array_equal(src.host_lors(777, 100), ref[777:877])


def _oracle_map(model, lors, grid, center, size):
    from oracle import preprocess_ref as P
    from oracle import pyoracle as O
    groups = P.map_process(lors.astype(np.float32))
    total = np.zeros(grid, np.float64)
    img = np.zeros(grid, np.float32)
    for a in model.AXIS:
        rec = np.ascontiguousarray(groups[a].astype(np.float32).T)
        if rec.shape[1] == 0:
            continue
        _, g, c, s = P.axis_view(img, center, size, a)
        m = O.tor_maplors(rec, np.ones(rec.shape[1], np.float32), g, c, s, model.kernel_width,
                          model.geo_sigma2_flag)
        total += np.transpose(m, model.perm_back(a))
    return total


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["random128", "random256band", "random256bands_xy",
                                  "blockpairs"])
def test_fused_map_equals_materialised_and_oracle(case):
    """random256band: the z group's 256 x 256 slices need row bands; random256bands_xy: 16-slice
    slabs force row bands on the x and y groups too, whose map binning then spreads its
    (LOR, slice range) items over the lanes."""
    from srf_b200 import tuning
    if case == "random256bands_xy":
        tuning.set_tuning(1, 16, 0)
    try:
        _fused_map_case(case)
    finally:
        tuning.set_tuning()


def _fused_map_case(case):
    from srf_b200 import SplitLoRsModel, recon
    from tests import _cases as K
    if case == "blockpairs":
        src = GeneratedPairs.block_pairs(small_pet(), chunk=3000)
        grid, voxel = (24, 24, 4), 8.0
    elif case.startswith("random256"):
        src = GeneratedPairs.random(RingScanner(390.0, 600, 320, 3.125), 20_000, 3, chunk=7000)
        grid, voxel = (256, 256, 16), 2.5
    else:
        src = GeneratedPairs.random(K.SCANNER, 40_000, 7, chunk=15_000)
        grid, voxel = (128, 128, 64), 3.2
    size = [g * voxel for g in grid]
    center = [0.0, 0.0, 0.0]
    model = SplitLoRsModel(K.KW_CONFIG, False)
    fused = recon.map_sum(model, src, list(grid), center, size)
    whole = torch.as_tensor(src.host_lors(0, len(src)), device="cuda")
    mem = recon.map_sum(model, whole, list(grid), center, size, chunk=len(src), order=False)
    assert torch.count_nonzero(mem) > 100
    assert float((fused - mem).norm() / mem.norm()) < 1e-6
    from srf_b200.data import Image
    from srf_b200.physics import map_generated
    n_or = min(len(src), 6000)
    ref = _oracle_map(model, src.host_lors(0, n_or), grid, center, size)
    img = Image(torch.zeros(grid, device="cuda"), center, size)
    part = map_generated(model, src, img, 0, n_or).data
    assert K.rel_l2(part.cpu().numpy(), ref) < 1e-5
