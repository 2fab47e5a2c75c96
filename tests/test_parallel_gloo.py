"""Sharded MLEM on two CPU ranks (gloo): the all-reduced update equals the
single-process update over all events. The projector here is the oracle (the test's
checker running on CPU); the sharding, the master sum and the update are the product's
``srf_b200.parallel`` code."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import preprocess_ref as P
from oracle import pyoracle as O
from srf_b200.data import Image, ListModeData, ListModeDataSplit
from srf_b200.parallel import ShardedMLEM, shard, shard_range
from srf_b200.physics import SplitLoRsModel


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def oracle_projection(model, image, data):
    out = {}
    for a in model.AXIS:
        img, g, c, s = P.axis_view(image.data.numpy(), image.center, image.size, a)
        lors = np.ascontiguousarray(data[a].lors.numpy().T)
        v = O.tor_projection(lors, img, g, c, s, model.kernel_width, model.geo_sigma2_flag,
                             model.tof_bin, model.tof_sigma2) if lors.shape[1] else np.zeros(0)
        out[a] = ListModeData(data[a].lors, torch.as_tensor(v, dtype=torch.float32))
    return ListModeDataSplit(out["x"], out["y"], out["z"])


def oracle_backprojection(model, data, image):
    total = np.zeros(image.data.shape, np.float64)
    for a in model.AXIS:
        _, g, c, s = P.axis_view(image.data.numpy(), image.center, image.size, a)
        lors = np.ascontiguousarray(data[a].lors.numpy().T)
        if lors.shape[1] == 0:
            continue
        b = O.tor_backprojection(lors, data[a].values.numpy(), g, c, s, model.kernel_width,
                                 model.geo_sigma2_flag, model.tof_bin, model.tof_sigma2)
        total += np.transpose(b, model.perm_back(a))
    return Image(torch.as_tensor(total.astype(np.float32)), image.center, image.size)


def _problem():
    from tests import _cases as K
    case = K.tor_case(n=600, seed=71, grid=(32, 32, 16), voxel=12.8, n_box=200)
    b, s2 = K.tof_params(530.0)
    model = SplitLoRsModel(K.KW_CONFIG, False, tof_sigma2=s2, tof_bin=b)
    data = ListModeDataSplit(*[
        ListModeData(torch.as_tensor(case["groups"][a].astype(np.float32)),
                     torch.ones(case["groups"][a].shape[0])) for a in "xyz"])
    x0 = Image(torch.as_tensor(case["image"]), case["center"], case["size"])
    effinv = Image(torch.full(case["image"].shape, 0.7), case["center"], case["size"])
    return model, data, effinv, x0


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        model, data, effinv, x0 = _problem()
        m = ShardedMLEM(model, shard(data, rank, world), effinv, x0,
                        project=oracle_projection, backproject=oracle_backprojection)
        m.step()
        x = m.step()
        q.put((rank, x.data.numpy()))
    finally:
        dist.destroy_process_group()


def test_shard_ranges_cover_everything():
    for n in (0, 1, 7, 100):
        for w in (1, 2, 3, 8):
            got = []
            for r in range(w):
                a, b = shard_range(n, r, w)
                got.extend(range(a, b))
            assert got == list(range(n))


def test_sharded_mlem_two_ranks_equals_single_process():
    model, data, effinv, x0 = _problem()
    single = ShardedMLEM(model, data, effinv, x0, project=oracle_projection,
                         backproject=oracle_backprojection)
    single.step()
    ref = single.step().data.numpy()

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        r, x = q.get(timeout=300)
        out[r] = x
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(2):
        num = np.linalg.norm(out[r] - ref)
        assert num / np.linalg.norm(ref) < 1e-6, r
    np.testing.assert_array_equal(out[0], out[1])  # every rank holds the same image


# ------------------------------------------------------------- sharded OSEM, effmap, frames


def oracle_project_back(model, image, data):
    proj = oracle_projection(model, image, data)
    return proj, oracle_backprojection(model, proj, image)


def cpu_update(x, effinv, bp):
    x.mul_(effinv * bp)


def _osem_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from srf_b200.parallel import ShardedOSEM
        model, data, effinv, x0 = _problem()
        m = ShardedOSEM(model, data, effinv, x0, n_subsets=3,
                        project_back=oracle_project_back, update=cpu_update)
        m.step()
        q.put((rank, m.step().data.numpy()))
    finally:
        dist.destroy_process_group()


def _spawn(target, world=2):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        r, x = q.get(timeout=300)
        out[r] = x
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return out


def test_subset_shards_partition_the_subsets():
    """Over the ranks, the parts of subset k are exactly recon.make_subsets' subset k."""
    from srf_b200.parallel import subset_shard
    from srf_b200.recon import make_subsets
    for n in (0, 1, 5, 17, 64):
        data = ListModeData(torch.arange(n, dtype=torch.float32)[:, None].repeat(1, 3),
                            torch.arange(n, dtype=torch.float32))
        for S in (1, 2, 3, 4):
            full = make_subsets(data, S)
            for W in (1, 2, 3):
                for k in range(S):
                    got = torch.cat([subset_shard(data, k, S, r, W).values for r in range(W)])
                    assert torch.equal(torch.sort(got).values, full[k].values), (n, S, W, k)


def test_sharded_osem_two_ranks_equals_single_process():
    from srf_b200.parallel import ShardedOSEM
    model, data, effinv, x0 = _problem()
    single = ShardedOSEM(model, data, effinv, x0, n_subsets=3,
                         project_back=oracle_project_back, update=cpu_update)
    single.step()
    ref = single.step().data.numpy()
    out = _spawn(_osem_worker)
    for r in range(2):
        assert np.linalg.norm(out[r] - ref) / np.linalg.norm(ref) < 1e-6, r
    np.testing.assert_array_equal(out[0], out[1])


class _PairSource:
    """A small chunked detector-pair source on the CPU (the random_lors generator)."""
    chunk = 250
    device = torch.device("cpu")

    def __len__(self):
        return 1100

    def __call__(self, start, count):
        from srf_b200.scanner import RingScanner
        from srf_b200.synthetic import random_lors
        return random_lors(count, RingScanner(400.0, 400, 32, 3.2), 11 + start // self.chunk)


def oracle_map_chunk(model, part, img):
    """Maplors of one chunk by the oracle: numpy map_process, then tor_maplors per axis."""
    groups = P.map_process(part.numpy().astype(np.float32))
    total = np.zeros(img.data.shape, np.float64)
    for a in model.AXIS:
        lors = np.ascontiguousarray(groups[a].astype(np.float32).T)
        if lors.shape[1] == 0:
            continue
        _, g, c, s = P.axis_view(img.data.numpy(), img.center, img.size, a)
        m = O.tor_maplors(lors, np.ones(lors.shape[1], np.float32), g, c, s,
                          model.kernel_width, model.geo_sigma2_flag)
        total += np.transpose(m, model.perm_back(a))
    return torch.as_tensor(total.astype(np.float32))


_MAP_GEOM = ((16, 16, 8), [0.0, 0.0, 0.0], [409.6, 409.6, 204.8])


def _map_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from srf_b200.parallel import sharded_efficiency_map
        model, _, _, _ = _problem()
        grid, center, size = _MAP_GEOM
        inv, total = sharded_efficiency_map(model, _PairSource(), grid, center, size, 400.0,
                                            102.4, map_chunk=oracle_map_chunk)
        q.put((rank, (inv.data.numpy(), total.numpy())))
    finally:
        dist.destroy_process_group()


def test_sharded_efficiency_map_two_ranks_equals_single_process():
    from srf_b200.recon import map_sum
    from srf_b200.preprocess import crop_mask, merge_effmap
    model, _, _, _ = _problem()
    grid, center, size = _MAP_GEOM
    ref = map_sum(model, _PairSource(), grid, center, size, map_chunk=oracle_map_chunk)
    assert float(ref.sum()) > 0
    ref_inv = merge_effmap(ref, crop_mask(grid, center, size, 400.0, 102.4, device="cpu"))
    out = _spawn(_map_worker)
    for r in range(2):
        inv, total = out[r]
        assert np.linalg.norm(total - ref.numpy()) / np.linalg.norm(ref.numpy()) < 1e-6
        assert np.linalg.norm(inv - ref_inv.numpy()) / np.linalg.norm(ref_inv.numpy()) < 1e-5
    np.testing.assert_array_equal(out[0][1], out[1][1])


def test_shard_frames_cover_every_frame_once():
    from srf_b200.parallel import shard_frames
    for n in (0, 1, 7, 64):
        for w in (1, 2, 3, 8):
            got = sorted(f for r in range(w) for f in shard_frames(n, r, w))
            assert got == list(range(n))
