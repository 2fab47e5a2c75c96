"""Reconstruction layer on the GPU: one ReconStep against the oracle's composition of
the reference ops, OSEM subsets, CUDA-graph replay, checkpoint/resume, the efficiency
map, batched frames and the differentiable projector."""

import os

import numpy as np
import pytest
import torch

from oracle import preprocess_ref as P
from oracle import pyoracle as O
from srf_b200 import ops, recon
from srf_b200.data import Image, ListModeData, ListModeDataSplit
from srf_b200.physics import CompleteLoRsModel, SplitLoRsModel
from srf_b200.preprocess import split_listmode
from tests import _cases as K

pytestmark = pytest.mark.gpu


def cu(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def prob():
    case = K.tor_case(n=3000, seed=81, grid=(64, 64, 32), voxel=6.4, n_box=500)
    b, s2 = K.tof_params(530.0)
    model = SplitLoRsModel(K.KW_CONFIG, False, tof_sigma2=s2, tof_bin=b)
    groups = {a: cu(case["groups"][a].astype(np.float32)) for a in "xyz"}
    data = split_listmode(groups)
    rng = np.random.default_rng(3)
    eff = (0.5 + rng.random(case["image"].shape)).astype(np.float32)
    return case, model, data, eff


def oracle_step(case, model, x_np, eff):
    bp = np.zeros(x_np.shape, np.float64)
    for a in "xyz":
        img, g, c, s = P.axis_view(x_np, case["center"], case["size"], a)
        lors = np.ascontiguousarray(case["groups"][a].T.astype(np.float32))
        pv = O.tor_projection(lors, img, g, c, s, model.kernel_width, False, model.tof_bin,
                              model.tof_sigma2)
        b = O.tor_backprojection(lors, pv, g, c, s, model.kernel_width, False, model.tof_bin,
                                 model.tof_sigma2)
        bp += np.transpose(b, model.perm_back(a))
    return x_np * eff * bp.astype(np.float32)


def test_recon_step_matches_oracle(prob):
    case, model, data, eff = prob
    x = Image(cu(case["image"]), case["center"], case["size"])
    e = Image(cu(eff), case["center"], case["size"])
    got = recon.ReconStep(model)(x, e, data).data.cpu().numpy()
    ref = oracle_step(case, model, case["image"], eff)
    assert K.rel_l2(got, ref) < 1e-5


def test_osem_one_subset_is_reference_mlem_and_graph_matches_eager(prob):
    case, model, data, eff = prob
    x0 = Image(cu(case["image"]), case["center"], case["size"])
    e = Image(cu(eff), case["center"], case["size"])
    eager = recon.OSEM(model, data, e, x0, n_subsets=1)
    eager.run(2)
    ref = oracle_step(case, model, oracle_step(case, model, case["image"], eff), eff)
    assert K.rel_l2(eager.x.data.cpu().numpy(), ref) < 2e-5
    for s in (1, 4):
        a = recon.OSEM(model, data, e, x0, n_subsets=s)
        b = recon.OSEM(model, data, e, x0, n_subsets=s, use_graph=True)
        a.run(3)
        b.run(3)
        assert K.rel_l2(b.x.data.cpu().numpy(), a.x.data.cpu().numpy()) < 1e-5


def test_checkpoint_and_resume(prob, tmp_path):
    case, model, data, eff = prob
    x0 = Image(cu(case["image"]), case["center"], case["size"])
    e = Image(cu(eff), case["center"], case["size"])
    prefix = str(tmp_path / "recon")
    o = recon.OSEM(model, data, e, x0, n_subsets=2)
    o.run(2, prefix=prefix)
    assert os.path.exists(prefix + "_0.npy") and os.path.exists(prefix + "_1.npy")
    img, nxt = recon.resume(prefix, case["center"], case["size"], "cuda")
    assert nxt == 2
    np.testing.assert_array_equal(img.data.cpu().numpy(), o.x.data.cpu().numpy())
    # continuing from the checkpoint equals running straight through
    o3 = recon.OSEM(model, data, e, x0, n_subsets=2)
    o3.run(3)
    r = recon.OSEM(model, data, e, img, n_subsets=2)
    r.run(1)
    assert K.rel_l2(r.x.data.cpu().numpy(), o3.x.data.cpu().numpy()) < 1e-5


def test_effmap_pipeline():
    from srf_b200.synthetic import random_lors
    grid, voxel = (64, 64, 32), 6.4
    size = [g * voxel for g in grid]
    b, s2 = K.tof_params(530.0)
    model = SplitLoRsModel(K.KW_CONFIG, False, tof_sigma2=s2, tof_bin=b)
    lors = random_lors(200000, K.SCANNER, 5, device="cuda")
    effinv, total = recon.efficiency_map(model, lors, grid, [0, 0, 0], size,
                                         K.SCANNER.inner_radius, K.SCANNER.axial_length,
                                         chunk=70000)
    e = effinv.data.cpu().numpy()
    assert np.all(np.isfinite(e)) and e.min() >= 0
    keep = P.crop_mask(grid, [0, 0, 0], size, K.SCANNER.inner_radius, K.SCANNER.axial_length)
    assert not e[~keep].any()
    pos = e[e > 0]
    assert abs(pos.min() - 1.0) < 1e-5  # the max of the normalised map inverts to 1
    # the map equals the oracle's merge of the same summed map
    ref = P.merge_effmap(total.cpu().numpy().astype(np.float64), keep)
    assert K.rel_l2(e, ref) < 1e-5


def test_siddon_osem_step_matches_oracle():
    sc = K.siddon_case(n=4000, seed=83, grid=(32, 32, 16), voxel=6.8)
    model = CompleteLoRsModel("m", tof_sigma2=1.0e6, tof_bin=6.0)
    data = ListModeData(cu(sc["events"]), torch.ones(sc["events"].shape[0], device="cuda"))
    x = Image(cu(sc["image"]), sc["center"], sc["size"])
    eff = np.full(sc["image"].shape, 0.8, np.float32)
    got = recon.ReconStep(model)(x, Image(cu(eff), sc["center"], sc["size"]), data)
    kimg = np.ascontiguousarray(np.transpose(sc["image"], (2, 1, 0)))
    pv = O.siddon_projection(sc["lors"], kimg, sc["grid"], sc["center"], sc["size"], 6.0, 1.0e6)
    bp = O.siddon_backprojection(sc["lors"], pv, sc["grid"], sc["center"], sc["size"], 6.0,
                                 1.0e6)
    ref = sc["image"] * eff * np.transpose(bp, (2, 1, 0))
    assert K.rel_l2(got.data.cpu().numpy(), ref) < 1e-5


# ------------------------------------------------------------------------ batched


def _frames(n_frames, seed, grid=(48, 48, 24), voxel=6.4):
    frames = []
    rng = np.random.default_rng(seed)
    for f in range(n_frames):
        n = int(rng.integers(800, 4000))
        ev = np.vstack([K.events(n, 1000 + seed * 100 + f, 530.0),
                        K.box_events(n // 5, 2000 + f)]).astype(np.float32)
        g = P.recon_process(ev, 530.0)
        frames.append({a: cu(g[a].astype(np.float32)) for a in "xyz"})
    size = [g * voxel for g in grid]
    return frames, list(grid), size


@pytest.mark.parametrize("tune", [(1, 0), (1, 16), (2, 0), (3, 0)])
def test_batched_ops_equal_per_frame(tune):
    """Batched ops equal per-frame calls in every kernel family (slab ids run over
    frames x slice ranges x row bands; (1, 16) forces row bands)."""
    from srf_b200 import tuning
    tuning.set_tuning(*tune)
    try:
        frames, grid, size = _frames(5, 1)
        b, s2 = K.tof_params(530.0)
        rng = np.random.default_rng(7)
        imgs = [rng.random(grid, dtype=np.float32) + 0.1 for _ in frames]
        for a in "xyz":
            lors = torch.cat([f[a] for f in frames]).contiguous()
            frame = torch.cat([torch.full((f[a].shape[0],), i, dtype=torch.int32, device="cuda")
                               for i, f in enumerate(frames)])
            perm = SplitLoRsModel.perm(a)
            kimgs = [np.ascontiguousarray(np.transpose(im, perm)) for im in imgs]
            _, g, c, s = P.axis_view(imgs[0], [0, 0, 0], size, a)
            stack = cu(np.stack(kimgs))
            pv = ops.tor_projection_batched(lors, frame, stack, len(frames), g, c, s,
                                            K.KW_CONFIG, False, b, s2, layout="nc")
            ref = torch.cat([ops.tor_projection(f[a], cu(k), g, c, s, K.KW_CONFIG, False, b, s2,
                                                layout="nc") for f, k in zip(frames, kimgs)])
            assert K.rel_l2(pv.cpu().numpy(), ref.cpu().numpy()) < 1e-6
            bp = ops.tor_backprojection_batched(lors, frame, pv, len(frames), g, c, s,
                                                K.KW_CONFIG, False, b, s2, layout="nc")
            off = 0
            for i, f in enumerate(frames):
                n = f[a].shape[0]
                one = ops.tor_backprojection(cu(kimgs[i]), f[a], pv[off:off + n], g, c, s,
                                             K.KW_CONFIG, False, b, s2, layout="nc")
                assert K.rel_l2(bp[i].cpu().numpy(), one.cpu().numpy()) < 1e-6
                off += n
            # the combined batched call gives both results at once
            pv2, bp2 = ops.tor_projection_backprojection_batched(
                lors, frame, stack, len(frames), g, c, s, K.KW_CONFIG, False, b, s2, layout="nc")
            assert K.rel_l2(pv2.cpu().numpy(), pv.cpu().numpy()) < 1e-6
            assert K.rel_l2(bp2.cpu().numpy(), bp.cpu().numpy()) < 1e-6
            # the same through permuted views of the [F, nx, ny, nz] stack (no copies), the
            # back-projection added into a stack that already holds values
            stored = cu(np.stack(imgs))
            sp = [0] + [d + 1 for d in perm]
            back = torch.full_like(stored, 0.5)
            pv3 = ops.tor_projection_backprojection_batched_strided(
                lors, frame, stored.permute(*sp), back.permute(*sp), g, c, s, K.KW_CONFIG,
                False, b, s2, layout="nc")
            assert K.rel_l2(pv3.cpu().numpy(), pv.cpu().numpy()) < 1e-6
            assert K.rel_l2((back.permute(*sp) - 0.5).cpu().numpy(), bp.cpu().numpy()) < 1e-6
    finally:
        tuning.set_tuning()


@pytest.mark.parametrize("use_graph", [False, True])
def test_batched_osem_equals_plain_loop(use_graph):
    from srf_b200.batched import BatchedOSEM
    frames, grid, size = _frames(6, 2)
    b, s2 = K.tof_params(530.0)
    model = SplitLoRsModel(K.KW_CONFIG, False, tof_sigma2=s2, tof_bin=b)
    eff = Image(cu(np.full(grid, 0.9, np.float32)), [0, 0, 0], size)
    x0 = cu(np.ones(grid, np.float32))
    bat = BatchedOSEM(model, frames, eff, x0, n_subsets=3, use_graph=use_graph)
    bat.run(2)
    for f, g in enumerate(frames):
        plain = recon.OSEM(model, split_listmode(g), eff, Image(x0, [0, 0, 0], size), n_subsets=3)
        plain.run(2)
        assert K.rel_l2(bat.x[f].cpu().numpy(), plain.x.data.cpu().numpy()) < 1e-5, f


# ----------------------------------------------------------------------- autograd


@pytest.fixture(scope="module")
def small():
    """32^3 sub-problem with ~20k LORs for the finite-difference checks."""
    grid, voxel = (32, 32, 32), 8.0
    size = [g * voxel for g in grid]
    ev = np.vstack([K.events(16000, 91, 530.0),
                    K.box_events(4000, 92, half=(120.0, 120.0, 120.0))]).astype(np.float32)
    groups = P.recon_process(ev, 530.0)
    b, s2 = K.tof_params(530.0)
    model = SplitLoRsModel(K.KW_CONFIG, False, tof_sigma2=s2, tof_bin=b)
    data = split_listmode({a: cu(groups[a].astype(np.float32)) for a in "xyz"})
    return grid, size, groups, model, data


def test_autograd_adjoint_and_reference_backprojection(small):
    from srf_b200.autograd import Projector
    grid, size, groups, model, data = small
    A = Projector(model, data, grid, [0, 0, 0], size)
    rng = np.random.default_rng(4)
    x = cu(rng.random(grid, dtype=np.float32) + 0.1).requires_grad_(True)
    p = A.forward(x)
    y = {a: torch.rand_like(v) for a, v in p.items()}
    sum(((p[a] * y[a]).sum() for a in p)).backward()
    aty = A.adjoint(y)
    assert K.rel_l2(x.grad.cpu().numpy(), aty.detach().cpu().numpy()) < 1e-6
    # d/dx sum log(Ax) = A^T(1/Ax): the reference's Backprojection with lors_value = A x
    x.grad = None
    p = A.forward(x)
    sum(torch.log(v).sum() for v in p.values()).backward()
    ref = np.zeros(grid, np.float64)
    for a in "xyz":
        img, g, c, s = P.axis_view(x.detach().cpu().numpy(), [0, 0, 0], size, a)
        lors = np.ascontiguousarray(groups[a].T.astype(np.float32))
        pv = O.tor_projection(lors, img, g, c, s, model.kernel_width, False, model.tof_bin,
                              model.tof_sigma2)
        bk = O.tor_backprojection(lors, pv, g, c, s, model.kernel_width, False, model.tof_bin,
                                  model.tof_sigma2)
        ref += np.transpose(bk, model.perm_back(a))
    assert K.rel_l2(x.grad.cpu().numpy(), ref) < 1e-5


def test_autograd_matches_fp64_finite_differences(small):
    """Poisson NLL + quadratic penalty: the autograd gradient (float32 kernels) against
    central differences of the loss evaluated in FP64 with the oracle's f64 projector
    (linearity gives A(x +- eps v) = Ax +- eps Av exactly in double)."""
    from srf_b200.autograd import Projector, poisson_nll, quadratic_penalty
    grid, size, groups, model, data = small
    A = Projector(model, data, grid, [0, 0, 0], size)
    rng = np.random.default_rng(5)
    x_np = (rng.random(grid, dtype=np.float32) + 0.2).astype(np.float32)
    sens_np = (0.5 + rng.random(grid)).astype(np.float32)
    beta = 0.01
    x = cu(x_np).requires_grad_(True)
    sens = cu(sens_np)
    loss = poisson_nll(A.forward(x), x, sens) + quadratic_penalty(x, beta)
    loss.backward()
    grad = x.grad.detach().cpu().numpy().astype(np.float64)

    def proj64(img):
        out = []
        for a in "xyz":
            kimg, g, c, s = P.axis_view(img, [0, 0, 0], size, a)
            lors = np.ascontiguousarray(groups[a].T.astype(np.float32))
            out.append(O.tor_projection(lors, kimg, g, c, s, model.kernel_width, False,
                                        model.tof_bin, model.tof_sigma2, mode="f64"))
        return np.concatenate(out)

    px = proj64(x_np)
    # LORs that touch no voxel have p = 0 for every image: the float loss clamps them to a
    # constant with zero gradient; they carry no information, so the FP64 loss drops them
    support = px > 0

    def loss64(xd, pd):
        d = [np.diff(xd, axis=k) for k in range(3)]
        return (float(np.sum(sens_np.astype(np.float64) * xd))
                - float(np.sum(np.log(pd[support])))
                + 0.5 * beta * sum(float(np.sum(t * t)) for t in d))

    for k in range(4):
        v = rng.standard_normal(grid).astype(np.float32)
        pv = proj64(v)
        eps = 1e-3
        fd = (loss64(x_np + eps * v.astype(np.float64), px + eps * pv)
              - loss64(x_np - eps * v.astype(np.float64), px - eps * pv)) / (2 * eps)
        an = float(np.sum(grad * v))
        assert abs(fd - an) <= 1e-4 * abs(fd), (k, fd, an)


def test_unrolled_osem_checkpointing(small):
    from srf_b200.autograd import Projector, quadratic_penalty, unrolled_osem
    grid, size, groups, model, data = small
    A = Projector(model, data, grid, [0, 0, 0], size)
    eff = cu(np.full(grid, 0.02, np.float32))
    x0 = cu(np.ones(grid, np.float32)).requires_grad_(True)
    outs = []
    for ckpt in (True, False):
        x0.grad = None
        x5 = unrolled_osem(A, x0, eff, n_iterations=5, checkpoint=ckpt)
        l = quadratic_penalty(x5, 0.01) + x5.sum()
        l.backward()
        outs.append((x5.detach().cpu().numpy(), x0.grad.cpu().numpy()))
    assert K.rel_l2(outs[0][0], outs[1][0]) < 1e-6
    # checkpointing recomputes every forward iteration; the back-projections sum with
    # atomics in a run-dependent order, and five iterations of 1/(Ax) amplify that
    # float32 reordering in the gradient to ~4e-5
    assert K.rel_l2(outs[0][1], outs[1][1]) < 2e-4
    # the forward is five reference MLEM iterations
    o = recon.OSEM(model, data, Image(eff, [0, 0, 0], size),
                   Image(cu(np.ones(grid, np.float32)), [0, 0, 0], size))
    o.run(5)
    assert K.rel_l2(outs[0][0], o.x.data.cpu().numpy()) < 1e-5


def test_effmap_from_chunked_source_equals_tensor_input():
    """The effmap pass over an on-device chunk source equals the pass over the same LORs
    held as one tensor."""
    from srf_b200 import SplitLoRsModel
    from srf_b200 import recon
    from srf_b200.synthetic import RandomLorSource
    from tests import _cases as K
    grid, voxel = (32, 32, 16), 6.4
    size = [g * voxel for g in grid]
    model = SplitLoRsModel(K.KW_CONFIG, False)
    src = RandomLorSource(250_000, K.SCANNER, 5, chunk=100_000)
    whole = torch.cat([src(s, min(src.chunk, len(src) - s))
                       for s in range(0, len(src), src.chunk)])
    args = (list(grid), [0, 0, 0], size, K.SCANNER.inner_radius, K.SCANNER.axial_length)
    _, a = recon.efficiency_map(model, src, *args)
    _, b = recon.efficiency_map(model, whole, *args, chunk=100_000)
    assert torch.count_nonzero(b) > 0
    assert float((a - b).norm() / b.norm()) < 1e-6


def test_order_by_direction_permutes_within_blocks_and_keeps_the_reconstruction():
    """Records stay in their 4096-record block, sorted by direction class (up to class
    boundaries, where host and device rounding may differ), and projection + back-projection
    over the reordered groups give the same image."""
    from srf_b200 import SplitLoRsModel
    from srf_b200 import preprocess as PP
    from srf_b200.data import Image
    from srf_b200.physics import backprojection, projection
    ev = K.events(40_000, 17, 530.0).astype(np.float32)
    groups = PP.recon_process(cu(ev), 530.0)
    ordered = PP.order_by_direction(groups)
    for a in "xyz":
        g, o = groups[a].cpu().numpy(), ordered[a].cpu().numpy()
        assert g.shape == o.shape
        for s in range(0, g.shape[0], 4096):
            gb, ob = g[s:s + 4096], o[s:s + 4096]
            np.testing.assert_array_equal(gb[np.lexsort(gb.T[::-1])], ob[np.lexsort(ob.T[::-1])])
            d = ob[:, 3:6].astype(np.float64) - ob[:, 0:3]
            u = d / np.linalg.norm(d, axis=1, keepdims=True)
            q = np.maximum(1 - u[:, 0] ** 2 - u[:, 1] ** 2, 1e-6)
            kx = np.clip(((np.sqrt((1 - u[:, 1] ** 2) / q) - 1) * 16).astype(int), 0, 15)
            ky = np.clip(((np.sqrt((1 - u[:, 0] ** 2) / q) - 1) * 16).astype(int), 0, 15)
            key = kx * 16 + ky
            assert np.mean(np.diff(key) < 0) < 0.01
    grid, voxel = (64, 64, 32), 6.4
    size = [n * voxel for n in grid]
    b, s2 = K.tof_params(530.0)
    model = SplitLoRsModel(K.KW_CONFIG, False, tof_sigma2=s2, tof_bin=b)
    img = Image(torch.rand(grid, device="cuda") + 0.5, [0, 0, 0], size)
    bp = [backprojection(model, projection(model, img, d), img).data
          for d in (PP.split_listmode(groups), PP.split_listmode(ordered))]
    assert torch.count_nonzero(bp[0]) > 0
    assert float((bp[1] - bp[0]).norm() / bp[0].norm()) < 1e-6


def test_order_by_direction_staged_equals_per_record():
    """Records of up to 10 columns are reordered through shared memory, wider ones one
    thread per record; both give the same order (checked bit for bit on the same records,
    contiguous and with a record stride wider than the record)."""
    from srf_b200 import _lib
    ev = K.events(30_000, 23, 530.0).astype(np.float32)
    g = _recon_groups(ev)["x"]
    n = g.shape[0]
    wide = torch.cat([g, torch.arange(2 * n, device="cuda", dtype=torch.float32).view(n, 2)],
                     1).contiguous()  # 12 columns: the per-record kernel
    out_wide = torch.empty_like(wide)
    _lib.call("srf_order_by_direction", wide.data_ptr(), n, 12, 12, out_wide.data_ptr(), None)
    narrow = g.contiguous()
    out_narrow = torch.empty_like(narrow)
    _lib.call("srf_order_by_direction", narrow.data_ptr(), n, 10, 10, out_narrow.data_ptr(),
              None)
    out_strided = torch.zeros_like(wide)  # 10 columns read and written at a 12-float stride
    _lib.call("srf_order_by_direction", wide.data_ptr(), n, 10, 12, out_strided.data_ptr(), None)
    torch.cuda.synchronize()
    assert n > 3 * 4096
    assert torch.equal(out_wide[:, :10], out_narrow)
    assert torch.equal(out_strided[:, :10], out_narrow)
    assert not out_strided[:, 10:].any()  # columns past ncols are left alone
    assert not torch.equal(out_narrow, narrow)  # the order did change


def _recon_groups(ev):
    from srf_b200 import preprocess as PP
    return PP.recon_process(cu(ev), 530.0)


def test_siddon_osem_ordered_equals_unordered():
    """Ray ordering by walk length changes the summation order only."""
    from srf_b200 import CompleteLoRsModel
    from srf_b200.data import Image, ListModeData
    from srf_b200.recon import OSEM
    sc = K.siddon_case(n=30_000, seed=23, grid=(64, 64, 32), voxel=3.4)
    model = CompleteLoRsModel(tof_sigma2=1.0e6, tof_bin=1.0e4)
    lors = cu(np.ascontiguousarray(sc["lors"].T))
    data = ListModeData(lors, torch.ones(lors.shape[0], device="cuda"))
    grid = tuple(sc["grid"])
    x0 = Image(torch.ones(grid, device="cuda"), sc["center"], sc["size"])
    eff = Image(torch.rand(grid, device="cuda") + 0.5, sc["center"], sc["size"])
    out = []
    for order in (False, True):
        o = OSEM(model, data, eff, x0, n_subsets=2, order=order)
        o.step()
        out.append(o.x.data)
    assert float((out[1] - out[0]).norm() / out[0].norm()) < 1e-6


def test_tor_osem_subsets_ordered_equals_unordered():
    """Subsets hold the caller's events k, k+S, ...; ordering inside them changes the
    summation order only."""
    from srf_b200 import SplitLoRsModel
    from srf_b200 import preprocess as PP
    from srf_b200.data import Image
    from srf_b200.recon import OSEM
    grid, voxel = (64, 64, 32), 6.4
    size = [g * voxel for g in grid]
    ev = K.events(30_000, 29, 530.0).astype(np.float32)
    data = PP.split_listmode(PP.recon_process(cu(ev), 530.0))
    b, s2 = K.tof_params(530.0)
    model = SplitLoRsModel(K.KW_CONFIG, False, tof_sigma2=s2, tof_bin=b)
    x0 = Image(torch.ones(grid, device="cuda"), [0, 0, 0], size)
    eff = Image(torch.rand(grid, device="cuda") + 0.5, [0, 0, 0], size)
    out = []
    for order in (False, True):
        o = OSEM(model, data, eff, x0, n_subsets=3, order=order)
        o.step()
        out.append(o.x.data)
    assert float((out[1] - out[0]).norm() / out[0].norm()) < 1e-6


def test_effmap_record_order_changes_only_summation_order():
    """Map records reordered by direction inside each chunk (the default) give the map of
    the records in map_process order, up to float summation order."""
    from srf_b200 import SplitLoRsModel
    from srf_b200 import recon
    from srf_b200.synthetic import random_lors
    from tests import _cases as K
    grid, voxel = (64, 64, 32), 6.4
    size = [g * voxel for g in grid]
    model = SplitLoRsModel(K.KW_CONFIG, False)
    lors = random_lors(300_000, K.SCANNER, 11, device="cuda")
    args = (list(grid), [0, 0, 0], size, K.SCANNER.inner_radius, K.SCANNER.axial_length)
    ea, a = recon.efficiency_map(model, lors, *args, chunk=120_000, order=True)
    eb, b = recon.efficiency_map(model, lors, *args, chunk=120_000, order=False)
    assert torch.count_nonzero(b) > 0
    assert float((a - b).norm() / b.norm()) < 1e-6
    assert float((ea.data - eb.data).norm() / eb.data.norm()) < 1e-5


# ------------------------------------------------------ sharded drivers on one rank


def test_sharded_drivers_on_one_rank_run_the_library_path(prob):
    """With no process group (one rank) the sharded drivers run the library's GPU path
    and equal the single-process drivers: ShardedOSEM = recon.OSEM (eager and graph),
    sharded_efficiency_map = recon.efficiency_map, ShardedBatchedOSEM = BatchedOSEM."""
    from srf_b200 import parallel
    from srf_b200.batched import BatchedOSEM
    from srf_b200.synthetic import RandomLorSource
    case, model, data, eff = prob
    x0 = Image(cu(case["image"]) + 0.5, case["center"], case["size"])
    e = Image(cu(eff), case["center"], case["size"])
    for use_graph in (False, True):
        a = parallel.ShardedOSEM(model, data, e, x0, n_subsets=4, use_graph=use_graph)
        b = recon.OSEM(model, data, e, x0, n_subsets=4)
        a.step(), a.step(), b.step(), b.step()
        assert K.rel_l2(a.x.data.cpu().numpy(), b.x.data.cpu().numpy()) < 1e-6
        a.release()

    grid, voxel = (32, 32, 16), 6.4
    size = [g * voxel for g in grid]
    src = RandomLorSource(250_000, K.SCANNER, 5, chunk=100_000)
    args = (list(grid), [0, 0, 0], size, K.SCANNER.inner_radius, K.SCANNER.axial_length)
    inv_a, tot_a = parallel.sharded_efficiency_map(model, src, *args)
    inv_b, tot_b = recon.efficiency_map(model, src, *args)
    assert torch.count_nonzero(tot_b) > 0
    assert float((tot_a - tot_b).norm() / tot_b.norm()) < 1e-6

    frames, fgrid, fsize = _frames(4, 2)
    feff = Image(cu(np.full(fgrid, 0.9, np.float32)), [0, 0, 0], fsize)
    fx0 = cu(np.ones(fgrid, np.float32))
    sb = parallel.ShardedBatchedOSEM(model, frames, feff, fx0, n_subsets=2)
    bb = BatchedOSEM(model, frames, feff, fx0, n_subsets=2)
    sb.step(), bb.step()
    imgs = sb.images()
    assert sorted(imgs) == list(range(4))
    for f in range(4):
        assert K.rel_l2(imgs[f].cpu().numpy(), bb.x[f].cpu().numpy()) < 1e-6
