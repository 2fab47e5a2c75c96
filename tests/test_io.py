"""List-mode files: .npy round trip, chunking, h5 without h5py (CPU), and streaming onto
the GPU in chunks equal to a one-shot upload (GPU)."""

import numpy as np
import pytest
import torch

from srf_b200 import io


def _events(n, seed=5):
    return np.random.default_rng(seed).normal(0, 100, (n, 7)).astype(np.float32)


def test_npy_round_trip(tmp_path):
    ev = _events(1000)
    p = tmp_path / "ev.npy"
    io.save_listmode(p, ev)
    got = io.load_listmode(p)
    assert got.dtype == np.float32 and got.shape == (1000, 7)
    np.testing.assert_array_equal(np.asarray(got), ev)


def test_bad_files(tmp_path):
    p = tmp_path / "bad.npy"
    np.save(p, np.zeros((5, 3), np.float32))
    with pytest.raises(ValueError):
        io.load_listmode(p)
    with pytest.raises(ValueError):
        io.load_listmode(tmp_path / "ev.txt")


def test_h5_needs_h5py(tmp_path):
    try:
        import h5py  # noqa: F401
    except ImportError:
        with pytest.raises(ImportError, match="h5py"):
            io.load_listmode(tmp_path / "ev.h5")
    else:
        ev = _events(100)
        io.save_listmode(tmp_path / "ev.h5", ev)
        np.testing.assert_array_equal(io.load_listmode(tmp_path / "ev.h5"), ev)


def test_chunk_bounds_cover_rows():
    for n, c in [(0, 4), (1, 4), (10, 3), (12, 4)]:
        b = io.chunk_bounds(n, c)
        assert [i for s, e in b for i in range(s, e)] == list(range(n))
        assert all(e - s <= c for s, e in b)


@pytest.mark.gpu
def test_stream_events_equals_one_upload(tmp_path):
    ev = _events(250_003)
    p = tmp_path / "ev.npy"
    io.save_listmode(p, ev)
    chunks = [c.clone() for c in io.stream_events(p, chunk=60_000)]
    assert len(chunks) == 5
    torch.testing.assert_close(torch.cat(chunks).cpu(), torch.from_numpy(ev), rtol=0, atol=0)


@pytest.mark.gpu
def test_stream_events_chunk_survives_one_advance():
    # a caller that pairs neighbouring chunks holds chunk k (uncloned) while it works on
    # chunk k+1; both must still hold their own source rows
    ev = _events(70_001, seed=9)
    prev, prev_rows = None, None
    bounds = io.chunk_bounds(ev.shape[0], 10_000)
    for k, c in enumerate(io.stream_events(ev, chunk=10_000)):
        s, e = bounds[k]
        c.mul_(1.0)  # caller work on chunk k, queued on the current stream
        if prev is not None:
            np.testing.assert_array_equal(prev.cpu().numpy(), prev_rows)
        np.testing.assert_array_equal(c.cpu().numpy(), ev[s:e])
        prev, prev_rows = c, ev[s:e]
    assert k == len(bounds) - 1


@pytest.mark.gpu
def test_load_split_equals_recon_process(tmp_path):
    from srf_b200 import preprocess as PP
    from tests import _cases as K
    ev = K.events(30_000, 11, 530.0).astype(np.float32)
    p = tmp_path / "ev.npy"
    io.save_listmode(p, ev)
    got = io.load_split(p, 530.0, chunk=7_000)["projection_data"]
    ref = PP.recon_process(torch.as_tensor(ev).cuda(), 530.0)
    for a in "xyz":
        # the same rows; chunking orders each group chunk by chunk
        g, r = got[a].lors.cpu().numpy(), ref[a].cpu().numpy()
        assert g.shape == r.shape
        np.testing.assert_array_equal(g[np.lexsort(g.T[::-1])], r[np.lexsort(r.T[::-1])])
        assert torch.all(got[a].values == 1)
