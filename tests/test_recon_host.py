"""Host logic of the OSEM driver (CPU): interleaved subsets of split and complete list-mode
data, and checkpoint files (naming of local_reconstruction.py:50-51, newest-first resume)."""

import numpy as np
import torch

from srf_b200 import recon
from srf_b200.data import Image, ListModeData, ListModeDataSplit


def _lm(n, off):
    lors = torch.arange(n * 10, dtype=torch.float32).reshape(n, 10) + off
    return ListModeData(lors, torch.arange(n, dtype=torch.float32) + off)


def test_subsets_interleave_split_data():
    data = ListModeDataSplit(_lm(7, 0), _lm(5, 1000), _lm(0, 2000))
    subs = recon.make_subsets(data, 3)
    assert len(subs) == 3
    for k, s in enumerate(subs):
        assert isinstance(s, ListModeDataSplit)
        for a in "xyz":
            assert torch.equal(s[a].lors, data[a].lors[k::3])
            assert torch.equal(s[a].values, data[a].values[k::3])
    # every event lands in exactly one subset
    for a in "xyz":
        got = torch.cat([s[a].values for s in subs]).sort().values
        assert torch.equal(got, data[a].values.sort().values)


def test_subsets_complete_data_and_single_subset():
    data = _lm(10, 0)
    subs = recon.make_subsets(data, 4)
    assert [len(s.values) for s in subs] == [3, 3, 2, 2]
    assert torch.equal(subs[1].lors, data.lors[1::4])
    one = recon.make_subsets(data, 1)
    assert len(one) == 1 and one[0].lors is data.lors


def test_checkpoints_and_resume(tmp_path):
    prefix = str(tmp_path / "recon")
    center, size = [0.0, 0.0, 0.0], [8.0, 8.0, 4.0]
    assert recon.latest_checkpoint(prefix) == (None, None)
    assert recon.resume(prefix, center, size, "cpu") == (None, 0)
    for it in (0, 1, 2, 10):
        img = Image(torch.full((4, 4, 2), float(it)), center, size)
        recon.save_checkpoint(prefix, it, img, seed=7)
    # files of another prefix and non-numeric suffixes are ignored
    np.save(str(tmp_path / "recon_final.npy"), np.zeros(3))
    np.save(str(tmp_path / "other_99.npy"), np.zeros(3))
    it, path = recon.latest_checkpoint(prefix)
    assert it == 10 and path.endswith("recon_10.npy")
    meta = np.load(str(tmp_path / "recon_10.meta.npz"))
    assert int(meta["iteration"]) == 10 and int(meta["seed"]) == 7
    np.testing.assert_array_equal(meta["size"], size)
    img, nxt = recon.resume(prefix, center, size, "cpu")
    assert nxt == 11 and float(img.data.mean()) == 10.0
    assert list(img.data.shape) == [4, 4, 2]
