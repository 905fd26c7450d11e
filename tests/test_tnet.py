"""Temporal network helpers against the reference notebook's printed outputs (nbs/API/tnet.ipynb)."""
import numpy as np
import pytest

from moraine_b200.tnet import TempNet, nimage_from_npair


def test_from_bandwidth():  # tnet.ipynb cells 11-12
    np.testing.assert_array_equal(TempNet.from_bandwidth(5, 2).image_pairs,
                                  [[0, 1], [0, 2], [1, 2], [1, 3], [2, 3], [2, 4], [3, 4]])
    full = TempNet.from_bandwidth(17).image_pairs
    r, s = np.triu_indices(17, 1)
    np.testing.assert_array_equal(full, np.stack((r, s), -1))
    assert full.dtype == np.int32


def test_image_pairs_idx():  # tnet.ipynb cells 14-16
    t = TempNet(np.stack(([0, 1, 2, 3], [1, 2, 3, 4]), axis=-1))
    np.testing.assert_array_equal(t.image_pairs, [[0, 1], [1, 2], [2, 3], [3, 4]])
    assert t.image_pairs_idx(ref=1, sec=2) == 1
    np.testing.assert_array_equal(t.image_pairs_idx(ref=[1, 2], sec=[2, 3]), [1, 2])
    np.testing.assert_array_equal(t.image_pairs_idx(ref=[0, 0], sec=[1, 2]), [0, -1])


def test_validation():
    with pytest.raises(ValueError, match="not sorted"):
        TempNet(np.array([[1, 2], [0, 1]]))
    with pytest.raises(ValueError, match="not directed"):
        TempNet(np.array([[0, 1], [1, 1]]))
    with pytest.raises(ValueError, match="not connected"):
        TempNet(np.array([[0, 2], [1, 2]]))


def test_nimage_from_npair():  # tnet.ipynb cell 18
    assert nimage_from_npair(6) == 4
    for n in (2, 17, 50, 100, 200):
        assert nimage_from_npair(n * (n - 1) // 2) == n
    with pytest.raises(ValueError):
        nimage_from_npair(7)
