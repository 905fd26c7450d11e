"""Raster <-> point cloud (moraine.pc.ras2pc / pc2ras) and DS candidates on the device,
against numpy's own indexing (the reference's code is that indexing) and the oracle."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _gix(rng, nl, w, n, negative=False):
    cells = rng.choice(nl * w, size=n, replace=False)
    g = np.stack([cells // w, cells % w], -1).astype(np.int64)
    if negative:  # numpy counts negative indices from the end
        g[::3, 0] -= nl
        g[1::4, 1] -= w
    return g


@pytest.mark.parametrize("dtype,rec", [(np.float32, ()), (np.complex64, (17,)), (np.bool_, (5, 7)),
                                       (np.int16, (3,)), (np.float64, (5,)), (np.complex128, (2, 3)),
                                       (np.uint8, (13,))])
def test_ras2pc_matches_numpy(cuda, dtype, rec):
    from moraine_b200.pc import ras2pc
    rng = np.random.default_rng(1)
    nl, w = 37, 23
    ras = (rng.standard_normal((nl, w, *rec)) * 50).astype(dtype)
    if np.dtype(dtype).kind == "c":
        ras = (ras + 1j * rng.standard_normal(ras.shape)).astype(dtype)
    g = _gix(rng, nl, w, 300, negative=True)
    ref = ras[g[:, 0], g[:, 1]]
    got = ras2pc(ras, g)
    assert got.dtype == ref.dtype and got.shape == ref.shape
    np.testing.assert_array_equal(got.view(np.uint8), ref.view(np.uint8))
    t = ras2pc(torch.from_numpy(ras).to(cuda), torch.from_numpy(g.astype(np.int32)).to(cuda))
    assert t.is_cuda
    np.testing.assert_array_equal(t.cpu().numpy().view(np.uint8), ref.view(np.uint8))
    assert ras2pc(ras, g[:0]).shape == (0, *rec)


def test_ras2pc_errors(cuda):
    from moraine_b200.pc import ras2pc
    ras = np.zeros((10, 8, 3), np.float32)
    for bad in ([[10, 0]], [[0, 8]], [[-11, 0]], [[0, -9]]):
        with pytest.raises(IndexError):
            ras2pc(ras, np.array(bad))
    with pytest.raises(IndexError):
        ras2pc(ras, np.array([[0.0, 1.0]]))
    with pytest.raises(NotImplementedError):
        ras2pc(ras, np.array([1, 2, 3]))
    # the library still works after a rejected index
    np.testing.assert_array_equal(ras2pc(ras, np.array([[9, 7]])), ras[[9], [7]])


@pytest.mark.parametrize("dtype,rec", [(np.float32, ()), (np.complex64, (11,)), (np.float64, (4,)),
                                       (np.complex128, (2,))])
def test_pc2ras_matches_numpy(cuda, dtype, rec):
    from moraine_b200.pc import pc2ras
    rng = np.random.default_rng(2)
    nl, w = 29, 31
    g = _gix(rng, nl, w, 200)
    pc = rng.standard_normal((200, *rec)).astype(dtype)
    ref = np.empty((nl, w, *rec), dtype=dtype)  # moraine/pc.py:223-236
    ref[:] = np.nan
    ref[g[:, 0], g[:, 1]] = pc
    got = pc2ras(g, pc, (nl, w))
    assert got.dtype == ref.dtype and got.shape == ref.shape
    np.testing.assert_array_equal(got.view(np.uint8), ref.view(np.uint8))  # NaN + 0j fill included


def test_pc2ras_errors(cuda):
    from moraine_b200.pc import pc2ras
    with pytest.raises(ValueError):
        pc2ras(np.array([[0, 0]]), np.array([3], np.int32), (2, 2))  # NaN does not fit an integer raster
    with pytest.raises(IndexError):
        pc2ras(np.array([[2, 0]]), np.array([3.0], np.float32), (2, 2))
    with pytest.raises(ValueError):
        pc2ras(np.array([[0, 0], [1, 1]]), np.array([3.0], np.float32), (2, 2))


@pytest.mark.parametrize("min_shp", [1, 50, 200])
def test_ds_candidates_match_notebook_glue(cuda, min_shp):
    """nbs/API/pl.ipynb cell 15: is_ds_can = shp_num >= min_shp; idx = where; pc_is_shp = is_shp[is_ds_can]."""
    from moraine_b200.pc import ds_candidates
    rng = np.random.default_rng(3)
    nl, w, az, r = 41, 53, 7, 9
    is_shp = rng.random((nl, w, az, r)) < 0.8
    shp_num = np.count_nonzero(is_shp, axis=(-2, -1)).astype(np.int32)
    idx, pc = ds_candidates(shp_num, is_shp, min_shp)
    is_ds = shp_num >= min_shp
    np.testing.assert_array_equal(idx, np.stack(np.where(is_ds), -1).astype(np.int32))
    np.testing.assert_array_equal(pc, is_shp[is_ds])
    o_idx, o_pc = O.ds_candidates(is_shp, shp_num, min_shp)
    np.testing.assert_array_equal(idx, o_idx)
    np.testing.assert_array_equal(pc, o_pc)
    idx2, none = ds_candidates(torch.from_numpy(shp_num).to(cuda), None, min_shp)
    assert none is None and torch.equal(idx2.cpu(), torch.from_numpy(idx))
