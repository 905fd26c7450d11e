"""The allocation-free DS-candidate extraction, checked against the workspace variant.

mr_ds_extract_noalloc serves callers that cannot give the library device workspace
memory; it keeps its scratch in a fixed array compiled into the library. This file is
named to be collected last, so a run that stops at its first failure has already run
every other test.
"""
import re
from pathlib import Path

import numpy as np
import pytest
import torch

from moraine_b200 import _dev, _lib

pytestmark = pytest.mark.gpu

HEADER = Path(__file__).resolve().parents[1] / "include" / "moraine_b200.h"


def _limit() -> int:
    """MR_DS_EXTRACT_NOALLOC_MAX_PIXELS as the header defines it."""
    m = re.search(r"#define MR_DS_EXTRACT_NOALLOC_MAX_PIXELS \((\d+)LL \* (\d+)LL\)", HEADER.read_text())
    assert m, "limit macro not found in the header"
    return int(m.group(1)) * int(m.group(2))


def _raster(shape, win, seed, device):
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    nl, w = shape
    is_shp = (torch.rand((nl, w, win), generator=g, device=device) < 0.3).to(torch.uint8)
    shp_num = is_shp.sum(-1, dtype=torch.int32)
    return shp_num.contiguous(), is_shp.contiguous()


def _extract(noalloc, shp_num, is_shp, min_shp):
    nl, w, win = is_shp.shape
    dev = is_shp.device
    idx = torch.full((nl * w, 2), -1, dtype=torch.int32, device=dev)
    pc = torch.zeros((nl * w, win), dtype=torch.uint8, device=dev)
    n = torch.zeros((1,), dtype=torch.int64, device=dev)
    lib = _lib.load()
    if noalloc:
        rc = lib.mr_ds_extract_noalloc(shp_num.data_ptr(), is_shp.data_ptr(), nl, w, win, min_shp, idx.data_ptr(),
                                       pc.data_ptr(), nl * w, n.data_ptr(), _dev.stream())
    else:
        ws = _dev.workspace(lib.mr_ds_extract_workspace_bytes(nl * w), dev)
        rc = lib.mr_ds_extract(shp_num.data_ptr(), is_shp.data_ptr(), nl, w, win, min_shp, idx.data_ptr(),
                               pc.data_ptr(), nl * w, n.data_ptr(), ws.data_ptr(), ws.numel(), _dev.stream())
    _lib.check(rc, "extract")
    k = int(n.item())
    return k, idx[:k].cpu().numpy(), pc[:k].cpu().numpy()


def test_noalloc_matches_workspace_variant_twice(cuda):
    # two calls in a row, the second on a smaller raster: the shared array keeps the first
    # call's counts, which must not leak into the second result
    for shape, win, seed, min_shp in [((700, 900), 35, 1, 12), ((123, 77), 121, 2, 40)]:
        shp_num, is_shp = _raster(shape, win, seed, cuda)
        k_ref, idx_ref, pc_ref = _extract(False, shp_num, is_shp, min_shp)
        k, idx, pc = _extract(True, shp_num, is_shp, min_shp)
        assert k == k_ref and k > 0
        np.testing.assert_array_equal(idx, idx_ref)
        np.testing.assert_array_equal(pc, pc_ref)


def test_noalloc_at_the_limit(cuda):
    # a raster of exactly the limit fills the whole array and is accepted
    limit = _limit()
    nl = 4096
    w = limit // nl
    assert nl * w == limit
    shp_num, is_shp = _raster((nl, w), 5, 3, cuda)
    k_ref, idx_ref, pc_ref = _extract(False, shp_num, is_shp, 2)
    k, idx, pc = _extract(True, shp_num, is_shp, 2)
    assert k == k_ref and k > 0
    np.testing.assert_array_equal(idx, idx_ref)
    np.testing.assert_array_equal(pc, pc_ref)


def test_noalloc_rejects_oversize_raster(cuda):
    lib = _lib.load()
    limit = _limit()
    nl, w = 4097, limit // 4096  # one row more than the limit
    assert nl * w > limit
    rc = lib.mr_ds_extract_noalloc(16, None, nl, w, 9, 3, 16, None, 100, 16, None)
    assert rc == _lib.MR_ERR_UNSUPPORTED
    assert "limit" in _lib.last_error()
