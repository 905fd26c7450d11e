"""SHP identification: drop-in ``ks_test`` and ``select_shp`` on the GPU.

Same signatures, defaults and output layouts as ``moraine.shp`` (moraine/shp.py:269-323).
"""
from __future__ import annotations

import torch

from . import _dev, _lib

__all__ = ["ks_test", "select_shp"]


def ks_test(rmli, az_half_win: int, r_half_win: int, block_size: int = 128, return_dist: bool = False):
    """Two-sample Kolmogorov-Smirnov test of every pixel against its window.

    ``rmli`` (nlines, width, nimages) float32. Returns ``p`` (nlines, width, az_win, r_win),
    or ``(dist, p)`` with ``return_dist``. ``p`` and ``dist`` equal the reference CPU path
    (moraine/shp.py:20-113) bit for bit; NaN outside the image and where either pixel
    holds a NaN. ``block_size`` is accepted for compatibility and ignored (the launch
    shape is planned from the image count and window).
    """
    kind = _dev.kind_of(rmli)
    in_dtype = rmli.dtype
    dev = _dev.require_cuda()
    x = _dev.to_device(rmli, torch.float32, dev)
    if x.ndim != 3:
        raise ValueError(f"ks_test: rmli must be 3-D (nlines, width, nimages), got shape {tuple(x.shape)}")
    nlines, width, nimages = x.shape
    az_win, r_win = 2 * az_half_win + 1, 2 * r_half_win + 1
    p = torch.empty((nlines, width, az_win, r_win), dtype=torch.float32, device=dev)
    dist = torch.empty_like(p) if return_dist else None
    lib = _lib.load()
    ws = _dev.workspace(lib.mr_ks_workspace_bytes(nlines, width, nimages), dev)
    _lib.call("mr_ks_test", x.data_ptr(), nlines, width, nimages, az_half_win, r_half_win, p.data_ptr(),
              _dev.ptr(dist), 0.0, None, None, ws.data_ptr(), ws.numel(), _dev.stream())

    def out(t):
        r = _dev.from_device(t, kind)
        if kind == _dev.NUMPY and str(in_dtype) != "float32":
            r = r.astype(in_dtype)
        return r

    return (out(dist), out(p)) if return_dist else out(p)


def select_shp(p, p_max: float):
    """``is_shp = p < p_max`` (bool, same shape as ``p``) and ``shp_num`` (int32 count per pixel).

    ``p`` is compared as float32 widened to double against the double ``p_max``
    (moraine/shp.py:320); NaN is never selected.
    """
    kind = _dev.kind_of(p)
    dev = _dev.require_cuda()
    x = _dev.to_device(p, torch.float32, dev)
    if x.ndim < 3:
        raise ValueError("select_shp: p must be (nlines, width, az_win, r_win)")
    lead = x.shape[:2]
    win = int(torch.tensor(x.shape[2:]).prod().item())
    npix = int(lead[0] * lead[1])
    is_shp = torch.empty(x.shape, dtype=torch.uint8, device=dev)
    shp_num = torch.empty(lead, dtype=torch.int32, device=dev)
    _lib.call("mr_select_shp", x.data_ptr(), npix, win, float(p_max), is_shp.data_ptr(), shp_num.data_ptr(),
              _dev.stream())
    return _dev.from_device(is_shp, kind, as_bool=True), _dev.from_device(shp_num, kind)
