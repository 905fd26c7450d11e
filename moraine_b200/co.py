"""Coherence estimation: drop-in ``emperical_co``, ``emperical_co_pc`` and ``uncompress_coh``.

Same signatures, defaults and output layouts as ``moraine.co`` (moraine/co.py:117-299).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _dev, _lib
from .tnet import TempNet, nimage_from_npair

__all__ = ["emperical_co", "emperical_co_pc", "uncompress_coh"]


def _window(is_shp) -> tuple[int, int]:
    az_win, r_win = int(is_shp.shape[-2]), int(is_shp.shape[-1])
    if az_win % 2 == 0 or r_win % 2 == 0:
        raise ValueError(f"SHP window ({az_win}, {r_win}) must have odd sides")
    return az_win, r_win


def emperical_co(rslc, is_shp, block_size: int = 128):
    """Raster covariance and coherence ``(nlines, width, N, N)`` complex64 over each pixel's SHPs.

    ``cov = sum / n_shp``, ``coh = sum / sqrt(sum|z_m|^2 sum|z_j|^2)`` (moraine/co.py:61-137).
    The reference runs this on the GPU only; here numpy input is accepted too (it is
    copied to the device and back).
    """
    kind = _dev.kind_of(rslc)
    dev = _dev.require_cuda()
    z = _dev.to_device(rslc, torch.complex64, dev)
    m = _dev.to_device(is_shp, torch.uint8, dev)
    nlines, width, nimages = z.shape
    az_win, r_win = _window(m)
    if tuple(m.shape[:2]) != (nlines, width):
        raise ValueError("emperical_co: is_shp must be (nlines, width, az_win, r_win)")
    cov = torch.empty((nlines, width, nimages, nimages), dtype=torch.complex64, device=dev)
    coh = torch.empty_like(cov)
    _lib.call("mr_emperical_co", z.data_ptr(), nlines, width, nimages, m.data_ptr(), az_win, r_win,
              cov.data_ptr(), coh.data_ptr(), _dev.stream())
    return _dev.from_device(cov, kind), _dev.from_device(coh, kind)


def emperical_co_pc(rslc, idx, pc_is_shp, block_size: int = 128, image_pairs=None, precision: str = "fp32"):
    """Point-cloud coherence ``(n_pc, n_pairs)`` complex64 (moraine/co.py:141-266).

    ``idx`` (n_pc, 2) (azimuth, range); ``pc_is_shp`` (n_pc, az_win, r_win) bool; pairs in
    ``image_pairs`` order (default: all pairs, row-major upper triangle). ``precision``
    (an addition to the reference signature): ``"fp32"`` (default, FP32 accumulation like
    the reference GPU kernel), ``"fp64"``, ``"bf16"`` or ``"bf16x3"`` (tensor cores).
    """
    kind = _dev.kind_of(rslc)
    dev = _dev.require_cuda()
    z = _dev.to_device(rslc, torch.complex64, dev)
    nlines, width, nimages = z.shape
    ix = _dev.to_device(idx, torch.int32, dev).reshape(-1, 2)
    m = _dev.to_device(pc_is_shp, torch.uint8, dev)
    az_win, r_win = _window(m)
    n_pc = ix.shape[0]
    if m.shape[0] != n_pc:
        raise ValueError("emperical_co_pc: idx and pc_is_shp disagree on the number of points")
    pairs = None
    if image_pairs is not None:
        ip = np.asarray(image_pairs.cpu() if isinstance(image_pairs, torch.Tensor) else image_pairs).astype(np.int32)
        default = TempNet.from_bandwidth(nimages).image_pairs
        if not (ip.shape == default.shape and np.array_equal(ip, default)):
            pairs = _dev.pairs_tensor(ip, dev)
        n_pairs = ip.shape[0]
    else:
        n_pairs = nimages * (nimages - 1) // 2
    coh = torch.empty((n_pc, n_pairs), dtype=torch.complex64, device=dev)
    prec = _lib.PREC[precision]
    if pairs is not None and prec != _lib.PREC["fp32"]:
        raise NotImplementedError("emperical_co_pc: custom image_pairs run in fp32 only")
    _lib.call("mr_emperical_co_pc", z.data_ptr(), nlines, width, nimages, ix.data_ptr(), n_pc, m.data_ptr(), 0,
              az_win, r_win, _dev.ptr(pairs), n_pairs, coh.data_ptr(), prec, _dev.stream())
    return _dev.from_device(coh, kind)


def uncompress_coh(coh, image_pairs=None):
    """(..., n_pairs) -> (..., N, N) Hermitian with unit diagonal (moraine/co.py:281-299)."""
    kind = _dev.kind_of(coh)
    dev = _dev.require_cuda()
    c = _dev.to_device(coh, torch.complex64, dev)
    lead = tuple(c.shape[:-1])
    if image_pairs is None:
        nimages = nimage_from_npair(c.shape[-1])
        pairs = None
    else:
        ip = np.asarray(image_pairs.cpu() if isinstance(image_pairs, torch.Tensor) else image_pairs)
        nimages = int(ip[-1, -1]) + 1
        pairs = _dev.pairs_tensor(ip, dev)
    n = int(np.prod(lead)) if lead else 1
    out = torch.empty(lead + (nimages, nimages), dtype=torch.complex64, device=dev)
    _lib.call("mr_uncompress_coh", c.data_ptr(), n, nimages, _dev.ptr(pairs), int(c.shape[-1]), out.data_ptr(),
              _dev.stream())
    return _dev.from_device(out, kind)


def ad_intf_pc(ref_rslc, sec_rslc, idx, pc_is_shp, block_size: int = 128, precision: str = "fp32"):
    """Adaptive multilook interferogram of one pair for point-cloud data (moraine/co.py:376-406).

    ``ref_rslc``, ``sec_rslc`` (nlines, width) complex64; ``idx`` (n_pc, 2); ``pc_is_shp``
    (n_pc, az_win, r_win) bool. Returns (n_pc,) complex64, equal to pair (0, 1) of
    ``emperical_co_pc`` on a stack whose first two dates are ``ref_rslc`` and ``sec_rslc``.
    ``precision`` (an addition to the reference signature): ``"fp32"`` (the reference GPU
    kernel's accumulation) or ``"fp64"``. The reference's CPU branch cannot run (it names an
    undefined ``rslc``, moraine/co.py:315); this one serves numpy input through the device.
    """
    kind = _dev.kind_of(ref_rslc)
    dev = _dev.require_cuda()
    a = _dev.to_device(ref_rslc, torch.complex64, dev)
    b = _dev.to_device(sec_rslc, torch.complex64, dev)
    if a.shape != b.shape or a.dim() != 2:
        raise ValueError("ad_intf_pc: ref_rslc and sec_rslc must be 2-D of the same shape")
    nlines, width = a.shape
    ix = _dev.to_device(idx, torch.int32, dev).reshape(-1, 2)
    m = _dev.to_device(pc_is_shp, torch.uint8, dev)
    az_win, r_win = _window(m)
    n_pc = ix.shape[0]
    if m.shape[0] != n_pc:
        raise ValueError("ad_intf_pc: idx and pc_is_shp disagree on the number of points")
    out = torch.empty((n_pc,), dtype=torch.complex64, device=dev)
    if n_pc:
        lib = _lib.load()
        ws = _dev.workspace(lib.mr_ad_intf_pc_workspace_bytes(nlines, width), dev)
        _lib.call("mr_ad_intf_pc", a.data_ptr(), b.data_ptr(), nlines, width, ix.data_ptr(), n_pc, m.data_ptr(), az_win,
                  r_win, out.data_ptr(), _lib.PREC[precision], ws.data_ptr(), ws.numel(), _dev.stream())
    return _dev.from_device(out, kind)
