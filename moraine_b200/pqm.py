"""Pixel quality: drop-in ``temp_coh`` (moraine/pqm.py:124-159)."""
from __future__ import annotations

import torch

from . import _dev
from .pl import _temp_coh_device

__all__ = ["temp_coh"]


def temp_coh(intf, rslc, image_pairs=None, block_size: int = 128):
    """Temporal coherence of interferograms (or coherence) against a phase history.

    ``t = |sum_q intf_q conj(r_m) r_j / sqrt(|intf_q|^2 |r_m|^2 |r_j|^2)| / n_pairs`` per
    point; 2-D (point cloud) or 3-D (raster) inputs. Unlike the reference CPU path
    (moraine/pqm.py:57-62), the inputs are left unmodified.
    """
    kind = _dev.kind_of(intf)
    dev = _dev.require_cuda()
    a = _dev.to_device(intf, torch.complex64, dev)
    r = _dev.to_device(rslc, torch.complex64, dev)
    assert a.ndim == r.ndim
    is_ras = a.ndim == 3
    if is_ras:
        h, w = a.shape[:2]
        a = a.reshape(-1, a.shape[-1])
        r = r.reshape(-1, r.shape[-1])
    out = _temp_coh_device("mr_temp_coh", a, r, image_pairs)
    if is_ras:
        out = out.reshape(h, w)
    return _dev.from_device(out, kind)
