"""Persistent-scatterer statistics on the device (moraine.ps).

``amp_disp`` keeps the reference's name and behaviour (moraine/ps.py:65-73): the amplitude
dispersion std(|z|) / mean(|z|) over the dates of every pixel of a (nlines, width, nimages)
stack, float32, NaN where the amplitudes are NaN or all zero.
"""
from __future__ import annotations

import torch

from . import _dev, _lib


def amp_disp(rslc):
    """Amplitude dispersion index (nlines, width) float32 of a complex64 SLC stack."""
    kind = _dev.kind_of(rslc)
    dev = _dev.require_cuda()
    z = _dev.to_device(rslc, torch.complex64, dev)
    if z.dim() != 3:
        raise ValueError("amp_disp: rslc must be (nlines, width, nimages)")
    nlines, width, n = z.shape
    out = torch.empty((nlines, width), dtype=torch.float32, device=dev)
    _lib.call("mr_amp_disp", z.data_ptr(), nlines * width, n, out.data_ptr(), _dev.stream())
    return _dev.from_device(out, kind)
