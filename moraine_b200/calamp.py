"""SLC amplitude and its calibration on the device (moraine.calamp).

``rslc2amp`` and ``calamp`` keep the reference's names and behaviour
(moraine/calamp.py:33-71): |z| as float32 for an SLC or a stack, and one image's amplitude
divided by its mean over the non-NaN pixels.
"""
from __future__ import annotations

import torch

from . import _dev, _lib


def rslc2amp(rslc):
    """Amplitude |rslc| (float32, same shape) of an SLC or an SLC stack."""
    kind = _dev.kind_of(rslc)
    dev = _dev.require_cuda()
    z = _dev.to_device(rslc, torch.complex64, dev)
    out = torch.empty(z.shape, dtype=torch.float32, device=dev)
    _lib.call("mr_rslc2amp", z.data_ptr(), z.numel(), out.data_ptr(), _dev.stream())
    return _dev.from_device(out, kind)


def calamp(amp):
    """Calibrated amplitude amp / nanmean(amp) of one image (float32)."""
    kind = _dev.kind_of(amp)
    dev = _dev.require_cuda()
    a = _dev.to_device(amp, torch.float32, dev)
    out = torch.empty(a.shape, dtype=torch.float32, device=dev)
    lib = _lib.load()
    ws = _dev.workspace(lib.mr_calamp_workspace_bytes(), dev)
    _lib.call("mr_calamp", a.data_ptr(), a.numel(), out.data_ptr(), ws.data_ptr(), ws.numel(), _dev.stream())
    return _dev.from_device(out, kind)
