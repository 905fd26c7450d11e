"""GAMMA raster ingest into HBM (moraine.gamma_ on the device).

``read_gamma_image`` and ``read_gamma_pdata`` keep the reference's names, arguments and
checks (moraine/gamma_.py:13-84) and return torch CUDA tensors: the file's bytes are read
into pinned host memory, copied to the device as they are, and decoded there
(``mr_gamma_decode``: byte swap plus the reference's no-data rule, |x| < 1e-30 -> NaN).
``read_gamma_stack`` reads one image per date straight into a (lines, width, dates) stack,
the layout of the DS chain, with the file reads of one date overlapping the decode of the
previous one.
"""
from __future__ import annotations

import os

import torch

from . import _dev, _lib

_TYPES = {"float": (0, 4, torch.float32), "fcomplex": (1, 8, torch.complex64), "int": (2, 4, torch.int32),
          "double": (3, 8, torch.float64)}


def _type(dtype: str):
    if dtype not in _TYPES:
        raise ValueError("Unsupported data type")
    return _TYPES[dtype]


def _read_pinned(path: str, offset: int, count: int) -> torch.Tensor:
    buf = torch.empty((count,), dtype=torch.uint8, pin_memory=True)
    with open(path, "rb") as f:
        f.seek(offset)
        got = f.readinto(memoryview(buf.numpy()))
    if got != count:
        raise OSError(f"{path}: read {got} of {count} bytes")
    return buf


def _decode(raw_dev: torch.Tensor, n: int, code: int, out: torch.Tensor, stride: int = 1) -> None:
    _lib.call("mr_gamma_decode", raw_dev.data_ptr(), n, code, out.data_ptr(), stride, _dev.stream())


def _lines(imag: str, width: int, nbyte: int, y0: int, ny: int | None) -> tuple[int, int]:
    size = os.path.getsize(imag)
    nlines = int(size / nbyte / width)
    assert y0 <= nlines, "y0 is larger than height."
    if ny is None:
        ny = nlines - y0
    assert y0 + ny <= nlines, "y0+ny is larger than height."
    return nlines, ny


def read_gamma_image(imag: str, width: int, dtype: str = "float", y0: int = 0, ny: int | None = None,
                     device=None) -> torch.Tensor:
    """Lines ``y0 .. y0 + ny`` of a GAMMA raster as a (ny, width) tensor on the device."""
    code, nb, tdt = _type(dtype)
    dev = torch.device(device) if device is not None else _dev.require_cuda()
    _, ny = _lines(imag, width, nb, y0, ny)
    n = ny * width
    out = torch.empty((ny, width), dtype=tdt, device=dev)
    if n == 0:
        return out
    host = _read_pinned(imag, y0 * width * nb, n * nb)
    raw = host.to(dev, non_blocking=True)
    _decode(raw, n, code, out)
    return out


def read_gamma_pdata(imag: str, dtype: str = "float", device=None) -> torch.Tensor:
    """A GAMMA point-data file (moraine/gamma_.py:59-84) as a 1-D tensor on the device."""
    code, nb, tdt = _type(dtype)
    dev = torch.device(device) if device is not None else _dev.require_cuda()
    n = os.path.getsize(imag) // nb
    out = torch.empty((n,), dtype=tdt, device=dev)
    if n:
        _decode(_read_pinned(imag, 0, n * nb).to(dev, non_blocking=True), n, code, out)
    return out


def read_gamma_stack(images: list[str], width: int, dtype: str = "fcomplex", y0: int = 0, ny: int | None = None,
                     device=None) -> torch.Tensor:
    """One GAMMA image per date into a (ny, width, len(images)) stack on the device."""
    code, nb, tdt = _type(dtype)
    dev = torch.device(device) if device is not None else _dev.require_cuda()
    if not images:
        raise ValueError("read_gamma_stack: no images")
    _, ny = _lines(images[0], width, nb, y0, ny)
    n = ny * width
    nd = len(images)
    stack = torch.empty((ny, width, nd), dtype=tdt, device=dev)
    if n == 0:
        return stack
    # two staging slots: the host reads date d + 1 while the device decodes date d
    host = [torch.empty((n * nb,), dtype=torch.uint8, pin_memory=True) for _ in range(2)]
    raw = [torch.empty((n * nb,), dtype=torch.uint8, device=dev) for _ in range(2)]
    done = [None, None]
    flat = stack.view(-1)
    for d, path in enumerate(images):
        _lines(path, width, nb, y0, ny)
        k = d & 1
        if done[k] is not None:
            done[k].synchronize()  # slot k's previous copy has left the pinned buffer
        with open(path, "rb") as f:
            f.seek(y0 * width * nb)
            got = f.readinto(memoryview(host[k].numpy()))
        if got != n * nb:
            raise OSError(f"{path}: read {got} of {n * nb} bytes")
        raw[k].copy_(host[k], non_blocking=True)
        _decode(raw[k], n, code, flat[d:], nd)
        ev = torch.cuda.Event()
        ev.record()
        done[k] = ev
    return stack
