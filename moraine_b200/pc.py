"""Raster <-> point cloud on the device (moraine.pc) and DS candidates.

``ras2pc`` and ``pc2ras`` keep the reference's names and arguments (moraine/pc.py:223-241)
for grid indices ``gix`` ((n, 2) integer rows of (line, pixel)); their gathers and
scatters are ``mr_ras2pc`` / ``mr_pc2ras``. A 1-D Hilbert index (``pc2ras`` also accepts
one in the reference, through ``pc_gix``) is not supported: the Hilbert curve belongs to the
point-cloud utilities, which this library leaves out.

``ds_candidates`` is the glue the reference writes between ``select_shp`` and
``emperical_co_pc`` (nbs/API/pl.ipynb cell 15: ``is_ds_can = shp_num >= 50``,
``idx = np.stack(np.where(is_ds_can), -1)``, ``pc_is_shp = is_shp[is_ds_can]``; in the CLI
``pc_logic_ras(shp_num, gix, 'ras>=50')`` and ``ras2pc_ras_chunk``, moraine/cli/pc.py:764,
:239), as one stream compaction (``mr_ds_extract``).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _dev, _lib

# what numpy's ``raster[:] = nan`` writes, per element type: a quiet NaN, and for complex
# types NaN + 0j
_FILL = {torch.float32: np.array([np.nan], np.float32), torch.float64: np.array([np.nan], np.float64),
         torch.complex64: np.array([np.nan, 0.0], np.float32), torch.complex128: np.array([np.nan, 0.0], np.float64),
         torch.float16: None, torch.bfloat16: None}


def _gix(gix, dev) -> torch.Tensor:
    g = _dev.to_device(gix, None, dev)
    if g.ndim != 2 or g.shape[1] != 2:
        raise NotImplementedError(f"grid index of shape {tuple(g.shape)}: only (n, 2) grid indices are supported "
                                  "(the 1-D Hilbert index is not)")
    if g.dtype.is_floating_point or g.dtype.is_complex or g.dtype == torch.uint8:
        raise IndexError("arrays used as indices must be of integer type")
    if g.dtype != torch.int32:
        if g.numel() and (int(g.max()) > np.iinfo(np.int32).max or int(g.min()) < np.iinfo(np.int32).min):
            raise IndexError("grid index beyond the int32 range")
        g = g.to(torch.int32)
    return g.contiguous()


def _record_bytes(t: torch.Tensor) -> int:
    n = 1
    for d in t.shape[2:]:
        n *= int(d)
    return n * t.element_size()


def ras2pc(ras, gix):
    """``ras[gix[:, 0], gix[:, 1]]``: the (n, ...) records of the raster at the grid index."""
    kind = _dev.kind_of(ras)
    is_bool = (ras.dtype == torch.bool) if isinstance(ras, torch.Tensor) else (np.asarray(ras).dtype == np.bool_)
    dev = _dev.require_cuda()
    r = _dev.to_device(ras, None, dev)
    if r.ndim < 2:
        raise IndexError(f"too many indices for a raster of {r.ndim} dimension(s)")
    g = _gix(gix, dev)
    n = g.shape[0]
    out = torch.empty((n, *r.shape[2:]), dtype=r.dtype, device=dev)
    err = torch.zeros((1,), dtype=torch.int32, device=dev)
    _lib.call("mr_ras2pc", r.data_ptr(), r.shape[0], r.shape[1], max(1, _record_bytes(r)), g.data_ptr(), n,
              out.data_ptr(), err.data_ptr(), _dev.stream())
    if n and int(err.item()):
        raise IndexError(f"ras2pc: grid index out of bounds for a {r.shape[0]} x {r.shape[1]} raster")
    return _dev.from_device(out, kind, as_bool=is_bool)


def pc2ras(idx, pc_data, shape: tuple):
    """A raster of ``shape`` (lines, width) filled with NaN, with ``pc_data`` written at ``idx``."""
    kind = _dev.kind_of(pc_data)
    dev = _dev.require_cuda()
    p = _dev.to_device(pc_data, None, dev)
    if p.dtype not in _FILL or _FILL[p.dtype] is None:
        raise ValueError(f"pc2ras: cannot fill a {p.dtype} raster with NaN")
    g = _gix(idx, dev)
    n = g.shape[0]
    if p.shape[0] != n:
        raise ValueError(f"pc2ras: {p.shape[0]} records for {n} indices")
    nl, w = (int(v) for v in shape)
    ras = torch.empty((nl, w, *p.shape[1:]), dtype=p.dtype, device=dev)
    rec = max(1, _record_bytes(ras))
    fill = _FILL[p.dtype]
    err = torch.zeros((1,), dtype=torch.int32, device=dev)
    _lib.call("mr_pc2ras", p.data_ptr(), g.data_ptr(), n, nl, w, rec, fill.ctypes.data, fill.nbytes, ras.data_ptr(),
              err.data_ptr(), _dev.stream())
    if n and int(err.item()):
        raise IndexError(f"pc2ras: grid index out of bounds for a {nl} x {w} raster")
    return _dev.from_device(ras, kind)


def ds_candidates(shp_num, is_shp=None, min_shp: int = 50):
    """``(idx, pc_is_shp)`` of the pixels with ``shp_num >= min_shp``, in row-major order:
    ``idx`` (n, 2) int32 (line, pixel); ``pc_is_shp`` (n, az_win, r_win) bool, or None when
    ``is_shp`` is not given."""
    kind = _dev.kind_of(shp_num)
    dev = _dev.require_cuda()
    s = _dev.to_device(shp_num, torch.int32, dev)
    if s.ndim != 2:
        raise ValueError(f"ds_candidates: shp_num must be 2-D, got shape {tuple(s.shape)}")
    nl, w = s.shape
    m = None
    win = 1
    if is_shp is not None:
        m = _dev.to_device(is_shp, torch.uint8, dev)
        if m.ndim != 4 or tuple(m.shape[:2]) != (nl, w):
            raise ValueError(f"ds_candidates: is_shp of shape {tuple(m.shape)} does not match shp_num {(nl, w)}")
        win = m.shape[2] * m.shape[3]
    npix = nl * w
    lib = _lib.load()
    ws = _dev.workspace(lib.mr_ds_extract_workspace_bytes(npix), dev)
    idx = torch.empty((npix, 2), dtype=torch.int32, device=dev)
    pc = torch.empty((npix, win), dtype=torch.uint8, device=dev) if m is not None else None
    n_dev = torch.zeros((1,), dtype=torch.int64, device=dev)
    _lib.call("mr_ds_extract", s.data_ptr(), _dev.ptr(m), nl, w, win, int(min_shp), idx.data_ptr(), _dev.ptr(pc),
              npix, n_dev.data_ptr(), ws.data_ptr(), ws.numel(), _dev.stream())
    n = int(n_dev.item())
    out_idx = _dev.from_device(idx[:n], kind)
    if pc is None:
        return out_idx, None
    return out_idx, _dev.from_device(pc[:n].view(n, m.shape[2], m.shape[3]), kind, as_bool=True)
