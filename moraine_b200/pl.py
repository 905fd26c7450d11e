"""Phase linking: drop-in ``emi``, ``ds_temp_coh`` and ``emperical_co_emi_temp_coh_pc``.

Same signatures, defaults and output layouts as ``moraine.pl`` (moraine/pl.py:68-168).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _dev, _lib
from .tnet import TempNet, nimage_from_npair

__all__ = ["emi", "ds_temp_coh", "emperical_co_emi_temp_coh_pc"]


EMI_COND_MAX = 1.0e4
EMI_REFINE_TOL = 1.0e-4


def _emi_device(c: torch.Tensor, nimages: int, ref: int, want_tcoh: bool = False, precision: str = "fp64",
                cond_max: float = EMI_COND_MAX, route: torch.Tensor | None = None,
                refine_tol: float = EMI_REFINE_TOL):
    dev = c.device
    n_pc = c.shape[0]
    ph = torch.empty((n_pc, nimages), dtype=torch.complex64, device=dev)
    q = torch.empty((n_pc,), dtype=torch.float32, device=dev)
    t = torch.empty((n_pc,), dtype=torch.float32, device=dev) if want_tcoh else None
    lib = _lib.load()
    ws = _dev.workspace(lib.mr_emi_workspace_bytes(n_pc, nimages), dev)
    if precision == "mixed":
        _lib.call("mr_emi_routed", c.data_ptr(), n_pc, nimages, ref, float(cond_max), ph.data_ptr(), q.data_ptr(),
                  _dev.ptr(t), _dev.ptr(route), ws.data_ptr(), ws.numel(), _dev.stream())
    elif precision == "refine":
        _lib.call("mr_emi_refined", c.data_ptr(), n_pc, nimages, ref, float(refine_tol), ph.data_ptr(),
                  q.data_ptr(), _dev.ptr(t), _dev.ptr(route), ws.data_ptr(), ws.numel(), _dev.stream())
    else:
        _lib.call("mr_emi", c.data_ptr(), n_pc, nimages, ref, _lib.PREC[precision], ph.data_ptr(), q.data_ptr(),
                  _dev.ptr(t), ws.data_ptr(), ws.numel(), _dev.stream())
    return ph, q, t


def emi(coh, ref: int = 0, precision: str = "fp64", cond_max: float = EMI_COND_MAX, return_route: bool = False,
        refine_tol: float = EMI_REFINE_TOL):
    """EMI phase linking of compressed coherence ``(n_pc, n_pairs)`` (all pairs).

    Returns ``ph`` (n_pc, N) complex64 (unit modulus, ``ph[:, ref]`` real positive) and
    ``emi_quality`` (n_pc,) float32, the smallest eigenvalue of ``inv(|Gamma|) o Gamma``
    (moraine/pl.py:19-77). Additions to the reference signature: ``precision`` of the whole
    computation, ``"fp64"`` (default), ``"fp32"``, ``"mixed"`` (FP32, with the points
    whose cond_1(|Gamma|) estimate exceeds ``cond_max`` or that are singular in FP32
    redone in FP64) or ``"refine"`` (FP64 inverse of |Gamma|, FP32 reduction, one FP64
    refinement step of the eigenvector, and the points whose phase error bound exceeds
    ``refine_tol`` rad redone in FP64); ``return_route=True`` (mixed or refine) adds a
    uint8 array of the route of every point (mixed: 0 FP32, 1 FP64 by condition, 2 FP64 as
    singular in FP32; refine: 0 refined, 1 redone in FP64, 2 singular).
    """
    if precision not in ("fp32", "fp64", "mixed", "refine"):
        raise ValueError(f"emi: precision must be 'fp32', 'fp64', 'mixed' or 'refine', not {precision!r}")
    if return_route and precision not in ("mixed", "refine"):
        raise ValueError("emi: return_route needs precision='mixed' or 'refine'")
    kind = _dev.kind_of(coh)
    dev = _dev.require_cuda()
    c = _dev.to_device(coh, torch.complex64, dev)
    nimages = nimage_from_npair(c.shape[-1])
    c2 = c.reshape(-1, c.shape[-1])
    route = torch.empty((c2.shape[0],), dtype=torch.uint8, device=dev) if return_route else None
    ph, q, _ = _emi_device(c2, nimages, int(ref), precision=precision, cond_max=cond_max, route=route,
                           refine_tol=refine_tol)
    ph = ph.reshape(tuple(c.shape[:-1]) + (nimages,))
    q = q.reshape(tuple(c.shape[:-1]))
    if return_route:
        return _dev.from_device(ph, kind), _dev.from_device(q, kind), _dev.from_device(
            route.reshape(tuple(c.shape[:-1])), kind)
    return _dev.from_device(ph, kind), _dev.from_device(q, kind)


def _temp_coh_device(name: str, c: torch.Tensor, ph: torch.Tensor, image_pairs):
    dev = c.device
    n, nimages = ph.shape
    pairs = None
    n_pairs = c.shape[-1]
    if image_pairs is not None:
        ip = np.asarray(image_pairs.cpu() if isinstance(image_pairs, torch.Tensor) else image_pairs).astype(np.int32)
        default = TempNet.from_bandwidth(nimages).image_pairs
        if not (ip.shape == default.shape and np.array_equal(ip, default)):
            pairs = _dev.pairs_tensor(ip, dev)
        n_pairs = ip.shape[0]
    elif n_pairs != nimages * (nimages - 1) // 2:
        raise ValueError(f"{name}: {n_pairs} pairs do not match all pairs of {nimages} images")
    if c.shape[-1] != n_pairs:
        raise ValueError(f"{name}: coherence has {c.shape[-1]} pairs, image_pairs has {n_pairs}")
    out = torch.empty((n,), dtype=torch.float32, device=dev)
    _lib.call(name, c.data_ptr(), ph.data_ptr(), n, nimages, _dev.ptr(pairs), n_pairs, out.data_ptr(),
              _dev.stream())
    return out


def ds_temp_coh(coh, ph, image_pairs=None, block_size: int = 128):
    """Temporal coherence ``|sum_q coh_q/|coh_q| conj(ph_m) ph_j| / n_pairs`` (moraine/pl.py:81-145)."""
    kind = _dev.kind_of(coh)
    dev = _dev.require_cuda()
    c = _dev.to_device(coh, torch.complex64, dev)
    p = _dev.to_device(ph, torch.complex64, dev)
    out = _temp_coh_device("mr_ds_temp_coh", c, p, image_pairs)
    return _dev.from_device(out, kind)


def emperical_co_emi_temp_coh_pc(rslc, idx, pc_is_shp, batch_size: int = 1000):
    """Coherence -> EMI -> temporal coherence per batch of points (moraine/pl.py:148-168).

    Results equal separate ``emperical_co_pc``, ``emi`` and ``ds_temp_coh`` calls exactly.
    Coherence only lives per batch on the device; ``batch_size`` is a lower bound on the
    device batch (the batch is widened to keep the GPU busy, within a memory cap).
    """
    from .co import emperical_co_pc  # noqa: PLC0415

    kind = _dev.kind_of(rslc)
    dev = _dev.require_cuda()
    z = _dev.to_device(rslc, torch.complex64, dev)
    ix = _dev.to_device(idx, torch.int32, dev).reshape(-1, 2)
    m = _dev.to_device(pc_is_shp, torch.uint8, dev)
    n_pc = ix.shape[0]
    nimages = z.shape[2]
    npairs = nimages * (nimages - 1) // 2
    cap = max(1, (2 << 30) // (8 * npairs))  # <= 2 GiB of coherence per batch
    bs = int(min(max(batch_size, 65536), cap))
    ph = torch.empty((n_pc, nimages), dtype=torch.complex64, device=dev)
    q = torch.empty((n_pc,), dtype=torch.float32, device=dev)
    t = torch.empty((n_pc,), dtype=torch.float32, device=dev)
    for s0 in range(0, n_pc, bs):
        s1 = min(n_pc, s0 + bs)
        c = emperical_co_pc(z, ix[s0:s1], m[s0:s1])
        p_, q_, _ = _emi_device(c, nimages, 0)
        ph[s0:s1] = p_
        q[s0:s1] = q_
        t[s0:s1] = _temp_coh_device("mr_ds_temp_coh", c, p_, None)
    return _dev.from_device(ph, kind), _dev.from_device(q, kind), _dev.from_device(t, kind)
