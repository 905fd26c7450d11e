"""The distributed-scatterer chain on one device: the production caller of the kernels.

Replaces the reference's file-based stage drivers (moraine/cli/shp.py:33-123,
moraine/cli/co.py:33-157, moraine/cli/pl.py:223-361) for one tile resident in HBM:

    rslc -> |z|^2 or |z| -> KS test + selection -> DS candidates
         -> [coherence -> EMI (+ temporal coherence)] per batch of DS points

Every intermediate (intensity, sort keys, SHP masks, counts, DS indices, coherence of
the current batch) stays on the device; buffers are allocated once per plan and reused.

``ks_input`` chooses what the KS test ranks: ``"intensity"`` (|z|^2, the rmli of the
reference's API notebooks and of the benchmark scene) or ``"amplitude"`` (|z| as
``rslc2amp`` computes it, the input of the reference's CLI, moraine/cli/shp.py:98). The
test depends only on ranks, but the two roundings make different ties, so each choice is
bit-exact with the reference only against its own input.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import torch

from . import _dev, _lib
from .pl import EMI_REFINE_TOL


@dataclass
class ChainResult:
    n_ds: int
    idx: torch.Tensor          # (n_ds, 2) int32
    ph: torch.Tensor           # (n_ds, N) complex64
    quality: torch.Tensor      # (n_ds,) float32
    t_coh: torch.Tensor        # (n_ds,) float32
    shp_num: torch.Tensor | None  # (nlines, width) int32 (None in graph mode)
    is_shp: torch.Tensor | None   # (nlines, width, az_win, r_win) uint8 (None in graph mode)
    stage_ms: dict = field(default_factory=dict)
    route: torch.Tensor | None = None  # (n_ds,) uint8 EMI route with emi_precision "mixed" or "refine"


class DsChain:
    """Plan and buffers for one (nlines, width, nimages, window) shape."""

    def __init__(self, nlines: int, width: int, nimages: int, az_half_win: int, r_half_win: int,
                 p_max: float = 0.05, min_shp: int = 50, precision: str = "fp32", batch: int | None = None,
                 device=None, timing: bool = False, emi_precision: str | None = None,
                 cond_max: float = 1.0e4, graph: bool = False, ks_input: str = "intensity",
                 refine_tol: float = EMI_REFINE_TOL):
        self.device = torch.device(device) if device is not None else _dev.require_cuda()
        if ks_input not in _lib.KS_INPUT:
            raise ValueError(f"ks_input must be 'intensity' or 'amplitude', not {ks_input!r}")
        self.ks_input = ks_input
        self.shape = (nlines, width, nimages)
        self.azh, self.rh = az_half_win, r_half_win
        self.az_win, self.r_win = 2 * az_half_win + 1, 2 * r_half_win + 1
        self.win = self.az_win * self.r_win
        self.p_max, self.min_shp = float(p_max), int(min_shp)
        self.prec = _lib.PREC[precision]
        # EMI: FP64 with an FP64 Gram, FP32 otherwise (its rounding is below the FP32/BF16
        # coherence error it starts from), unless asked for; "mixed" routes ill-conditioned
        # points to FP64
        if emi_precision is None:
            emi_precision = "fp64" if precision == "fp64" else "fp32"
        if emi_precision not in ("fp32", "fp64", "mixed", "refine"):
            raise ValueError(f"emi_precision must be 'fp32', 'fp64', 'mixed' or 'refine', not {emi_precision!r}")
        self.emi_precision = emi_precision
        self.emi_prec = _lib.PREC[emi_precision]
        self.cond_max = float(cond_max)
        self.refine_tol = float(refine_tol)
        self.timing = timing
        self.npairs = nimages * (nimages - 1) // 2
        npix = nlines * width
        self.batch = int(self.default_batch(npix, nimages) if batch is None else batch)
        lib = _lib.load()
        d = self.device
        self.rmli = torch.empty((nlines, width, nimages), dtype=torch.float32, device=d)
        self.ks_ws = _dev.workspace(lib.mr_ks_workspace_bytes(nlines, width, nimages), d)
        self.is_shp = torch.empty((nlines, width, self.az_win, self.r_win), dtype=torch.uint8, device=d)
        self.shp_num = torch.empty((nlines, width), dtype=torch.int32, device=d)
        self.ex_ws = _dev.workspace(lib.mr_ds_extract_workspace_bytes(npix), d)
        self.idx = torch.empty((npix, 2), dtype=torch.int32, device=d)
        self.n_ds_dev = torch.zeros((1,), dtype=torch.int64, device=d)
        self.coh = torch.empty((self.batch, self.npairs), dtype=torch.complex64, device=d)
        self.emi_ws = _dev.workspace(lib.mr_emi_workspace_bytes(self.batch, nimages), d)
        self.ph = torch.empty((npix, nimages), dtype=torch.complex64, device=d)
        self.quality = torch.empty((npix,), dtype=torch.float32, device=d)
        self.t_coh = torch.empty((npix,), dtype=torch.float32, device=d)
        self.route = (torch.empty((npix,), dtype=torch.uint8, device=d) if emi_precision in ("mixed", "refine")
                      else None)
        # CUDA-graph mode: the whole chain (mr_ds_chain_async, the DS count kept on the device)
        # captured once and replayed for every stack copied into a static input buffer
        self.graph = bool(graph)
        self._graph = None
        if self.graph:
            if (nimages > 128 or precision not in ("fp32", "fp64")
                    or emi_precision not in ("fp32", "fp64", "refine")):
                raise ValueError("DsChain(graph=True) needs nimages <= 128, an fp32/fp64 Gram and fp32, fp64 or "
                                 "refined EMI")
            if emi_precision == "refine" and self.refine_tol != EMI_REFINE_TOL:
                raise ValueError("DsChain(graph=True) refines to the library's default tolerance "
                                 f"({EMI_REFINE_TOL} rad)")
            self.x = torch.empty((nlines, width, nimages), dtype=torch.complex64, device=d)
            gbytes = lib.mr_ds_chain_workspace_bytes(nlines, width, nimages, az_half_win, r_half_win, self.batch)
            self.g_ws = _dev.workspace(gbytes + 256, d)
            self.g_base = (self.g_ws.data_ptr() + 255) & ~255
            self.g_bytes = gbytes
            self.n_ds_g = torch.zeros((1,), dtype=torch.int64, device=d)

    @staticmethod
    def default_batch(npix: int, nimages: int) -> int:
        """DS points per coherence + EMI batch: at most 8 GiB of coherence."""
        npairs = nimages * (nimages - 1) // 2
        return max(1024, min(npix, (8 << 30) // (8 * npairs)))

    @staticmethod
    def footprint(nlines: int, width: int, nimages: int, az_half_win: int, r_half_win: int,
                  batch: int | None = None) -> int:
        """Device bytes the buffers of a plan of this shape occupy."""
        lib = _lib.load()
        npix = nlines * width
        win = (2 * az_half_win + 1) * (2 * r_half_win + 1)
        npairs = nimages * (nimages - 1) // 2
        batch = DsChain.default_batch(npix, nimages) if batch is None else batch
        return int(npix * nimages * 4 + lib.mr_ks_workspace_bytes(nlines, width, nimages) + npix * win + npix * 4
                   + lib.mr_ds_extract_workspace_bytes(npix) + npix * 8 + 8 + batch * npairs * 8
                   + lib.mr_emi_workspace_bytes(batch, nimages) + npix * nimages * 8 + npix * 8)

    def _chain_async(self) -> None:
        nlines, width, n = self.shape
        _lib.call("mr_ds_chain_async", self.x.data_ptr(), nlines, width, n, self.azh, self.rh,
                  _lib.KS_INPUT[self.ks_input], self.p_max, self.min_shp, self.prec, self.emi_prec,
                  self.idx.data_ptr(), self.ph.data_ptr(), self.quality.data_ptr(), self.t_coh.data_ptr(),
                  nlines * width, self.n_ds_g.data_ptr(), self.batch, self.g_base, self.g_bytes, _dev.stream())

    def _run_graph(self, rslc: torch.Tensor) -> ChainResult:
        self.x.copy_(rslc)
        if self._graph is None:
            self._chain_async()  # first call outside the capture: kernel attributes, module load
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._chain_async()
            self._graph = g
        self._graph.replay()
        n_ds = int(self.n_ds_g.item())
        return ChainResult(n_ds, self.idx[:n_ds], self.ph[:n_ds], self.quality[:n_ds], self.t_coh[:n_ds], None, None)

    def run(self, rslc: torch.Tensor, own: tuple[int, int, int, int] | None = None) -> ChainResult:
        """The chain on one stack. ``own = (line0, line1, pixel0, pixel1)`` limits the DS points to
        that part of the stack (a tile's region without its halo); the masks and counts are
        still computed for every pixel, the counts outside ``own`` are then set to 0."""
        nlines, width, n = self.shape
        if tuple(rslc.shape) != self.shape or rslc.dtype != torch.complex64 or not rslc.is_cuda:
            raise ValueError(f"DsChain.run: expected a CUDA complex64 stack of shape {self.shape}, got "
                             f"{rslc.dtype} {tuple(rslc.shape)} on {rslc.device}")
        rslc = rslc.contiguous()
        if own is not None:
            l0, l1, p0, p1 = (int(v) for v in own)
            if not (0 <= l0 <= l1 <= nlines and 0 <= p0 <= p1 <= width):
                raise ValueError(f"DsChain.run: own {own} is not inside the {nlines} x {width} stack")
            if self.graph:
                raise ValueError("DsChain.run: own is not available in graph mode")
        if self.graph:
            return self._run_graph(rslc)
        s = _dev.stream()
        ev = []

        def mark(name):
            if self.timing:
                e = torch.cuda.Event(enable_timing=True)
                e.record()
                ev.append((name, e))

        mark("start")
        prologue = "mr_intensity" if self.ks_input == "intensity" else "mr_rslc2amp"
        _lib.call(prologue, rslc.data_ptr(), rslc.numel(), self.rmli.data_ptr(), s)
        mark("intensity")
        _lib.call("mr_ks_test", self.rmli.data_ptr(), nlines, width, n, self.azh, self.rh, None, None, self.p_max,
                  self.is_shp.data_ptr(), self.shp_num.data_ptr(), self.ks_ws.data_ptr(), self.ks_ws.numel(), s)
        if own is not None and (l0, l1, p0, p1) != (0, nlines, 0, width):
            self.shp_num[:l0].zero_()
            self.shp_num[l1:].zero_()
            self.shp_num[l0:l1, :p0].zero_()
            self.shp_num[l0:l1, p1:].zero_()
        mark("ks_select")
        npix = nlines * width
        _lib.call("mr_ds_extract", self.shp_num.data_ptr(), None, nlines, width, self.win, self.min_shp,
                  self.idx.data_ptr(), None, npix, self.n_ds_dev.data_ptr(), self.ex_ws.data_ptr(),
                  self.ex_ws.numel(), s)
        mark("extract")
        n_ds = int(self.n_ds_dev.item())
        for b0 in range(0, n_ds, self.batch):
            nb = min(self.batch, n_ds - b0)
            _lib.call("mr_emperical_co_pc", rslc.data_ptr(), nlines, width, n, self.idx[b0].data_ptr(), nb,
                      self.is_shp.data_ptr(), 1, self.az_win, self.r_win, None, self.npairs, self.coh.data_ptr(),
                      self.prec, s)
            mark("coherence")
            if self.emi_precision == "refine":
                _lib.call("mr_emi_refined", self.coh.data_ptr(), nb, n, 0, self.refine_tol, self.ph[b0].data_ptr(),
                          self.quality[b0:].data_ptr(), self.t_coh[b0:].data_ptr(), self.route[b0:].data_ptr(),
                          self.emi_ws.data_ptr(), self.emi_ws.numel(), s)
            elif self.route is not None:
                _lib.call("mr_emi_routed", self.coh.data_ptr(), nb, n, 0, self.cond_max, self.ph[b0].data_ptr(),
                          self.quality[b0:].data_ptr(), self.t_coh[b0:].data_ptr(), self.route[b0:].data_ptr(),
                          self.emi_ws.data_ptr(), self.emi_ws.numel(), s)
            else:
                _lib.call("mr_emi", self.coh.data_ptr(), nb, n, 0, self.emi_prec, self.ph[b0].data_ptr(),
                          self.quality[b0:].data_ptr(), self.t_coh[b0:].data_ptr(), self.emi_ws.data_ptr(),
                          self.emi_ws.numel(), s)
            mark("emi_tcoh")
        stage = {}
        if self.timing:
            torch.cuda.synchronize()
            for (_, a), (name, b) in zip(ev[:-1], ev[1:]):
                stage[name] = stage.get(name, 0.0) + a.elapsed_time(b)
        return ChainResult(n_ds, self.idx[:n_ds], self.ph[:n_ds], self.quality[:n_ds], self.t_coh[:n_ds],
                           self.shp_num, self.is_shp, stage,
                           self.route[:n_ds] if self.route is not None else None)
