"""Tile serving: a request loop that runs the DS chain on tiles as they arrive.

Replaces the reference's batch drivers (moraine/cli/shp.py:33, moraine/cli/co.py:33,
moraine/cli/pl.py:223), which walk a zarr stack chunk by chunk through Dask, with a
resident service on one GPU:

* requests (a tile of any size, nimage and window) are queued in arrival order;
* a request is admitted when a slot is free and its device footprint fits the HBM budget
  next to the tiles already running (continuous admission: a tile that arrives while others
  are on the GPU starts as soon as a slot and memory free up, without waiting for a batch
  to drain);
* every slot owns a CUDA stream, so the kernels of admitted tiles overlap on the device;
  rmli, SHP masks, DS indices and coherence stay in HBM between the stages of a tile;
* each result records its arrival, admission and completion times, from which
  ``latency_summary`` gives p50/p99 end-to-end tile latency.

Every DS point is computed by the same kernels with the same per-point arithmetic whether
its tile runs alone or beside others, so results do not depend on the mix.
"""
from __future__ import annotations

import collections
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import Callable

import numpy as np
import torch

from .chain import DsChain


@dataclass
class TileRequest:
    """One tile: a (nlines, width, nimages) complex64 stack and the chain's parameters."""
    rslc: torch.Tensor
    az_half_win: int = 5
    r_half_win: int = 5
    p_max: float = 0.05
    min_shp: int = 50
    precision: str = "fp64"             # coherence Gram arithmetic
    emi_precision: str | None = None    # EMI arithmetic (default: follows the Gram)
    ks_input: str = "intensity"         # what the KS test ranks: "intensity" |z|^2 or "amplitude" |z|
    request_id: int = 0
    arrival: float | None = None   # time.perf_counter() of arrival; set by submit() if None


@dataclass
class TileResult:
    request_id: int
    n_ds: int
    idx: torch.Tensor       # (n_ds, 2) int32, host
    ph: torch.Tensor        # (n_ds, N) complex64, host
    quality: torch.Tensor   # (n_ds,) float32, host
    t_coh: torch.Tensor     # (n_ds,) float32, host
    arrival: float
    admitted: float
    done: float
    footprint: int
    extra: dict = field(default_factory=dict)

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def footprint(req: TileRequest) -> int:
    """Device bytes a request holds while it runs (its stack plus the chain's buffers)."""
    nl, w, n = req.rslc.shape
    stack = 0 if req.rslc.is_cuda else nl * w * n * 8
    return stack + DsChain.footprint(nl, w, n, req.az_half_win, req.r_half_win)


def latency_summary(results: list[TileResult]) -> dict:
    lat = np.array([r.latency for r in results], dtype=np.float64) * 1e3
    if lat.size == 0:
        return {"requests": 0}
    first = min(r.arrival for r in results)
    last = max(r.done for r in results)
    n_ds = int(sum(r.n_ds for r in results))
    return {"requests": int(lat.size), "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()), "max_ms": float(lat.max()),
            "n_ds": n_ds, "span_s": last - first, "ds_pixels_per_s": n_ds / max(last - first, 1e-9)}


_DROP = "drop"  # _take's answer to a slot whose kept memory blocks the head request


class _Item:
    __slots__ = ("req", "fut", "fp")

    def __init__(self, req: TileRequest, fut: Future, fp: int):
        self.req, self.fut, self.fp = req, fut, fp


class DsServer:
    """Request loop over one GPU with ``slots`` concurrent tiles and an HBM admission budget.

    ``runner`` replaces the device chain (``runner(request, stream) -> TileResult fields``);
    it exists for tests of the admission logic without a GPU.

    Accounting: a slot keeps its plan (the chain's buffers) for the next tile of the same
    shape, and the memory it freed stays in its stream's pool of the caching allocator, so
    an idle slot still holds device memory. Each slot is therefore charged the larger of
    what it held before and its running tile's footprint, and keeps that charge when the
    tile ends (``keep_slot_memory``, on for the device chain, off for ``runner``).
    """

    def __init__(self, hbm_budget: float = 150e9, slots: int = 4, device=None,
                 runner: Callable | None = None, footprint_fn: Callable = footprint,
                 keep_slot_memory: bool | None = None):
        self.budget = int(hbm_budget)
        self.slots = int(slots)
        self.used = 0
        self.peak_used = 0
        self.active = 0
        self.peak_active = 0
        self.admitted_order: list[int] = []
        self._queue: collections.deque[_Item] = collections.deque()
        self._cv = threading.Condition()
        self._closed = False
        self._footprint = footprint_fn
        self._runner = runner
        self._keep = (runner is None) if keep_slot_memory is None else bool(keep_slot_memory)
        self._charge = [0] * self.slots  # what each slot counts in self.used
        self._idle: set[int] = set()     # slots waiting for a request
        if runner is None:
            self.device = torch.device(device) if device is not None else torch.device("cuda",
                                                                                       torch.cuda.current_device())
        else:
            self.device = None
        self._workers = [threading.Thread(target=self._work, args=(i,), daemon=True) for i in range(self.slots)]
        for t in self._workers:
            t.start()

    # -------------------------------------------------------------- client side
    def submit(self, req: TileRequest) -> Future:
        fp = int(self._footprint(req))
        if fp > self.budget:
            raise MemoryError(f"tile {req.request_id} needs {fp / 1e9:.2f} GB, over the "
                              f"{self.budget / 1e9:.2f} GB budget")
        if req.arrival is None:
            req.arrival = time.perf_counter()
        fut: Future = Future()
        with self._cv:
            if self._closed:
                raise RuntimeError("server is closed")
            self._queue.append(_Item(req, fut, fp))
            self._cv.notify_all()
        return fut

    def close(self, wait: bool = True) -> None:
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        if wait:
            for t in self._workers:
                t.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -------------------------------------------------------------- slots
    def _fits(self, slot: int) -> bool:
        held = self._charge[slot]
        return self.used - held + max(held, self._queue[0].fp) <= self.budget

    def _take(self, slot: int):
        """The next request for this slot; None when the server closes; _DROP when the head
        request is blocked by memory that idle slots keep, this one's included: the slot then
        gives its memory back (``_drop``) and asks again."""
        with self._cv:
            self._idle.add(slot)
            try:
                while True:
                    held = self._charge[slot]
                    if self._queue and self._fits(slot):
                        item = self._queue.popleft()  # arrival order: the head is admitted first
                        self._charge[slot] = max(held, item.fp)
                        self.used += self._charge[slot] - held
                        self.active += 1
                        self.peak_used = max(self.peak_used, self.used)
                        self.peak_active = max(self.peak_active, self.active)
                        self.admitted_order.append(item.req.request_id)
                        return item
                    if self._closed and not self._queue:
                        return None
                    if self._queue and held > 0 and not any(self._fits(o) for o in self._idle):
                        return _DROP
                    self._cv.wait()
            finally:
                self._idle.discard(slot)

    def _drop(self, slot: int, plan: dict) -> None:
        """Free this slot's kept memory (its plan and its stream's cached blocks) and its charge."""
        plan.clear()
        if self._runner is None:
            torch.cuda.empty_cache()
        with self._cv:
            self.used -= self._charge[slot]
            self._charge[slot] = 0
            self._cv.notify_all()

    def _release(self, item: _Item, slot: int) -> None:
        with self._cv:
            if not self._keep:
                self.used -= self._charge[slot]
                self._charge[slot] = 0
            self.active -= 1
            self._cv.notify_all()

    def _work(self, slot: int) -> None:
        stream = None
        if self._runner is None:
            torch.cuda.set_device(self.device)
            stream = torch.cuda.Stream(self.device)
        plan: dict = {}
        while True:
            item = self._take(slot)
            if item is None:
                return
            if item is _DROP:
                self._drop(slot, plan)
                continue
            admitted = time.perf_counter()
            try:
                if self._runner is not None:
                    out = self._runner(item.req, slot)
                else:
                    with torch.cuda.stream(stream):
                        out = self._run_chain(item.req, plan, stream)
                res = TileResult(request_id=item.req.request_id, arrival=item.req.arrival, admitted=admitted,
                                 done=time.perf_counter(), footprint=item.fp, **out)
                item.fut.set_result(res)
            except BaseException as e:  # noqa: BLE001 - handed to the caller's future
                item.fut.set_exception(e)
            finally:
                self._release(item, slot)

    def _run_chain(self, req: TileRequest, plan: dict, stream) -> dict:
        nl, w, n = req.rslc.shape
        key = (nl, w, n, req.az_half_win, req.r_half_win, req.p_max, req.min_shp, req.precision, req.emi_precision,
               req.ks_input)
        chain = plan.get(key)
        if chain is None:
            plan.clear()  # one plan per slot: a new shape frees the previous buffers
            chain = DsChain(nl, w, n, req.az_half_win, req.r_half_win, req.p_max, req.min_shp,
                            precision=req.precision, emi_precision=req.emi_precision, ks_input=req.ks_input,
                            device=self.device)
            plan[key] = chain
        x = req.rslc
        if not x.is_cuda:
            d = torch.empty(x.shape, dtype=torch.complex64, device=self.device)
            d.copy_(x, non_blocking=True)
            x = d
        r = chain.run(x)
        out = {"n_ds": r.n_ds, "idx": r.idx.cpu(), "ph": r.ph.cpu(), "quality": r.quality.cpu(),
               "t_coh": r.t_coh.cpu()}
        stream.synchronize()
        return out
