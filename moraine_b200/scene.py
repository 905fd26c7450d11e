"""Scenes streamed from host storage through the DS chain in halo tiles.

Replaces the reference's overlapped chunk reads and trims (``dask_from_zarr_overlap``,
moraine/cli/dask_.py:116-143; ``all_chunk_slices_with_overlap`` and
``chunkwise_slicing_mapping``, moraine/chunk_.py:62-118; ``trim_overlap`` in
moraine/cli/shp.py:104) for a stack that need not fit in device memory: the scene is cut
into chunks, each read with ``depth = (az_half_win, r_half_win)`` extra lines and pixels on
every side (clipped at the scene border), and each tile keeps the DS points of its chunk.
A pixel's SHP mask, coherence and phase history depend only on the stack inside its
window, which the halo holds, so the union over tiles equals the whole-scene chain bit for
bit, returned in the same row-major order.

B200 layout of the stream:

* one device plan (``DsChain``) of the largest tile shape serves every tile: smaller
  tiles at the bottom or right border are padded there with NaN samples, which the KS test
  treats exactly as pixels outside the image (a NaN in a series gives p = NaN, never an
  SHP), so padding changes no result of the chunk;
* DS points are extracted from the chunk only (``DsChain.run(own=...)``): coherence and
  EMI, nearly all the device time, never run on halo pixels;
* a reader thread fills one of two pinned host buffers with the next tile while the device
  runs the current one; the host-to-device copy runs on its own stream, and the chain
  waits for it with an event, so reads, copies and compute overlap.

Sources: ``ArraySource`` for anything that slices like numpy (an ndarray, a ``np.memmap``
of a raw stack, a zarr or h5py array), ``GammaSource`` for one big-endian GAMMA
``fcomplex`` file per date (moraine/gamma_.py:13), decoded on the device.
"""
from __future__ import annotations

import itertools
import os
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _dev, _lib


@dataclass(frozen=True)
class Tile:
    """One chunk of the scene: ``read`` is what is read (chunk plus halo, clipped to the scene),
    ``own`` the chunk itself, ``inner`` where the chunk sits inside ``read``; each a
    ((start, stop) per axis) tuple."""
    read: tuple
    own: tuple
    inner: tuple


def chunk_slices(shape, chunks, depths) -> list[Tile]:
    """The tiles of a scene, row-major over the chunk grid.

    Follows moraine/chunk_.py:91-118 (``chunkwise_slicing_mapping``; its ``in`` slices are
    those of ``all_chunk_slices_with_overlap``, :62-80): along each axis of length n, chunk k
    owns [k c, min((k + 1) c, n)) and is read over [max(k c - d, 0), min((k + 1) c + d, n));
    a chunk size below 0 means the whole axis.
    """
    if not (len(shape) == len(chunks) == len(depths)):
        raise ValueError("chunk_slices: shape, chunks and depths must have the same length")
    per_axis = []
    for n, c, d in zip(shape, chunks, depths):
        n, c, d = int(n), int(c), int(d)
        if c < 0:
            c = n
        if c == 0 or d < 0:
            raise ValueError(f"chunk_slices: chunk {c} and depth {d} must be > 0 and >= 0")
        axis = []
        for o0 in range(0, n, c):
            o1 = min(o0 + c, n)
            i0, i1 = max(o0 - d, 0), min(o1 + d, n)
            axis.append(((i0, i1), (o0, o1), (o0 - i0, o1 - i0)))
        per_axis.append(axis)
    return [Tile(*(tuple(parts) for parts in zip(*combo))) for combo in itertools.product(*per_axis)]


# ----------------------------------------------------------------------------- sources
_NAN_C64 = np.complex64(complex(np.nan, np.nan))


class ArraySource:
    """A (nlines, width, nimages) complex64 stack in host storage that slices like numpy."""

    def __init__(self, stack):
        if len(stack.shape) != 3:
            raise ValueError(f"ArraySource: expected a (nlines, width, nimages) stack, got shape {stack.shape}")
        if np.dtype(stack.dtype) != np.complex64:
            raise ValueError(f"ArraySource: expected complex64 samples, got {stack.dtype}")
        self.stack = stack
        self.shape = tuple(int(v) for v in stack.shape)

    def alloc_host(self, ty: int, tx: int, pin: bool) -> torch.Tensor:
        return torch.empty((ty, tx, self.shape[2]), dtype=torch.complex64, pin_memory=pin)

    def stage(self, rows, cols, host: torch.Tensor) -> None:
        """Tile rows x cols into the host buffer, NaN below and right of it."""
        h = host.numpy()
        ty, tx = rows[1] - rows[0], cols[1] - cols[0]
        h[:ty, :tx] = self.stack[rows[0]:rows[1], cols[0]:cols[1]]
        h[ty:] = _NAN_C64
        h[:ty, tx:] = _NAN_C64

    def upload(self, host: torch.Tensor, tile: torch.Tensor) -> None:
        tile.copy_(host, non_blocking=True)

    @property
    def read_bytes_per_pixel(self) -> int:
        return 8 * self.shape[2]


class GammaSource:
    """One GAMMA ``fcomplex`` raster per date (big-endian, moraine/gamma_.py:13-56), read
    through memory maps; the byte swap and the no-data rule (|z| < 1e-30 -> NaN) run on the
    device (``mr_gamma_decode``), interleaving the dates into the tile."""

    def __init__(self, images: list[str], width: int):
        if not images:
            raise ValueError("GammaSource: no images")
        size = os.path.getsize(images[0])
        nlines = size // (8 * width)
        for p in images:
            if os.path.getsize(p) != size:
                raise ValueError(f"GammaSource: {p} has {os.path.getsize(p)} bytes, {images[0]} has {size}")
        self.maps = [np.memmap(p, dtype=">c8", mode="r", shape=(nlines, width)) for p in images]
        self.shape = (int(nlines), int(width), len(images))

    def alloc_host(self, ty: int, tx: int, pin: bool) -> torch.Tensor:
        return torch.empty((self.shape[2], ty, tx, 8), dtype=torch.uint8, pin_memory=pin)

    def stage(self, rows, cols, host: torch.Tensor) -> None:
        h = host.numpy().view(">c8")[..., 0]  # (dates, ty, tx) big-endian
        ty, tx = rows[1] - rows[0], cols[1] - cols[0]
        for d, m in enumerate(self.maps):
            h[d, :ty, :tx] = m[rows[0]:rows[1], cols[0]:cols[1]]
        h[:, ty:] = _NAN_C64
        h[:, :ty, tx:] = _NAN_C64

    def upload(self, host: torch.Tensor, tile: torch.Tensor) -> None:
        raw = host.to(tile.device, non_blocking=True)
        nd, ty, tx = host.shape[:3]
        flat = tile.view(-1)
        stream = _dev.stream()
        for d in range(nd):
            _lib.call("mr_gamma_decode", raw[d].data_ptr(), ty * tx, 1, flat[d:].data_ptr(), nd, stream)

    @property
    def read_bytes_per_pixel(self) -> int:
        return 8 * self.shape[2]


# ----------------------------------------------------------------------------- runner
@dataclass
class SceneResult:
    """Whole-scene results (None when ``run`` was given a sink)."""
    n_ds: int
    idx: np.ndarray             # (n_ds, 2) int32 scene (line, pixel), row-major order
    ph: np.ndarray              # (n_ds, nimages) complex64
    quality: np.ndarray         # (n_ds,) float32
    t_coh: np.ndarray           # (n_ds,) float32
    shp_num: np.ndarray | None  # (nlines, width) int32
    stats: dict = field(default_factory=dict)


@dataclass
class SceneRows:
    """The results of one chunk row (``lines`` = (first, stop) scene lines it owns), handed to
    ``SceneRunner.run``'s ``sink`` in scene order."""
    lines: tuple
    idx: np.ndarray             # (n, 2) int32 scene (line, pixel), row-major order
    ph: np.ndarray              # (n, nimages) complex64
    quality: np.ndarray         # (n,) float32
    t_coh: np.ndarray           # (n,) float32
    shp_num: np.ndarray | None  # (lines[1] - lines[0], width) int32


class SceneRunner:
    """The DS chain over a whole scene in halo tiles of ``chunks = (lines, pixels)`` (< 0: the
    whole axis), streamed from a host source. Arguments after ``chunks`` are those of
    ``DsChain``; ``chain_factory(lines, pixels, nimages)`` replaces the plan (tests)."""

    def __init__(self, shape, az_half_win: int, r_half_win: int, chunks=(512, -1), p_max: float = 0.05,
                 min_shp: int = 50, precision: str = "fp64", emi_precision: str | None = None,
                 ks_input: str = "intensity", batch: int | None = None, device=None, chain_factory=None):
        nlines, width, nimages = (int(v) for v in shape)
        self.shape = (nlines, width, nimages)
        self.tiles = chunk_slices((nlines, width), chunks, (az_half_win, r_half_win))
        ty = max(t.read[0][1] - t.read[0][0] for t in self.tiles)
        tx = max(t.read[1][1] - t.read[1][0] for t in self.tiles)
        self.tile_shape = (ty, tx, nimages)
        if chain_factory is None:
            from .chain import DsChain  # noqa: PLC0415

            dev = torch.device(device) if device is not None else _dev.require_cuda()

            def chain_factory(lines, pixels, n):
                return DsChain(lines, pixels, n, az_half_win, r_half_win, p_max, min_shp, precision=precision,
                               batch=batch, device=dev, emi_precision=emi_precision, ks_input=ks_input)
        self.chain = chain_factory(ty, tx, nimages)
        self.device = torch.device(getattr(self.chain, "device", device or "cpu"))

    def run(self, source, return_shp_num: bool = True, sink=None) -> SceneResult:
        """All tiles of ``source`` through the chain; results on the host in scene row-major order.

        With ``sink`` (a callable), the results are not gathered: each chunk row's are handed
        to ``sink(SceneRows)`` in scene order, one row behind the device so that its copies
        are done without stalling the stream (the reference writes each chunk to its zarr
        store the same way), and the returned ``SceneResult`` holds only counts and stats."""
        if tuple(source.shape) != self.shape:
            raise ValueError(f"SceneRunner.run: source has shape {tuple(source.shape)}, the plan {self.shape}")
        nlines, width, n = self.shape
        ty, tx, _ = self.tile_shape
        dev = self.device
        cuda = dev.type == "cuda"
        t0 = time.perf_counter()
        hosts = [source.alloc_host(ty, tx, cuda) for _ in range(2)]
        tiles_dev = [torch.empty((ty, tx, n), dtype=torch.complex64, device=dev) for _ in range(2)]
        copy_stream = torch.cuda.Stream(device=dev) if cuda else None
        uploaded = [None, None]  # host slot -> event after its last host-to-device copy
        consumed = [None, None]  # device slot -> event after the last chain that read it

        def stage(k: int) -> None:
            slot = k & 1
            if uploaded[slot] is not None:
                uploaded[slot].synchronize()  # the slot's previous tile has left the host buffer
            t = self.tiles[k]
            source.stage(t.read[0], t.read[1], hosts[slot])

        pending, shp_parts, row = [], [], []
        waiting = []  # chunk rows copied to the host, not yet handed to the sink
        delivered = 0
        read_bytes = 0
        empty = (np.empty((0, 2), np.int32), np.empty((0, n), np.complex64), np.empty((0,), np.float32),
                 np.empty((0,), np.float32))

        def deliver(entry) -> int:
            lines, parts, shp_row, ev = entry
            if ev is not None:
                ev.synchronize()
            arrays = tuple(x.numpy() for x in parts) if parts is not None else empty
            shp = None
            if shp_row is not None:
                shp = np.empty((lines[1] - lines[0], width), np.int32)
                for (rows, cols), part in shp_row:
                    shp[rows[0] - lines[0]:rows[1] - lines[0], cols[0]:cols[1]] = part.numpy()
            sink(SceneRows(lines, *arrays, shp))
            return len(arrays[0])

        pool = ThreadPoolExecutor(max_workers=1)
        try:
            fut = pool.submit(stage, 0)
            for k, t in enumerate(self.tiles):
                slot = k & 1
                fut.result()
                if cuda:
                    with torch.cuda.stream(copy_stream):
                        if consumed[slot] is not None:
                            copy_stream.wait_event(consumed[slot])
                        source.upload(hosts[slot], tiles_dev[slot])
                        ev = torch.cuda.Event()
                        ev.record(copy_stream)
                    uploaded[slot] = ev
                    torch.cuda.current_stream(dev).wait_event(ev)
                else:
                    source.upload(hosts[slot], tiles_dev[slot])
                if k + 1 < len(self.tiles):
                    fut = pool.submit(stage, k + 1)
                read_bytes += (t.read[0][1] - t.read[0][0]) * (t.read[1][1] - t.read[1][0]) * \
                    source.read_bytes_per_pixel
                (r0, r1), (c0, c1) = t.inner
                res = self.chain.run(tiles_dev[slot], own=(r0, r1, c0, c1))
                # copy the tile's results out of the plan's buffers before the next tile reuses them
                if res.n_ds:
                    idx = res.idx.clone()
                    idx[:, 0] += t.read[0][0]
                    idx[:, 1] += t.read[1][0]
                    row.append((idx, res.ph.clone(), res.quality.clone(), res.t_coh.clone()))
                if return_shp_num:
                    shp_parts.append((t.own, _to_host(res.shp_num[r0:r1, c0:c1], cuda)))
                if cuda:
                    ev = torch.cuda.Event()
                    ev.record()
                    consumed[slot] = ev
                if k + 1 == len(self.tiles) or self.tiles[k + 1].own[0] != t.own[0]:
                    if sink is None:
                        if row:
                            pending.append(self._merge_row(row, width, cuda))
                    else:
                        parts = self._merge_row(row, width, cuda) if row else None
                        ev = None
                        if cuda:
                            ev = torch.cuda.Event()
                            ev.record()
                        waiting.append((t.own[0], parts, shp_parts if return_shp_num else None, ev))
                        shp_parts = []
                        while len(waiting) > 1:  # the row before this one: its copies are done
                            delivered += deliver(waiting.pop(0))
                    row = []
        finally:
            pool.shutdown(wait=True)
        while waiting:
            delivered += deliver(waiting.pop(0))
        if cuda:
            torch.cuda.current_stream(dev).synchronize()
        if sink is not None:
            wall = time.perf_counter() - t0
            stats = dict(tiles=len(self.tiles), tile_shape=self.tile_shape, read_bytes=read_bytes, wall_s=wall,
                         ds_per_s=delivered / wall if wall > 0 else 0.0)
            return SceneResult(delivered, None, None, None, None, None, stats)
        n_ds = sum(len(p[0]) for p in pending)
        cat = (lambda i, dt, tail: np.concatenate([p[i].numpy() for p in pending]) if pending
               else np.empty((0,) + tail, dt))
        shp = None
        if return_shp_num:
            shp = np.empty((nlines, width), np.int32)
            for (rows, cols), part in shp_parts:
                shp[rows[0]:rows[1], cols[0]:cols[1]] = part.numpy()
        wall = time.perf_counter() - t0
        stats = dict(tiles=len(self.tiles), tile_shape=self.tile_shape, read_bytes=read_bytes, wall_s=wall,
                     ds_per_s=n_ds / wall if wall > 0 else 0.0)
        return SceneResult(n_ds, cat(0, np.int32, (2,)), cat(1, np.complex64, (n,)), cat(2, np.float32, ()),
                           cat(3, np.float32, ()), shp, stats)

    @staticmethod
    def _merge_row(row, width: int, cuda: bool):
        """The DS points of one chunk row (tiles side by side) in row-major order, copied to the host."""
        idx, ph, q, tc = (torch.cat([r[i] for r in row]) for i in range(4))
        if len(row) > 1:
            order = torch.argsort(idx[:, 0].to(torch.int64) * width + idx[:, 1], stable=True)
            idx, ph, q, tc = idx[order], ph[order], q[order], tc[order]
        return tuple(_to_host(x, cuda) for x in (idx, ph, q, tc))


def _to_host(x: torch.Tensor, cuda: bool) -> torch.Tensor:
    """Stream-ordered copy into pinned host memory (complete after the stream synchronises)."""
    if not cuda:
        return x.clone()
    h = torch.empty(x.shape, dtype=x.dtype, pin_memory=True)
    h.copy_(x, non_blocking=True)
    return h
