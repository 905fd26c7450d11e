"""Sharding a scene over GPUs: azimuth bands with halos, one process per GPU.

The DS chain has no exchange step: a pixel's SHP mask, coherence and phase history depend
only on the stack inside its window, so a scene splits into azimuth bands that each GPU
processes alone. A band reads ``az_half_win`` extra lines on each side (the halo, as the
reference's Dask overlap in moraine/cli/shp.py:89-104 and moraine/chunk_.py:62) and keeps
the DS points whose centre line it owns; the union over bands equals the whole-scene result
bit for bit, in the same row-major order when the bands are concatenated by rank.
"""
from __future__ import annotations

from dataclasses import dataclass

import torch


@dataclass(frozen=True)
class Band:
    rank: int
    world: int
    own0: int    # first owned line
    own1: int    # one past the last owned line
    read0: int   # first line read (owned lines plus the halo above)
    read1: int   # one past the last line read

    @property
    def lines(self) -> int:
        return self.read1 - self.read0


def band_partition(nlines: int, world: int, az_half_win: int) -> list[Band]:
    """Split ``nlines`` into ``world`` contiguous bands of near-equal size with halos."""
    if world < 1 or nlines < 1:
        raise ValueError("band_partition: need nlines >= 1 and world >= 1")
    bands = []
    for r in range(world):
        o0 = nlines * r // world
        o1 = nlines * (r + 1) // world
        bands.append(Band(r, world, o0, o1, max(0, o0 - az_half_win), min(nlines, o1 + az_half_win)))
    return bands


def owned(idx: torch.Tensor, band: Band) -> torch.Tensor:
    """Boolean mask over band-local DS indices (D, 2) of the points whose centre line the band owns."""
    line = idx[:, 0].long() + band.read0
    return (line >= band.own0) & (line < band.own1)


def to_scene(idx: torch.Tensor, band: Band) -> torch.Tensor:
    """Band-local (line, pixel) indices to scene indices."""
    out = idx.clone()
    out[:, 0] += band.read0
    return out


def run_band(chain_factory, rslc_band: torch.Tensor, band: Band):
    """Run the DS chain on one band; returns (scene idx, ph, quality, t_coh) of its owned points.

    ``chain_factory(nlines, width, nimages)`` builds the chain (``moraine_b200.chain.DsChain``
    with the caller's window, thresholds and device).
    """
    nl, w, n = rslc_band.shape
    if nl != band.lines:
        raise ValueError(f"band {band.rank}: stack has {nl} lines, the band reads {band.lines}")
    res = chain_factory(nl, w, n).run(rslc_band)
    keep = owned(res.idx, band)
    return to_scene(res.idx[keep], band), res.ph[keep], res.quality[keep], res.t_coh[keep]
