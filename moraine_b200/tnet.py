"""Temporal network: the pair list that orders compressed coherence.

Mirrors ``moraine.tnet`` (moraine/tnet.py:15-130): ``TempNet.from_bandwidth(N)`` gives the
pairs (m, j), m < j, of the row-major upper triangle (``numpy.triu_indices(N, 1)``) whose
temporal baseline ``j - m`` is at most ``bandwidth``; ``nimage_from_npair`` inverts
Q = N(N-1)/2. Host-side logic only (zarr save/load is not provided).
"""
from __future__ import annotations

import math

import numpy as np

__all__ = ["TempNet", "nimage_from_npair"]


def _pairs_from_bandwidth(nimages: int, bandwidth: int | None = None) -> np.ndarray:
    if bandwidth is None:
        bandwidth = nimages
    assert nimages >= bandwidth
    ref, sec = np.triu_indices(nimages, 1)
    keep = (sec - ref) <= bandwidth
    return np.stack((ref[keep], sec[keep]), axis=-1).astype(np.int32)


def _sorted(p: np.ndarray) -> bool:
    a, b = p[:-1], p[1:]
    return not np.any((a[:, 0] > b[:, 0]) | ((a[:, 0] == b[:, 0]) & (a[:, 1] > b[:, 1])))


def _directed(p: np.ndarray) -> bool:
    return bool(np.all(p[:, 0] < p[:, 1]))


def _connected(p: np.ndarray) -> bool:
    # the first pair of every reference image must link it to the next image
    first = np.ones(len(p), dtype=bool)
    first[1:] = p[1:, 0] != p[:-1, 0]
    return bool(np.all(p[first, 0] == p[first, 1] - 1))


class TempNet:
    def __init__(self, image_pairs, check_if_valid: bool = True):
        image_pairs = np.asarray(image_pairs)
        if check_if_valid:
            if not _sorted(image_pairs):
                raise ValueError("input image pairs are not sorted.")
            if not _directed(image_pairs):
                raise ValueError("input image pairs are not directed (reference index larger than or "
                                 "equal to secondary index).")
            if not _connected(image_pairs):
                raise ValueError("input image pairs are not connected.")
        self._image_pairs = image_pairs.astype(np.int32)
        self._n_images = int(self._image_pairs[-1, -1]) + 1
        self._image_pairs_1d = self._image_pairs[:, 0].astype(np.int64) * self._n_images + self._image_pairs[:, 1]

    @classmethod
    def from_bandwidth(cls, nimages: int, bandwidth: int | None = None) -> "TempNet":
        return cls(_pairs_from_bandwidth(nimages, bandwidth), check_if_valid=False)

    @property
    def image_pairs(self) -> np.ndarray:
        return self._image_pairs

    def image_pairs_idx(self, image_pairs=None, ref=None, sec=None):
        """Index of each (ref, sec) pair in the network, -1 where it is absent."""
        single = False
        if image_pairs is not None:
            ref, sec = image_pairs[:, 0], image_pairs[:, 1]
        else:
            if isinstance(ref, (int, np.integer)):
                assert isinstance(sec, (int, np.integer))
                single = True
                ref, sec = np.array([ref]), np.array([sec])
            else:
                ref, sec = np.array(ref), np.array(sec)
            assert len(ref) == len(sec)
        q = np.asarray(ref).astype(np.int64) * self._n_images + np.asarray(sec)
        pos = np.searchsorted(self._image_pairs_1d, q)
        hit = (pos < len(self._image_pairs_1d)) & (self._image_pairs_1d[np.minimum(pos, len(self._image_pairs_1d) - 1)] == q)
        pos = np.where(hit, pos, -1)
        return pos[0] if single else pos


def nimage_from_npair(npair: int) -> int:
    """Number of images N with N(N-1)/2 == npair; ValueError otherwise."""
    guess = math.ceil(math.sqrt(2 * npair))
    for d in (0, -1, 1, -2, 2):
        n = guess + d
        if n >= 0 and n * (n - 1) == 2 * npair:
            return n
    raise ValueError("input is not correct value of number of all pairs")
