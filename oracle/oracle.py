"""CPU oracle of the distributed-scatterer chain — TEST INFRASTRUCTURE ONLY.

A restatement of the reference (kanglcn/moraine) algorithms on the host: plain C for the
KS merge, the Gram and the temporal coherence (``cpu_oracle.c``), numpy float64 /
complex128 for EMI. Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline leg use it, as the checker; the product path never calls it.

Parity of this oracle is pinned against the reference's own functions run in the build
container (``tests/golden/make_golden.py`` writes the fixtures, ``tests/test_oracle.py``
checks them).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from ctypes import c_double, c_int, c_int64, c_void_p
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libcpu_oracle.so"

_lib = None


def build() -> Path:
    """Compile ``cpu_oracle.c`` (make in this directory)."""
    r = subprocess.run(["make", "-s", "-C", str(HERE)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}{r.stderr}")
    return LIB


def _load():
    global _lib
    if _lib is None:
        if not LIB.exists() or LIB.stat().st_mtime < (HERE / "cpu_oracle.c").stat().st_mtime:
            build()
        lib = ctypes.CDLL(str(LIB))
        lib.oracle_ks_p.restype = c_double
        lib.oracle_ks_p.argtypes = [c_double]
        lib.oracle_ks_test.argtypes = [c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_int]
        lib.oracle_ks_select.argtypes = [c_void_p, c_int, c_int, c_int, c_int, c_int, c_double, c_void_p, c_void_p,
                                         c_int]
        lib.oracle_co_pc.argtypes = [c_void_p, c_int, c_int, c_int, c_void_p, c_int64, c_void_p, c_int, c_int,
                                     c_void_p, c_int, c_void_p, c_int]
        lib.oracle_co_raster.argtypes = [c_void_p, c_int, c_int, c_int, c_void_p, c_int, c_int, c_void_p, c_void_p,
                                         c_int]
        lib.oracle_temp_coh.argtypes = [c_void_p, c_void_p, c_int64, c_int, c_void_p, c_int, c_int, c_void_p,
                                        c_int]
        _lib = lib
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(c_void_p)


def nthreads_default() -> int:
    return len(os.sched_getaffinity(0))


# ----------------------------------------------------------------------------- pairs
def triu_pairs(n: int) -> np.ndarray:
    """moraine/tnet.py:15-20 with bandwidth = n: all pairs m < j, row-major."""
    r, s = np.triu_indices(n, 1)
    return np.stack((r, s), -1).astype(np.int32)


def nimage_from_npair(q: int) -> int:
    """moraine/tnet.py:123-130."""
    g = math.ceil(math.sqrt(2 * q))
    for d in (0, -1, 1, -2, 2):
        if (g + d) * (g + d - 1) == 2 * q:
            return g + d
    raise ValueError("input is not correct value of number of all pairs")


# ----------------------------------------------------------------------------- KS
def ks_p(x: float) -> float:
    """moraine/shp.py:20-32 in double (Python floats, libm exp)."""
    x2 = -2 * x * x
    p = p2 = 0.0
    sign = 1
    for i in range(1, 101):
        p += sign * 2 * math.exp(x2 * i * i)
        if p == p2:
            return p
        sign = -sign
        p2 = p
    return p


def ks_p_table(n: int) -> np.ndarray:
    """float32 p for every integer statistic k = 0..n (moraine/shp.py:74-76)."""
    en = math.sqrt(n / 2)
    return np.array([np.float32(ks_p((en + 0.12 + 0.11 / en) * abs(k / n))) for k in range(n + 1)], np.float32)


def ks_test(rmli: np.ndarray, az_half_win: int, r_half_win: int, return_dist: bool = False, nthreads: int = 0):
    """moraine/shp.py:269-287 (CPU path): p (and dist) float32 (nlines, width, az_win, r_win)."""
    rmli = np.ascontiguousarray(rmli, dtype=np.float32)
    nl, w, n = rmli.shape
    shape = (nl, w, 2 * az_half_win + 1, 2 * r_half_win + 1)
    p = np.empty(shape, np.float32)
    dist = np.empty(shape, np.float32) if return_dist else None
    _load().oracle_ks_test(_p(rmli), nl, w, n, az_half_win, r_half_win, _p(p),
                           _p(dist) if dist is not None else None, nthreads or nthreads_default())
    return (dist, p) if return_dist else p


def select_shp(p: np.ndarray, p_max: float):
    """moraine/shp.py:309-323: is_shp = p < p_max (float32 widened to float64), count per pixel."""
    is_shp = p.astype(np.float64) < float(p_max)
    return is_shp, np.count_nonzero(is_shp, axis=(-2, -1)).astype(np.int32)


def ks_select(rmli: np.ndarray, az_half_win: int, r_half_win: int, p_max: float, nthreads: int = 0):
    """select_shp(ks_test(rmli), p_max) without the float32 p array (whole scenes):
    is_shp (nlines, width, az_win, r_win) bool and shp_num int32."""
    rmli = np.ascontiguousarray(rmli, dtype=np.float32)
    nl, w, n = rmli.shape
    is_shp = np.empty((nl, w, 2 * az_half_win + 1, 2 * r_half_win + 1), np.uint8)
    num = np.empty((nl, w), np.int32)
    _load().oracle_ks_select(_p(rmli), nl, w, n, az_half_win, r_half_win, float(p_max), _p(is_shp), _p(num),
                             nthreads or nthreads_default())
    return is_shp.view(bool), num


def ds_candidates(is_shp: np.ndarray, shp_num: np.ndarray, min_shp: int):
    """nbs/API/pl.ipynb cell 15: idx = stack(where(shp_num >= min_shp)), pc_is_shp = is_shp[that]."""
    sel = shp_num >= min_shp
    return np.stack(np.where(sel), -1).astype(np.int32), is_shp[sel]


# ----------------------------------------------------------------------------- coherence
def emperical_co_pc(rslc, idx, pc_is_shp, image_pairs=None, nthreads: int = 0) -> np.ndarray:
    """moraine/co.py:194-227: complex128 coherence (n_pc, n_pairs), float64 accumulation."""
    rslc = np.ascontiguousarray(rslc, dtype=np.complex64)
    nl, w, n = rslc.shape
    idx = np.ascontiguousarray(idx, dtype=np.int32).reshape(-1, 2)
    m = np.ascontiguousarray(pc_is_shp).astype(np.uint8)
    pairs = triu_pairs(n) if image_pairs is None else np.ascontiguousarray(image_pairs, dtype=np.int32)
    out = np.empty((idx.shape[0], pairs.shape[0]), np.complex128)
    _load().oracle_co_pc(_p(rslc), nl, w, n, _p(idx), idx.shape[0], _p(m), m.shape[-2], m.shape[-1], _p(pairs),
                         pairs.shape[0], _p(out), nthreads or nthreads_default())
    return out


def emperical_co(rslc, is_shp, nthreads: int = 0):
    """moraine/co.py:61-137 restated on the CPU: complex128 cov and coh (nlines, width, N, N)."""
    rslc = np.ascontiguousarray(rslc, dtype=np.complex64)
    nl, w, n = rslc.shape
    m = np.ascontiguousarray(is_shp).astype(np.uint8)
    cov = np.empty((nl, w, n, n), np.complex128)
    coh = np.empty_like(cov)
    _load().oracle_co_raster(_p(rslc), nl, w, n, _p(m), m.shape[-2], m.shape[-1], _p(cov), _p(coh),
                             nthreads or nthreads_default())
    return cov, coh


def uncompress_coh(coh: np.ndarray, image_pairs=None) -> np.ndarray:
    """moraine/co.py:281-299."""
    if image_pairs is None:
        n = nimage_from_npair(coh.shape[-1])
        image_pairs = triu_pairs(n)
    else:
        n = int(image_pairs[-1, -1]) + 1
    out = np.zeros(coh.shape[:-1] + (n, n), dtype=coh.dtype)
    r, s = image_pairs[:, 0], image_pairs[:, 1]
    out[..., r, s] = coh
    out[..., s, r] = coh.conj()
    out[..., np.arange(n), np.arange(n)] = 1
    return out


# ----------------------------------------------------------------------------- EMI
def emi(coh: np.ndarray, ref: int = 0, chunk: int = 4096):
    """moraine/pl.py:46-65 promoted to float64 / complex128.

    Returns ph (complex128), quality (float64), the eigen-gap ratio
    (lambda_2 - lambda_1) / max|lambda| of M and cond(|Gamma|) per point. An FP32
    computation of the same phases is expected to differ by up to about
    eps32 * cond / gap (see ``phase_tolerance``).
    """
    coh = np.asarray(coh).astype(np.complex128)
    n = nimage_from_npair(coh.shape[-1])
    npts = coh.shape[0]
    ph = np.empty((npts, n), np.complex128)
    q = np.empty(npts, np.float64)
    gap = np.empty(npts, np.float64)
    cond = np.empty(npts, np.float64)
    for s0 in range(0, npts, chunk):
        g = uncompress_coh(coh[s0:s0 + chunk])
        a = np.abs(g)
        wa = np.abs(np.linalg.eigvalsh(a))
        cond[s0:s0 + chunk] = wa.max(-1) / np.maximum(wa.min(-1), 1e-300)
        m = np.linalg.inv(a) * g
        w, v = np.linalg.eigh(m)
        v0 = v[..., 0] * v[..., ref, 0].conj()[..., None]
        ph[s0:s0 + chunk] = v0 / np.abs(v0)
        q[s0:s0 + chunk] = w[..., 0]
        gap[s0:s0 + chunk] = (w[..., 1] - w[..., 0]) / np.maximum(np.abs(w).max(-1), 1e-300)
    return ph, q, gap, cond


def emi_c64(coh: np.ndarray, ref: int = 0):
    """moraine/pl.py:46-65 in the reference's own arithmetic: complex64 / float32 LAPACK
    (inv of |Gamma|, eigh of M), as the reference's CPU path computes it. The CPU baseline's
    arm, not a checker: results follow the complex64 rounding, not FP64."""
    coh = np.asarray(coh, np.complex64)
    g = uncompress_coh(coh)
    m = np.linalg.inv(np.abs(g)) * g
    w, v = np.linalg.eigh(m)
    v0 = v[..., 0] * v[..., ref, 0].conj()[..., None]
    return (v0 / np.abs(v0)).astype(np.complex64), w[..., 0].astype(np.float32)


def phase_tolerance(cond: np.ndarray, gap: np.ndarray, eps: float, floor: float = 1e-4) -> np.ndarray:
    """Per-point phase tolerance (rad) for a computation with unit roundoff ``eps``."""
    return np.maximum(floor, 4.0 * eps * cond / np.maximum(gap, 1e-12))


# ----------------------------------------------------------------------------- temporal coherence
def ds_temp_coh(coh, ph, image_pairs=None, nthreads: int = 0) -> np.ndarray:
    """moraine/pl.py:81-100 in double."""
    return _temp_coh(coh, ph, image_pairs, 0, nthreads)


def temp_coh(intf, rslc, image_pairs=None, nthreads: int = 0) -> np.ndarray:
    """moraine/pqm.py:47-71 and 124-159 in double, inputs left untouched; 2-D or 3-D."""
    intf = np.asarray(intf)
    if intf.ndim == 3:
        h, w = intf.shape[:2]
        out = _temp_coh(intf.reshape(-1, intf.shape[-1]), np.asarray(rslc).reshape(h * w, -1), image_pairs, 1,
                        nthreads)
        return out.reshape(h, w)
    return _temp_coh(intf, rslc, image_pairs, 1, nthreads)


def _temp_coh(intf, ph, image_pairs, pqm, nthreads):
    intf = np.ascontiguousarray(intf, dtype=np.complex64)
    ph = np.ascontiguousarray(ph, dtype=np.complex64)
    n = ph.shape[-1]
    pairs = triu_pairs(n) if image_pairs is None else np.ascontiguousarray(image_pairs, dtype=np.int32)
    out = np.empty(ph.shape[0], np.float64)
    _load().oracle_temp_coh(_p(intf), _p(ph), ph.shape[0], n, _p(pairs), pairs.shape[0], pqm, _p(out),
                            nthreads or nthreads_default())
    return out


# ----------------------------------------------------------------------------- chain
def intensity(rslc: np.ndarray) -> np.ndarray:
    """re*re + im*im in float32, each operation rounded once (the device prologue)."""
    re = np.ascontiguousarray(rslc.real, dtype=np.float32)
    im = np.ascontiguousarray(rslc.imag, dtype=np.float32)
    return (re * re) + (im * im)


def chain(rslc, az_half_win, r_half_win, p_max=0.05, min_shp=50, nthreads: int = 0, emi_chunk: int = 4096,
          ks_input: str = "intensity"):
    """KS -> select -> DS candidates -> coherence -> EMI -> temporal coherence, on the host.

    ks_input: "intensity" ranks |z|^2 (the API notebooks, nbs/API/pl.ipynb cell 15) and
    "amplitude" ranks |z| (the CLI, rslc2amp before ks_test, moraine/cli/shp.py:98)."""
    rmli = intensity(rslc) if ks_input == "intensity" else rslc2amp(rslc)
    p = ks_test(rmli, az_half_win, r_half_win, nthreads=nthreads)
    is_shp, shp_num = select_shp(p, p_max)
    idx, pc = ds_candidates(is_shp, shp_num, min_shp)
    coh = emperical_co_pc(rslc, idx, pc, nthreads=nthreads)
    ph, q, gap, cond = emi(coh.astype(np.complex64), chunk=emi_chunk)
    tc = ds_temp_coh(coh.astype(np.complex64), ph.astype(np.complex64), nthreads=nthreads)
    return dict(p=p, is_shp=is_shp, shp_num=shp_num, idx=idx, coh=coh, ph=ph, quality=q, gap=gap, cond=cond,
                t_coh=tc)


# ----------------------------------------------------------------------------- GAMMA rasters
GAMMA_TYPES = {"float": ">f4", "fcomplex": ">c8", "int": ">i4", "double": ">f8"}


def gamma_decode(raw: bytes, dtype: str) -> np.ndarray:
    """moraine/gamma_.py:46-56: big-endian samples to native, |x| < 1e-30 -> NaN (not for int)."""
    dt = GAMMA_TYPES[dtype]
    data = np.frombuffer(raw, dtype=dt).copy()
    if dtype != "int":
        mask = np.abs(data) < 1e-30
        data[mask] = (np.nan + 1j * np.nan) if dtype == "fcomplex" else np.nan
    return data.astype(data.dtype.newbyteorder("="))


def read_gamma_image(path, width: int, dtype: str = "float", y0: int = 0, ny: int | None = None) -> np.ndarray:
    """moraine/gamma_.py:13-56 restated: lines y0 .. y0 + ny of a GAMMA raster."""
    nb = int(GAMMA_TYPES[dtype][-1])
    size = Path(path).stat().st_size
    nlines = size // nb // width
    if ny is None:
        ny = nlines - y0
    with open(path, "rb") as f:
        f.seek(y0 * width * nb)
        raw = f.read(ny * width * nb)
    return gamma_decode(raw, dtype).reshape(-1, width)


# ----------------------------------------------------------------------------- PS-side statistics
def rslc2amp(rslc) -> np.ndarray:
    """moraine/calamp.py:16-23: |z| as float32, as the reference's Numba build computes it: the
    float32 rounding of the double square root of the double sum of squares (inf if a part is)."""
    z = np.asarray(rslc, np.complex64)
    re, im = z.real.astype(np.float64), z.imag.astype(np.float64)
    with np.errstate(invalid="ignore", over="ignore"):
        a = np.sqrt(re * re + im * im).astype(np.float32)
    a[np.isinf(re) | np.isinf(im)] = np.inf
    return a


def amp_disp(rslc) -> np.ndarray:
    """moraine/ps.py:17-27: std(|z|) / mean(|z|) over the dates, in float64, stored float32."""
    a = rslc2amp(rslc).astype(np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        return (a.std(-1) / a.mean(-1)).astype(np.float32)


def calamp(amp) -> np.ndarray:
    """moraine/calamp.py:46-60: amp / nanmean(amp), the mean in float64."""
    a = np.asarray(amp, np.float32)
    with np.errstate(invalid="ignore", divide="ignore"):
        return (a / np.float32(np.nanmean(a.astype(np.float64)))).astype(np.float32)
