"""Generate the golden fixtures of the parity tests from the reference itself.

Runs the reference's own CPU (Numba) functions from a Moraine source checkout — pass its
path as the first argument or in the ``MORAINE_REFERENCE`` environment variable — on small
seeded inputs and writes ``tests/golden/*.npz``. Only needed when the fixtures are regenerated; the
tests read the committed ``.npz`` files and never import the reference.

Recipe for importing the reference without its optional dependencies: drop
CUDA_VISIBLE_DEVICES (its ``is_cuda_available`` tests only for the variable), stub
``zarr`` (used by ``tnet`` for save/load only), and load ``utils_, tnet, shp, co, pqm, pl``
as submodules of a bare ``moraine`` package object (its ``__init__`` pulls in plotting
and deep-learning modules).
"""
from __future__ import annotations

import importlib.util
import math
import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


def load_reference(src: str):
    os.environ.pop("CUDA_VISIBLE_DEVICES", None)
    sys.modules.setdefault("zarr", types.ModuleType("zarr"))
    pkg = types.ModuleType("moraine")
    pkg.__path__ = [str(Path(src) / "moraine")]
    sys.modules["moraine"] = pkg

    def ld(name):
        spec = importlib.util.spec_from_file_location(f"moraine.{name}", str(Path(src) / "moraine" / f"{name}.py"))
        m = importlib.util.module_from_spec(spec)
        sys.modules[f"moraine.{name}"] = m
        spec.loader.exec_module(m)
        setattr(pkg, name, m)
        return m

    ld("utils_")
    tnet = ld("tnet")
    shp = ld("shp")
    co = ld("co")
    pqm = ld("pqm")
    pkg.TempNet, pkg.nimage_from_npair = tnet.TempNet, tnet.nimage_from_npair
    pkg.emperical_co_pc, pkg.uncompress_coh = co.emperical_co_pc, co.uncompress_coh
    pkg.uncompress_single_coh_numba = co.uncompress_single_coh_numba
    pl = ld("pl")
    return types.SimpleNamespace(tnet=tnet, shp=shp, co=co, pqm=pqm, pl=pl)


def ks_tables(mr):
    ns = list(range(1, 81)) + [96, 100, 128, 150, 200, 256, 300, 400, 512]
    out = {}
    for n in ns:
        en = math.sqrt(n / 2)
        out[f"n{n}"] = np.array([mr.shp._ks_p_numba((en + 0.12 + 0.11 / en) * abs(k / n)) for k in range(n + 1)],
                                dtype=np.float64).astype(np.float32)
    np.savez_compressed(HERE / "ks_p_tables.npz", **out)


def tricky_rmli(rng, nl, w, n):
    """Exponential intensities with NaNs, ties, signed zeros, infinities and copies."""
    x = rng.exponential(1.0, (nl, w, n)).astype(np.float32)
    x[0, 0, 3] = np.nan                      # NaN in the middle of a series
    x[5, 7, :] = np.nan                      # all-NaN pixel
    x[3, 2, -1] = np.nan                     # NaN at the end
    x[1, 1, :] = 2.5                         # constant series (ties with itself)
    x[1, 2, :] = 2.5                         # identical neighbour (D = 0)
    x[2, 3, : n // 2] = 0.0                  # zeros ...
    x[2, 4, : n // 2] = -0.0                 # ... and negative zeros
    x[4, 4, 0] = np.inf
    x[6, 6, :] = np.round(x[6, 6, :] * 4) / 4  # quantised values -> cross-pixel ties
    x[6, 7, :] = np.round(x[6, 7, :] * 4) / 4
    x[7, 1, :] = x[7, 2, ::-1]               # permutation of a neighbour (D = 0)
    return x


def ks_small(mr, rng):
    res = {}
    for tag, (nl, w, n, azh, rh) in {"a": (16, 20, 17, 2, 3), "b": (9, 11, 8, 5, 5), "c": (12, 12, 40, 3, 1)}.items():
        x = tricky_rmli(rng, nl, w, n)
        dist, p = mr.shp.ks_test(x, azh, rh, return_dist=True)
        p2 = mr.shp.ks_test(x, azh, rh)
        is_shp, shp_num = mr.shp.select_shp(p2, 0.05)
        res.update({f"{tag}_rmli": x, f"{tag}_win": np.array([azh, rh]), f"{tag}_p": p2, f"{tag}_pd": p,
                    f"{tag}_dist": dist, f"{tag}_is_shp": is_shp, f"{tag}_shp_num": shp_num})
    np.savez_compressed(HERE / "ks_small.npz", **res)


def co_small(mr, rng):
    """The reference notebook's coherence inputs (nbs/API/co.ipynb cells 15, 25), seeded."""
    rslc = (rng.random((5, 10, 17), dtype=np.float32) + 1j * rng.random((5, 10, 17), dtype=np.float32)).astype(
        np.complex64)
    azh, rh = 1, 2
    is_shp = rng.choice([False, True], size=(5, 10, 2 * azh + 1, 2 * rh + 1), p=[0.3, 0.7])
    for i in range(5):
        for j in range(10):
            is_shp[i, j, azh, rh] = True
            for k in range(2 * azh + 1):
                for l in range(2 * rh + 1):
                    if not (0 <= i + k - azh < 5 and 0 <= j + l - rh < 10):
                        is_shp[i, j, k, l] = False
    shp_num = np.count_nonzero(is_shp, axis=(-2, -1))
    sel = shp_num >= 3
    idx = np.stack(np.where(sel), -1)
    pc = is_shp[sel]
    coh = mr.co.emperical_co_pc(rslc, idx, pc)
    pairs_bw = mr.tnet.TempNet.from_bandwidth(17, bandwidth=3).image_pairs
    coh_bw = mr.co.emperical_co_pc(rslc, idx, pc, image_pairs=pairs_bw)
    unc = mr.co.uncompress_coh(coh_bw, pairs_bw)
    ph, q = mr.pl.emi(coh)
    t = mr.pl.ds_temp_coh(coh, ph)
    tq = mr.pqm.temp_coh(coh.copy(), ph.copy())
    np.savez_compressed(HERE / "co_small.npz", rslc=rslc, is_shp=is_shp, idx=idx, pc_is_shp=pc, coh=coh,
                        pairs_bw=pairs_bw, coh_bw=coh_bw, unc_bw=unc, ph=ph, quality=q, t_coh=t, t_coh_pqm=tq)


def chain_small(mr):
    sys.path.insert(0, str(REPO))
    from moraine_b200.synth import CONFIGS, make_stack  # noqa: PLC0415

    cfg = CONFIGS["c0"].scaled(nlines=48, width=48, n_patches=6, min_shp=20)
    rslc = make_stack(cfg).numpy()
    re, im = rslc.real.astype(np.float32), rslc.imag.astype(np.float32)
    rmli = (re * re) + (im * im)
    p = mr.shp.ks_test(rmli, cfg.az_half_win, cfg.r_half_win)
    is_shp, shp_num = mr.shp.select_shp(p, cfg.p_max)
    sel = shp_num >= cfg.min_shp
    idx = np.stack(np.where(sel), -1)
    pc = is_shp[sel]
    coh = mr.co.emperical_co_pc(rslc, idx, pc)
    ph, q = mr.pl.emi(coh)
    t = mr.pl.ds_temp_coh(coh, ph)
    ph_f, q_f, t_f = mr.pl.emperical_co_emi_temp_coh_pc(rslc, idx, pc, batch_size=100)
    np.savez_compressed(HERE / "chain_small.npz", rslc=rslc, rmli=rmli, win=np.array([cfg.az_half_win,
                        cfg.r_half_win]), p_max=np.float64(cfg.p_max), min_shp=np.int64(cfg.min_shp),
                        is_shp_bits=np.packbits(is_shp.reshape(-1)), shp_num=shp_num, idx=idx,
                        coh_head=coh[:64], ph=ph, quality=q, t_coh=t, ph_fused=ph_f, quality_fused=q_f,
                        t_coh_fused=t_f)


def chain_images(mr, name: str, side: int, min_shp: int, max_pts: int):
    """The reference chain on a crop of a benchmark scene model at its own image count
    (c1: N = 50, 15 x 31 window; c2: N = 100, 11 x 21 window): SHP masks, coherence of the
    first points, EMI and temporal coherence of at most ``max_pts`` DS points."""
    sys.path.insert(0, str(REPO))
    from moraine_b200.synth import CONFIGS, make_stack  # noqa: PLC0415

    base = CONFIGS[name]
    cfg = base.scaled(nlines=side, width=side, min_shp=min_shp,
                      n_patches=max(4, round(base.n_patches * side * side / (base.nlines * base.width))))
    rslc = make_stack(cfg).numpy()
    re, im = rslc.real.astype(np.float32), rslc.imag.astype(np.float32)
    rmli = (re * re) + (im * im)
    p = mr.shp.ks_test(rmli, cfg.az_half_win, cfg.r_half_win)
    is_shp, shp_num = mr.shp.select_shp(p, cfg.p_max)
    sel = shp_num >= cfg.min_shp
    idx = np.stack(np.where(sel), -1)[:max_pts]
    pc = is_shp[sel][:max_pts]
    coh = mr.co.emperical_co_pc(rslc, idx, pc)
    ph, q = mr.pl.emi(coh)
    t = mr.pl.ds_temp_coh(coh, ph)
    np.savez_compressed(HERE / f"chain_{name}_n{cfg.nimages}.npz", rslc=rslc,
                        win=np.array([cfg.az_half_win, cfg.r_half_win]), p_max=np.float64(cfg.p_max),
                        min_shp=np.int64(cfg.min_shp), is_shp_bits=np.packbits(is_shp.reshape(-1)),
                        shp_num=shp_num, idx=idx, coh_head=coh[:8], ph=ph, quality=q, t_coh=t)


def gamma_samples(rng, dtype: str, count: int) -> np.ndarray:
    """Big-endian samples with the values the no-data rule separates (around 1e-30)."""
    specials = [0.0, -0.0, 1e-31, -1e-31, 9.999999e-31, 1.0000001e-30, 1e-30, -1e-30, 2e-30, 1e-38, 1e-45,
                np.inf, -np.inf, np.nan, 1.0, -3.5, 1e30]
    if dtype == "int":
        v = rng.integers(-2**31, 2**31 - 1, size=count, dtype=np.int64).astype(np.int32)
        v[:5] = [0, 1, -1, 2**31 - 1, -2**31]
        return v.astype(">i4")
    if dtype == "fcomplex":
        re = rng.standard_normal(count).astype(np.float32)
        im = rng.standard_normal(count).astype(np.float32)
        k = len(specials)
        re[:k] = np.array(specials, np.float32)
        im[:k] = np.array(specials[::-1], np.float32)
        re[k:2 * k] = np.array(specials, np.float32)  # pairs with a tiny real part and a zero imaginary one
        im[k:2 * k] = 0
        re[2 * k:2 * k + 4] = [7e-31, 5e-31, 0, 1e-30]
        im[2 * k:2 * k + 4] = [7e-31, 9e-31, 1e-30, 0]
        c = np.empty(count, np.complex64)
        c.real, c.imag = re, im
        return c.astype(">c8")
    f = np.float32 if dtype == "float" else np.float64
    v = (rng.standard_normal(count) * 10).astype(f)
    v[:len(specials)] = np.array(specials, f)
    return v.astype(">f4" if dtype == "float" else ">f8")


def gamma_small(src: str, rng):
    """moraine/gamma_.py:13-56: read_gamma_image on big-endian files of every dtype."""
    import tempfile  # noqa: PLC0415

    spec = importlib.util.spec_from_file_location("moraine_gamma_ref", str(Path(src) / "moraine" / "gamma_.py"))
    g = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(g)
    out = {}
    width, nlines = 13, 11
    with tempfile.TemporaryDirectory() as td:
        for dtype in ("float", "fcomplex", "int", "double"):
            raw = gamma_samples(rng, dtype, width * nlines)
            f = Path(td) / f"img.{dtype}"
            raw.tofile(f)
            out[f"{dtype}_raw"] = np.frombuffer(raw.tobytes(), np.uint8)
            out[f"{dtype}_all"] = g.read_gamma_image(str(f), width, dtype)
            out[f"{dtype}_y3_n5"] = g.read_gamma_image(str(f), width, dtype, y0=3, ny=5)
    out["shape"] = np.array([nlines, width])
    np.savez_compressed(HERE / "gamma_small.npz", **out)


def ps_small(src: str, rng):
    """moraine/ps.py:65 amp_disp and moraine/calamp.py:33,63 rslc2amp / calamp (Numba CPU path)."""
    pkg = sys.modules.get("moraine")
    if pkg is None or not hasattr(pkg, "utils_"):
        load_reference(src)
    pkg = sys.modules["moraine"]

    def ld(name):
        spec = importlib.util.spec_from_file_location(f"moraine.{name}", str(Path(src) / "moraine" / f"{name}.py"))
        m = importlib.util.module_from_spec(spec)
        sys.modules[f"moraine.{name}"] = m
        spec.loader.exec_module(m)
        return m

    ps, cal = ld("ps"), ld("calamp")
    nl, w, n = 23, 19, 17
    z = (rng.standard_normal((nl, w, n)) + 1j * rng.standard_normal((nl, w, n))).astype(np.complex64)
    z *= (10.0 ** rng.uniform(-1, 1, (nl, w, 1))).astype(np.float32)
    z[0, 0, 3] = np.nan            # a NaN date
    z[1, 1, :] = 0                 # all-zero pixel
    z[2, 2, 5] = np.inf + 0j       # an infinite sample
    amp = cal.rslc2amp(z)
    amp0 = amp[:, :, 0].copy()
    amp0[3, 4] = np.nan
    np.savez_compressed(HERE / "ps_small.npz", rslc=z, amp=amp, amp_disp=ps.amp_disp(z), amp0=amp0,
                        calamp=cal.calamp(amp0))


CHUNK_CASES = [((10, 7), (4, -1), (2, 1)), ((2000, 2000), (500, 512), (5, 10)), ((97, 53), (16, 16), (7, 15)),
               ((5, 5), (8, 8), (2, 2)), ((33, 40), (1, 40), (0, 0)), ((20, 18, 5), (8, 6, -1), (2, 3, 0)),
               ((64, 64), (13, 9), (20, 20))]


def chunk_small(src: str):
    """moraine/chunk_.py:62-118: all_chunk_slices_with_overlap and chunkwise_slicing_mapping, the
    halo tiling of dask_from_zarr_overlap (moraine/cli/dask_.py:116) and trim_overlap."""
    sys.modules.setdefault("moraine", types.ModuleType("moraine")).__path__ = [str(Path(src) / "moraine")]
    rt = types.ModuleType("moraine.rtree")  # chunk_ imports HilbertRtree for its point-cloud helpers only
    rt.HilbertRtree = None
    sys.modules["moraine.rtree"] = rt
    spec = importlib.util.spec_from_file_location("moraine.chunk_", str(Path(src) / "moraine" / "chunk_.py"))
    ch = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ch)

    def arr(slices):
        return np.array([[[sl.start, sl.stop] for sl in t] for t in slices], dtype=np.int64)

    out = {}
    for k, (shape, chunks, depths) in enumerate(CHUNK_CASES):
        out[f"case{k}"] = np.array([shape, chunks, depths], dtype=np.int64)
        out[f"overlap{k}"] = arr(ch.all_chunk_slices_with_overlap(shape, chunks, depths))
        i, o, m = ch.chunkwise_slicing_mapping(shape, chunks, depths)
        out[f"in{k}"], out[f"out{k}"], out[f"map{k}"] = arr(i), arr(o), arr(m)
    np.savez_compressed(HERE / "chunk_small.npz", **out)


def main():
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    src = args[0] if args else os.environ.get("MORAINE_REFERENCE")
    if not src:
        sys.exit("usage: make_golden.py <moraine source checkout> [--gamma-only|--ps-only|--chunk-only|--images-only]"
                 " (or set MORAINE_REFERENCE)")
    if "--images-only" in sys.argv:
        mr = load_reference(src)
        chain_images(mr, "c1", 28, 20, 192)
        chain_images(mr, "c2", 24, 20, 192)
        return
    if "--gamma-only" in sys.argv:
        gamma_small(src, np.random.default_rng(20240602))
        return
    if "--ps-only" in sys.argv:
        ps_small(src, np.random.default_rng(20240603))
        return
    if "--chunk-only" in sys.argv:
        chunk_small(src)
        return
    mr = load_reference(src)
    rng = np.random.default_rng(20240601)
    ks_tables(mr)
    ks_small(mr, rng)
    co_small(mr, rng)
    chain_small(mr)
    chain_images(mr, "c1", 28, 20, 192)
    chain_images(mr, "c2", 24, 20, 192)
    gamma_small(src, np.random.default_rng(20240602))
    ps_small(src, np.random.default_rng(20240603))
    chunk_small(src)
    import numba  # noqa: PLC0415

    (HERE / "MANIFEST.txt").write_text(
        "Golden fixtures written by tests/golden/make_golden.py from the reference's CPU (Numba) path.\n"
        f"reference: kanglcn/moraine {open(Path(src) / 'settings.ini').read().split('version = ')[1].split()[0]}\n"
        f"numpy {np.__version__}, numba {numba.__version__}\n")
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
