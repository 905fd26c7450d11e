"""The CPU oracle pinned against the reference's own outputs (golden fixtures) and KATs."""
import math

import numpy as np
import pytest
from scipy import stats

from oracle import oracle as O


def test_ks_p_table_matches_reference(golden):
    g = golden("ks_p_tables.npz")
    for key in g.files:
        n = int(key[1:])
        np.testing.assert_array_equal(O.ks_p_table(n), g[key], err_msg=f"N={n}")


def test_ks_p_c_and_python_agree():
    for n in (5, 17, 50, 100, 200):
        en = math.sqrt(n / 2)
        for k in range(n + 1):
            x = (en + 0.12 + 0.11 / en) * (k / n)
            assert O._load().oracle_ks_p(x) == O.ks_p(x)


def test_ks_acceptance_is_non_monotone():
    # k = 0 gives p = 0 (the series ends on an even term), so identical pixels are selected
    t = O.ks_p_table(17)
    assert t[0] == 0.0 and t[1] > 0.99
    acc = (t.astype(np.float64) < 0.05)
    assert acc[0] and not acc[1:8].any() and acc[8:].all()


@pytest.mark.parametrize("tag", ["a", "b", "c"])
def test_ks_test_matches_reference(golden, tag):
    g = golden("ks_small.npz")
    x, (azh, rh) = g[f"{tag}_rmli"], g[f"{tag}_win"]
    p = O.ks_test(x, int(azh), int(rh))
    np.testing.assert_array_equal(p, g[f"{tag}_p"])
    dist, pd = O.ks_test(x, int(azh), int(rh), return_dist=True)
    np.testing.assert_array_equal(pd, g[f"{tag}_pd"])
    # the reference leaves dist uninitialised where only the neighbour is NaN
    ok = ~np.isnan(g[f"{tag}_p"])
    np.testing.assert_array_equal(dist[ok], g[f"{tag}_dist"][ok])
    is_shp, shp_num = O.select_shp(p, 0.05)
    np.testing.assert_array_equal(is_shp, g[f"{tag}_is_shp"])
    np.testing.assert_array_equal(shp_num, g[f"{tag}_shp_num"])


def test_ks_dist_matches_scipy():
    """KAT of nbs/API/shp.ipynb cell 24: dist equals scipy's asymptotic two-sample statistic."""
    rng = np.random.default_rng(7)
    x = np.sort(rng.normal(size=(5, 5, 5)).astype(np.float32), axis=-1)
    x[0, 0] = np.sort(rng.uniform(size=5)).astype(np.float32)
    dist, _ = O.ks_test(x, 5, 5, return_dist=True)
    for a in range(5):
        for r in range(5):
            for k in range(11):
                for l in range(11):
                    sa, sr = a + k - 5, r + l - 5
                    if 0 <= sa < 5 and 0 <= sr < 5:
                        d = stats.ks_2samp(x[a, r], x[sa, sr], method="asymp").statistic
                        assert abs(dist[a, r, k, l] - d) < 1e-7
                    else:
                        assert np.isnan(dist[a, r, k, l])


def test_select_shp_kat():
    """nbs/API/shp.ipynb cells 26-27: select_shp == (p < 0.05, count_nonzero)."""
    rng = np.random.default_rng(3)
    p = rng.random(40 * 40 * 5 * 5).astype(np.float32)
    p[rng.choice(p.size, 300, replace=False)] = np.nan
    p = p.reshape(40, 40, 5, 5)
    is_shp, shp_num = O.select_shp(p, 0.05)
    np.testing.assert_array_equal(is_shp, p < 0.05)
    np.testing.assert_array_equal(shp_num, np.count_nonzero(p < 0.05, axis=(-2, -1)))


def test_co_pc_matches_reference(golden):
    g = golden("co_small.npz")
    coh = O.emperical_co_pc(g["rslc"], g["idx"], g["pc_is_shp"])
    np.testing.assert_allclose(coh, g["coh"], atol=1e-6, rtol=0)
    coh_bw = O.emperical_co_pc(g["rslc"], g["idx"], g["pc_is_shp"], image_pairs=g["pairs_bw"])
    np.testing.assert_allclose(coh_bw, g["coh_bw"], atol=1e-6, rtol=0)
    unc = O.uncompress_coh(g["coh_bw"], g["pairs_bw"])
    np.testing.assert_array_equal(unc, g["unc_bw"])


def test_co_raster_brute_force():
    """KAT of nbs/API/co.ipynb cell 20: raster cov/coh against a direct loop."""
    rng = np.random.default_rng(11)
    rslc = (rng.random((5, 10, 7)) + 1j * rng.random((5, 10, 7))).astype(np.complex64)
    is_shp = rng.random((5, 10, 3, 5)) < 0.7
    is_shp[:, :, 1, 2] = True
    cov, coh = O.emperical_co(rslc, is_shp)
    for i in range(5):
        for j in range(10):
            zs = [rslc[i + m - 1, j + n - 2] for m in range(3) for n in range(5)
                  if is_shp[i, j, m, n] and 0 <= i + m - 1 < 5 and 0 <= j + n - 2 < 10]
            z = np.array(zs, np.complex128)
            s = z.T @ z.conj()
            a = (np.abs(z) ** 2).sum(0)
            np.testing.assert_allclose(cov[i, j], s / len(zs), atol=1e-12)
            np.testing.assert_allclose(coh[i, j], s / np.sqrt(a[:, None] * a[None, :]), atol=1e-12)


def test_raster_pc_layout():
    """nbs/API/co.ipynb cell 35: raster coh[is_ds][:, triu] == emperical_co_pc."""
    rng = np.random.default_rng(5)
    rslc = (rng.random((6, 9, 6)) + 1j * rng.random((6, 9, 6))).astype(np.complex64)
    is_shp = rng.random((6, 9, 3, 5)) < 0.5
    is_shp[:, :, 1, 2] = True
    _, coh = O.emperical_co(rslc, is_shp)
    sel = np.count_nonzero(is_shp, axis=(-2, -1)) >= 3
    idx = np.stack(np.where(sel), -1)
    pc = O.emperical_co_pc(rslc, idx, is_shp[sel])
    r, s = np.triu_indices(6, 1)
    np.testing.assert_allclose(coh[sel][:, r, s], pc, atol=1e-12)


def test_emi_and_temp_coh_vs_reference(golden):
    g = golden("co_small.npz")
    ph, q, gap, cond = O.emi(g["coh"])
    # the reference runs complex64 LAPACK: its phases differ from FP64 by up to about
    # eps32 * cond(|Gamma|) / gap
    tol = O.phase_tolerance(cond, gap, eps=6e-8)
    dphi = np.abs(np.angle(ph * np.conj(g["ph"]))).max(-1)
    assert np.all(dphi <= tol), (dphi / tol).max()
    # eigenvalue error of an FP32 solve ~ eps32 * ||M||, ||M|| <~ cond(|Gamma|)
    assert np.all(np.abs(q - g["quality"]) <= 10 * 6e-8 * cond * np.maximum(1.0, np.abs(q)))
    t = O.ds_temp_coh(g["coh"], g["ph"])
    np.testing.assert_allclose(t, g["t_coh"], atol=1e-6)
    tq = O.temp_coh(g["coh"], g["ph"])
    np.testing.assert_allclose(tq, g["t_coh_pqm"], atol=1e-6)


def test_chain_small_matches_reference(golden):
    g = golden("chain_small.npz")
    azh, rh = (int(v) for v in g["win"])
    rmli = O.intensity(g["rslc"])
    np.testing.assert_array_equal(rmli, g["rmli"])
    p = O.ks_test(rmli, azh, rh)
    is_shp, shp_num = O.select_shp(p, float(g["p_max"]))
    np.testing.assert_array_equal(np.packbits(is_shp.reshape(-1)), g["is_shp_bits"])
    np.testing.assert_array_equal(shp_num, g["shp_num"])
    idx, pc = O.ds_candidates(is_shp, shp_num, int(g["min_shp"]))
    np.testing.assert_array_equal(idx, g["idx"])
    coh = O.emperical_co_pc(g["rslc"], idx, pc)
    np.testing.assert_allclose(coh[:64], g["coh_head"], atol=1e-6)
    # reference fused helper == separate calls (nbs/API/pl.ipynb cell 38)
    np.testing.assert_array_equal(g["ph"], g["ph_fused"])
    np.testing.assert_array_equal(g["t_coh"], g["t_coh_fused"])


def test_ks_input_choice_changes_ties():
    """|z| and |z|^2 rank near-tied samples differently, so the KS input of a chain is part of
    its result: the CLI's rslc2amp (moraine/cli/shp.py:98) and the notebooks' |z|^2 give
    different p values on samples whose magnitudes agree to rounding."""
    rng = np.random.default_rng(11)
    z = (rng.standard_normal((24, 24, 30)) + 1j * rng.standard_normal((24, 24, 30))).astype(np.complex64)
    # range neighbours share four dates up to a phase rotation: equal magnitudes, different roundings
    z[:, 1::2, :4] = z[:, 0:-1:2, :4] * np.complex64(np.exp(0.7j))
    amp, inten = O.rslc2amp(z), O.intensity(z)
    assert (amp[:, 1::2, :4] == amp[:, 0:-1:2, :4]).mean() > (inten[:, 1::2, :4] == inten[:, 0:-1:2, :4]).mean() + 0.1
    pa, pi = O.ks_test(amp, 3, 3), O.ks_test(inten, 3, 3)
    # ranks agree except at the ties |z| makes
    same = (pa == pi) | (np.isnan(pa) & np.isnan(pi))
    assert 0 < (~same).sum() < same.size // 50


def _ks_p_float32_path(n: int) -> np.ndarray:
    """The p table of the reference's CUDA kernel (moraine/shp.py:166-197, T = float32):
    dmax = k / N in float32, x = (en + 0.12 + 0.11 / en) * dmax in double rounded to float32,
    x2 = -2 x^2, terms summed in float32. numpy's float32 exp stands in for CUDA's expf
    (both within a few ulp of exp), so this is the path's value up to that rounding."""
    en = np.sqrt(np.float32(n) / np.float32(2))
    out = np.empty(n + 1, np.float32)
    for k in range(n + 1):
        dmax = np.abs(np.float32(k) / np.float32(n))
        x = np.float32((float(en) + 0.12 + 0.11 / float(en)) * float(dmax))
        x2 = np.float32(-2.0 * float(x) * float(x))
        p = p2 = np.float32(0)
        sign = 1
        for i in range(1, 101):
            p = np.float32(p + np.float32(sign * 2) * np.exp(np.float32(np.float32(x2 * np.float32(i)) * np.float32(i))))
            if p == p2:
                break
            sign = -sign
            p2 = p
        out[k] = p
    return out


def test_ks_p_meets_the_gpu_path_tolerance():
    """The reference checks its CUDA kernel against its Numba path with dist equal and p
    almost equal to 6 decimals (nbs/API/shp.ipynb, the cupy comparison cells). The p table here
    follows the Numba path bit for bit, so it must sit within that tolerance of the CUDA
    kernel's float32 formula for every N and k, with the same SHP decisions at p_max = 0.05."""
    for n in list(range(2, 81)) + [96, 100, 128, 150, 200, 256, 300, 400, 512]:
        f64, f32 = O.ks_p_table(n), _ks_p_float32_path(n)
        assert np.abs(f64.astype(np.float64) - f32).max() < 1.5e-6, n
        np.testing.assert_array_equal(f64.astype(np.float64) < 0.05, f32.astype(np.float64) < 0.05, err_msg=str(n))


@pytest.mark.parametrize("name", ["chain_c1_n50", "chain_c2_n100"])
def test_oracle_chain_at_benchmark_image_counts(golden, name):
    """The oracle chain against the reference's own on crops of the benchmark scene models
    at their image counts (N = 50, 15 x 31 window; N = 100, 11 x 21 window)."""
    g = golden(f"{name}.npz")
    rslc = g["rslc"]
    azh, rh = (int(v) for v in g["win"])
    p = O.ks_test(O.intensity(rslc), azh, rh)
    is_shp, num = O.select_shp(p, float(g["p_max"]))
    np.testing.assert_array_equal(np.packbits(is_shp.reshape(-1)), g["is_shp_bits"])
    np.testing.assert_array_equal(num, g["shp_num"])
    idx, pc = O.ds_candidates(is_shp, num, int(g["min_shp"]))
    k = g["idx"].shape[0]
    np.testing.assert_array_equal(idx[:k], g["idx"])
    coh = O.emperical_co_pc(rslc, idx[:k], pc[:k])
    np.testing.assert_allclose(coh[:8], g["coh_head"], atol=1e-6)
    c64 = coh.astype(np.complex64)
    ph, q, gap, cond = O.emi(c64)
    # the reference's EMI runs complex64 LAPACK: within that arithmetic's bound of FP64
    tol = O.phase_tolerance(cond, gap, eps=4 * 6e-8)
    err = np.abs(np.angle(ph * np.conj(g["ph"]))).max(-1)
    assert np.all(err <= tol), (err / tol).max()
    assert np.all(np.abs(q - g["quality"]) <= 1e-6 * cond * np.maximum(1, np.abs(q)))
    # the reference sums the temporal coherence of its own phases in float32
    np.testing.assert_allclose(O.ds_temp_coh(c64, g["ph"]), g["t_coh"], atol=5e-5)


def test_ks_select_equals_ks_test_then_select(golden):
    """The whole-scene path (table of p over k) decides like ks_test + select_shp."""
    g = golden("chain_c2_n100.npz")
    rmli = O.intensity(g["rslc"])
    azh, rh = (int(v) for v in g["win"])
    is_shp, num = O.ks_select(rmli, azh, rh, 0.05)
    ref_m, ref_n = O.select_shp(O.ks_test(rmli, azh, rh), 0.05)
    np.testing.assert_array_equal(is_shp, ref_m)
    np.testing.assert_array_equal(num, ref_n)
    g = golden("ks_small.npz")
    for tag in ("a", "b", "c"):
        x, (a, r) = g[f"{tag}_rmli"], g[f"{tag}_win"]
        m, c = O.ks_select(x, int(a), int(r), 0.05)
        np.testing.assert_array_equal(m, g[f"{tag}_is_shp"])
        np.testing.assert_array_equal(c, g[f"{tag}_shp_num"])
