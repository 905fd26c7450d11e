"""Parity of the CUDA path (through the C ABI) with the reference fixtures and the oracle."""
import numpy as np
import pytest
import torch

import moraine_b200 as mb
from moraine_b200.chain import DsChain
from moraine_b200.synth import CONFIGS, make_stack
from oracle import oracle as O

pytestmark = pytest.mark.gpu

EPS32, EPS64 = 6e-8, 1.2e-16
# relative error of a coherence accumulated in FP32 over up to ~500 looks (sqrt(S) eps32)
EPS_GRAM32 = 2e-6


# ----------------------------------------------------------------------------- KS
@pytest.mark.parametrize("tag", ["a", "b", "c"])
def test_ks_matches_reference_fixture(cuda, golden, tag):
    g = golden("ks_small.npz")
    x, (azh, rh) = g[f"{tag}_rmli"], (int(v) for v in g[f"{tag}_win"])
    p = mb.ks_test(x, azh, rh)
    np.testing.assert_array_equal(p, g[f"{tag}_p"])
    dist, pd = mb.ks_test(x, azh, rh, return_dist=True)
    np.testing.assert_array_equal(pd, g[f"{tag}_pd"])
    ok = ~np.isnan(g[f"{tag}_p"])
    np.testing.assert_array_equal(dist[ok], g[f"{tag}_dist"][ok])
    is_shp, shp_num = mb.select_shp(p, 0.05)
    np.testing.assert_array_equal(is_shp, g[f"{tag}_is_shp"])
    np.testing.assert_array_equal(shp_num, g[f"{tag}_shp_num"])


def _fused_select(rmli_t, azh, rh, p_max=0.05):
    from moraine_b200 import _dev, _lib
    nl, w, n = rmli_t.shape
    win = (2 * azh + 1) * (2 * rh + 1)
    is_shp = torch.empty((nl, w, win), dtype=torch.uint8, device=rmli_t.device)
    num = torch.empty((nl, w), dtype=torch.int32, device=rmli_t.device)
    p = torch.empty((nl, w, win), dtype=torch.float32, device=rmli_t.device)
    ws = _dev.workspace(_lib.load().mr_ks_workspace_bytes(nl, w, n), rmli_t.device)
    _lib.call("mr_ks_test", rmli_t.data_ptr(), nl, w, n, azh, rh, p.data_ptr(), None, p_max, is_shp.data_ptr(),
              num.data_ptr(), ws.data_ptr(), ws.numel(), _dev.stream())
    return p.cpu().numpy(), is_shp.cpu().numpy().astype(bool), num.cpu().numpy()


@pytest.mark.parametrize("name,size", [("c0", 200), ("c1", 72), ("c2", 64), ("c3", 40)])
def test_ks_bit_exact_vs_oracle(cuda, name, size):
    """Bit-exact p, mask and counts at the configs' image counts and windows."""
    cfg = CONFIGS[name].scaled(nlines=size, width=size + 3)
    z = make_stack(cfg)
    rmli = O.intensity(z.numpy())
    p_ref = O.ks_test(rmli, cfg.az_half_win, cfg.r_half_win)
    is_ref, num_ref = O.select_shp(p_ref, cfg.p_max)
    p, is_shp, num = _fused_select(torch.from_numpy(rmli).to(cuda), cfg.az_half_win, cfg.r_half_win, cfg.p_max)
    np.testing.assert_array_equal(p.reshape(p_ref.shape), p_ref)
    np.testing.assert_array_equal(is_shp.reshape(is_ref.shape), is_ref)
    np.testing.assert_array_equal(num, num_ref)


def test_ks_edges(cuda):
    rng = np.random.default_rng(0)
    # window larger than the image, N = 1 and N = 2, NaN everywhere
    for (nl, w, n, azh, rh) in [(3, 4, 6, 5, 7), (5, 5, 1, 1, 1), (6, 7, 2, 2, 2), (1, 9, 33, 0, 4), (9, 1, 65, 3, 0)]:
        x = rng.exponential(size=(nl, w, n)).astype(np.float32)
        x[0, 0, 0] = np.nan
        np.testing.assert_array_equal(mb.ks_test(x, azh, rh), O.ks_test(x, azh, rh))
    x = np.full((4, 4, 8), np.nan, np.float32)
    assert np.isnan(mb.ks_test(x, 1, 1)).all()


# ----------------------------------------------------------------------------- coherence
def test_co_pc_matches_reference_fixture(cuda, golden):
    g = golden("co_small.npz")
    coh = mb.emperical_co_pc(g["rslc"], g["idx"], g["pc_is_shp"])
    np.testing.assert_allclose(coh, g["coh"], atol=1e-6, rtol=0)
    coh_bw = mb.emperical_co_pc(g["rslc"], g["idx"], g["pc_is_shp"], image_pairs=g["pairs_bw"])
    np.testing.assert_allclose(coh_bw, g["coh_bw"], atol=1e-6, rtol=0)
    np.testing.assert_array_equal(mb.uncompress_coh(g["coh_bw"], g["pairs_bw"]), g["unc_bw"])
    np.testing.assert_array_equal(mb.uncompress_coh(g["coh"]), O.uncompress_coh(g["coh"]))


@pytest.mark.parametrize("precision,tol", [("fp32", 2e-6), ("fp64", 1e-7), ("bf16x3", 3e-5), ("bf16", 1.5e-2)])
@pytest.mark.parametrize("name,size", [("c0", 64), ("c1", 48), ("c2", 48), ("c3", 24)])
def test_co_pc_vs_oracle(cuda, name, size, precision, tol):
    cfg = CONFIGS[name].scaled(nlines=size, width=size)
    z = make_stack(cfg).numpy()
    p = O.ks_test(O.intensity(z), cfg.az_half_win, cfg.r_half_win)
    is_shp, num = O.select_shp(p, cfg.p_max)
    idx, pc = O.ds_candidates(is_shp, num, 1)
    ref = O.emperical_co_pc(z, idx, pc)
    if precision.startswith("bf16") and cfg.nimages > 128:
        with pytest.raises(NotImplementedError):
            mb.emperical_co_pc(z, idx, pc, precision=precision)
        return
    coh = mb.emperical_co_pc(z, idx, pc, precision=precision)
    assert np.abs(coh - ref).max() < tol


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_ad_intf_pc_equals_first_pair(cuda, golden, precision):
    """The reference's own check (nbs/API/co.ipynb#cell46-47): ad_intf_pc of dates 0 and 1
    equals pair (0, 1) of emperical_co_pc, exactly; and both agree with the oracle."""
    g = golden("co_small.npz")
    rslc, idx, pc = g["rslc"], g["idx"], g["pc_is_shp"]
    coh = mb.emperical_co_pc(rslc, idx, pc, precision=precision)
    intf = mb.ad_intf_pc(rslc[:, :, 0].copy(), rslc[:, :, 1].copy(), idx, pc, precision=precision)
    assert intf.shape == (idx.shape[0],) and intf.dtype == np.complex64
    np.testing.assert_array_equal(intf, coh[:, 0])
    two = O.emperical_co_pc(rslc[:, :, :2].copy(), idx, pc)[:, 0]
    np.testing.assert_allclose(intf, two, atol=2e-6 if precision == "fp32" else 2e-7, rtol=0)
    with pytest.raises(ValueError):
        mb.ad_intf_pc(rslc[:, :, 0], rslc[:-1, :, 1], idx, pc)


def test_co_raster_vs_oracle(cuda):
    rng = np.random.default_rng(4)
    z = (rng.standard_normal((9, 13, 7)) + 1j * rng.standard_normal((9, 13, 7))).astype(np.complex64)
    m = rng.random((9, 13, 3, 5)) < 0.6
    m[:, :, 1, 2] = True
    cov, coh = mb.emperical_co(z, m)
    cov_r, coh_r = O.emperical_co(z, m)
    np.testing.assert_allclose(cov, cov_r, atol=2e-6, rtol=1e-5)
    np.testing.assert_allclose(coh, coh_r, atol=2e-6)
    sel = np.count_nonzero(m, axis=(-2, -1)) >= 3
    idx = np.stack(np.where(sel), -1)
    r, s = np.triu_indices(7, 1)
    np.testing.assert_allclose(coh[sel][:, r, s], mb.emperical_co_pc(z, idx, m[sel]), atol=1e-6)


# ----------------------------------------------------------------------------- EMI, temporal coherence
def test_emi_vs_reference_fixture(cuda, golden):
    g = golden("co_small.npz")
    ph, q = mb.emi(g["coh"])
    _, _, gap, cond = O.emi(g["coh"])
    tol = O.phase_tolerance(cond, gap, eps=EPS32)
    assert np.all(np.abs(np.angle(ph * np.conj(g["ph"]))).max(-1) <= tol)
    np.testing.assert_allclose(mb.ds_temp_coh(g["coh"], g["ph"]), g["t_coh"], atol=1e-6)
    np.testing.assert_allclose(mb.temp_coh(g["coh"], g["ph"]), g["t_coh_pqm"], atol=1e-6)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name,size", [("c0", 64), ("c1", 40), ("c2", 40), ("c3", 20)])
def test_emi_vs_fp64_oracle(cuda, name, size, precision):
    """EMI alone on identical complex64 coherence: FP64 and FP32 reductions vs LAPACK FP64."""
    cfg = CONFIGS[name].scaled(nlines=size, width=size)
    z = make_stack(cfg).numpy()
    p = O.ks_test(O.intensity(z), cfg.az_half_win, cfg.r_half_win)
    is_shp, num = O.select_shp(p, cfg.p_max)
    idx, pc = O.ds_candidates(is_shp, num, 1)
    coh = O.emperical_co_pc(z, idx, pc).astype(np.complex64)
    ph_r, q_r, gap, cond = O.emi(coh)
    ph, q = mb.emi(coh, precision=precision)
    # complex64 output rounding bounds the floor; the arithmetic bounds the rest
    eps = 1e3 * EPS64 if precision == "fp64" else 4 * EPS32
    tol = O.phase_tolerance(cond, gap, eps=eps, floor=3e-7 if precision == "fp64" else 2e-6)
    err = np.abs(np.angle(ph * np.conj(ph_r))).max(-1)
    # |Gamma| numerically singular at this precision (e.g. a single look: |Gamma| = ones):
    # the kernel reports NaN there; the reference's inv() raises for exactly singular input
    singular = cond * (EPS32 if precision == "fp32" else EPS64) > 0.05
    nan = np.isnan(err)
    assert not np.any(nan & ~singular)
    ok = ~nan
    assert np.all(err[ok] <= tol[ok]), (err[ok] / tol[ok]).max()
    # |d lambda| <= |dM| ~ eps cond(|Gamma|) |M|: relative 1e-5, or the arithmetic's bound
    qtol = np.maximum(1e-5, eps * cond if precision == "fp64" else 1e-5 * cond) * np.maximum(1, np.abs(q_r))
    bad = ok & (np.abs(q - q_r) > qtol)
    assert not bad.any(), (np.abs(q - q_r)[bad][:4], q_r[bad][:4], cond[bad][:4])
    # well-conditioned points within 1 mrad
    well = cond / np.maximum(gap, 1e-12) < 1e3
    assert err[well].max(initial=0) < 1e-3


def _abs_gamma_cond(coh):
    g = np.abs(O.uncompress_coh(coh.astype(np.complex128)))
    return np.linalg.cond(g, 1)


@pytest.mark.parametrize("name,size", [("c2", 40), ("c3", 24), ("c1", 32)])
def test_emi_mixed_routing(cuda, name, size):
    """Mixed precision: unrouted points equal the FP32 run and routed points the FP64 run, bit
    for bit; the route follows cond_1(|Gamma|)."""
    cfg = CONFIGS[name].scaled(nlines=size, width=size, nimages=min(100, CONFIGS[name].nimages))
    z = make_stack(cfg).numpy()
    p = O.ks_test(O.intensity(z), cfg.az_half_win, cfg.r_half_win)
    is_shp, num = O.select_shp(p, cfg.p_max)
    idx, pc = O.ds_candidates(is_shp, num, 1)
    coh = torch.from_numpy(O.emperical_co_pc(z, idx, pc).astype(np.complex64)).to(cuda)
    n = O.nimage_from_npair(coh.shape[1])
    from moraine_b200.pl import _emi_device
    runs = {prec: _emi_device(coh, n, 0, True, prec) for prec in ("fp32", "fp64")}
    route = torch.empty((coh.shape[0],), dtype=torch.uint8, device=cuda)
    mixed = _emi_device(coh, n, 0, True, "mixed", cond_max=1e4, route=route)
    r = route.cpu().numpy()
    assert set(np.unique(r)) <= {0, 1, 2}
    assert (r == 0).any() and (r != 0).any()
    for k in range(3):
        m = mixed[k].cpu()
        for sel, prec in ((r == 0, "fp32"), (r != 0, "fp64")):
            a = m[torch.from_numpy(sel)].view(torch.int32 if m.dtype == torch.float32 else torch.float32)
            b = runs[prec][k].cpu()[torch.from_numpy(sel)]
            b = b.view(torch.int32 if b.dtype == torch.float32 else torch.float32)
            assert torch.equal(a, b), (name, k, prec)
    # the estimate is cond_1(|Gamma|) itself, evaluated in FP32
    cond = _abs_gamma_cond(coh.cpu().numpy())
    assert np.all(cond[r == 1] > 1e4 / 2)
    assert np.all((cond[r == 0] < 1e4 * 2) | ~np.isfinite(cond[r == 0]))
    # everything routed by condition / nothing routed
    route.fill_(9)
    _emi_device(coh, n, 0, False, "mixed", cond_max=1.0, route=route)
    assert torch.all(route.cpu() != 0)
    _emi_device(coh, n, 0, False, "mixed", cond_max=1e30, route=route)
    assert not torch.any(route.cpu() == 1)
    # python API
    ph, q, rt = mb.emi(coh.cpu().numpy(), precision="mixed", return_route=True)
    np.testing.assert_array_equal(rt, r)
    with pytest.raises(ValueError):
        mb.emi(coh.cpu().numpy(), precision="fp32", return_route=True)


@pytest.mark.parametrize("name,size", [("c0", 64), ("c1", 40), ("c2", 40), ("c3", 24)])
def test_emi_refine_vs_fp64_oracle(cuda, name, size):
    """Refined mixed precision (FP64 inverse, FP32 reduction, one FP64 refinement step):
    kept points are within their own bound (1e-4 rad) of the FP64 computation, points
    redone in FP64 equal the FP64 run bit for bit, and the route follows the bound."""
    cfg = CONFIGS[name].scaled(nlines=size, width=size)
    z = make_stack(cfg).numpy()
    p = O.ks_test(O.intensity(z), cfg.az_half_win, cfg.r_half_win)
    is_shp, num = O.select_shp(p, cfg.p_max)
    idx, pc = O.ds_candidates(is_shp, num, 1)
    coh = O.emperical_co_pc(z, idx, pc).astype(np.complex64)
    ph_r, q_r, gap, cond = O.emi(coh)
    ph, q, route = mb.emi(coh, precision="refine", return_route=True)
    ph64, q64 = mb.emi(coh, precision="fp64")
    if cfg.nimages > 128:  # FP64 throughout above 128 images: every point reported recomputed
        assert np.all(route == 1)
        np.testing.assert_array_equal(ph.view(np.int32), ph64.view(np.int32))
        return
    assert set(np.unique(route)) <= {0, 1, 2}
    kept, redone = route == 0, route == 1
    assert kept.mean() > 0.5
    tol64 = O.phase_tolerance(cond, gap, eps=1e3 * EPS64, floor=3e-7)
    err = np.abs(np.angle(ph * np.conj(ph_r))).max(-1)
    assert np.all(err[kept] <= tol64[kept] + 1e-4), (err[kept] - tol64[kept]).max()
    # the refinement reaches FP64-class accuracy on the typical point
    assert np.median(err[kept]) < 1e-6
    np.testing.assert_array_equal(ph[redone].view(np.int32), ph64[redone].view(np.int32))
    np.testing.assert_array_equal(q[redone].view(np.int32), q64[redone].view(np.int32))
    assert np.all(np.isnan(ph[route == 2]))
    qtol = np.maximum(1e-5, 1e3 * EPS64 * cond) * np.maximum(1, np.abs(q_r))
    assert np.all(np.abs(q - q_r)[kept] <= qtol[kept])
    # a bound nothing meets sends every point to FP64; one everything meets keeps them all
    _, _, r0 = mb.emi(coh, precision="refine", return_route=True, refine_tol=1e-30)
    assert np.all(r0 != 0)
    # a bound everything meets redoes only the points whose gap estimate is not positive
    # (no bound can be certified for them), a subset of those redone at the default
    ph1, _, r1 = mb.emi(coh, precision="refine", return_route=True, refine_tol=1e30)
    assert np.all(redone[r1 == 1])
    np.testing.assert_array_equal(ph1[kept].view(np.int32), ph[kept].view(np.int32))


def test_chain_refine_route(cuda):
    cfg = CONFIGS["c2"].scaled(nlines=40, width=40)
    z = make_stack(cfg, device=cuda)
    kw = dict(device=cuda, precision="fp64")
    res = DsChain(40, 40, cfg.nimages, cfg.az_half_win, cfg.r_half_win, cfg.p_max, 1, emi_precision="refine",
                  **kw).run(z)
    ref = DsChain(40, 40, cfg.nimages, cfg.az_half_win, cfg.r_half_win, cfg.p_max, 1, **kw).run(z)
    assert res.route is not None and res.route.shape == (res.n_ds,)
    err = (res.ph * ref.ph.conj()).angle().abs().amax(-1)
    keep = res.route == 0
    assert keep.float().mean() > 0.5
    assert float(err[keep].max()) < 2e-4
    again = (res.route == 1)
    assert torch.equal(res.ph[again], ref.ph[again])


@pytest.mark.parametrize("n", [2, 3, 4, 5, 15, 16, 17, 18, 31, 32, 33, 47, 64, 65, 99, 100, 101, 112, 113, 127, 128])
def test_emi_refine_every_block_shape(cuda, n):
    """The refined EMI (pivot-pair sweep, FP32 reduction, FP64 correction) at every parity and
    16-block boundary of N: kept points agree with the FP64 run within the refinement bound,
    recomputed points equal it bit for bit."""
    rng = np.random.default_rng(n)
    looks = 2 * n + 8
    z = rng.normal(size=(96, looks, n)) + 1j * rng.normal(size=(96, looks, n))
    C = np.einsum("pli,plj->pij", z, z.conj())
    d = np.sqrt(np.einsum("pii->pi", C).real)
    C = C / (d[:, :, None] * d[:, None, :])
    r, s = np.triu_indices(n, 1)
    coh = C[:, r, s].astype(np.complex64)
    ph, q, route = mb.emi(coh, precision="refine", return_route=True)
    ph64, q64 = mb.emi(coh, precision="fp64")
    kept, redone = route == 0, route == 1
    assert kept.mean() > 0.5
    err = np.abs(np.angle(ph * np.conj(ph64))).max(-1)
    assert np.all(err[kept] <= 2e-4), err[kept].max()
    np.testing.assert_array_equal(ph[redone].view(np.int32), ph64[redone].view(np.int32))
    np.testing.assert_allclose(q[kept], q64[kept], rtol=1e-4, atol=1e-5)


def test_refine_reruns_across_sub_batches(cuda):
    """More points than one sub-batch (capped at 4,096 points here): the points routed to FP64
    in every sub-batch are recomputed together after the last one. Copies of a point give the
    same bits and route wherever they fall; with a bound nothing meets, every point is
    recomputed (a list three sub-batches long) and equals the FP64 run."""
    from moraine_b200 import _lib
    cfg = CONFIGS["c2"].scaled(nlines=40, width=40)
    z = make_stack(cfg).numpy()
    p = O.ks_test(O.intensity(z), cfg.az_half_win, cfg.r_half_win)
    is_shp, num = O.select_shp(p, cfg.p_max)
    idx, pc = O.ds_candidates(is_shp, num, 1)
    base = O.emperical_co_pc(z, idx, pc).astype(np.complex64)
    reps = -(-12000 // base.shape[0])
    coh = np.tile(base, (reps, 1))
    lib = _lib.load()
    assert lib.mr_set_emi_sub_batch(4096) == 0
    try:
        assert coh.shape[0] > 2 * 4096
        ph, q, route = mb.emi(coh, precision="refine", return_route=True)
        m = base.shape[0]
        for k in range(1, reps):
            np.testing.assert_array_equal(ph[k * m:(k + 1) * m].view(np.int32), ph[:m].view(np.int32))
            np.testing.assert_array_equal(route[k * m:(k + 1) * m], route[:m])
        ph64, q64 = mb.emi(coh, precision="fp64")
        redone = route == 1
        np.testing.assert_array_equal(ph[redone].view(np.int32), ph64[redone].view(np.int32))
        ph_all, q_all, r_all = mb.emi(coh, precision="refine", return_route=True, refine_tol=1e-30)
        assert np.all(r_all != 0)
        ok = r_all == 1  # route 2: singular in FP64 as well, NaN
        assert ok.mean() > 0.99
        np.testing.assert_array_equal(ph_all[ok].view(np.int32), ph64[ok].view(np.int32))
        np.testing.assert_array_equal(q_all[ok].view(np.int32), q64[ok].view(np.int32))
        # the same bits as without the cap
        assert lib.mr_set_emi_sub_batch(0) == 0
        ph_one, _, route_one = mb.emi(coh, precision="refine", return_route=True)
        np.testing.assert_array_equal(ph_one.view(np.int32), ph.view(np.int32))
        np.testing.assert_array_equal(route_one, route)
    finally:
        lib.mr_set_emi_sub_batch(0)


def test_refine_small_pivot_goes_to_fp64(cuda):
    """A point whose |Gamma| meets a tiny pivot in natural order (|gamma_01|^2 within 1e-10
    of 1, so the second pivot of the symmetric sweep is below 1e-9) is flagged by the sweep
    and recomputed by the pivoted FP64 path: the same bits as the FP64 run."""
    rng = np.random.default_rng(5)
    n = 12
    th = np.linspace(0.1, 1.5, 200001)  # a complex64 value of modulus 1 - O(1e-11)
    re, im = np.cos(th).astype(np.float32), np.sin(th).astype(np.float32)
    deficit = 1 - (re.astype(np.float64) ** 2 + im.astype(np.float64) ** 2)
    k = int(np.flatnonzero((deficit > 1e-11) & (deficit < 1e-10))[0])
    g = np.full((n, n), 0.3) + 0.05 * rng.random((n, n))
    g = (g + g.T) / 2
    np.fill_diagonal(g, 1.0)
    ph = np.exp(1j * rng.uniform(-np.pi, np.pi, n))
    G = g * np.outer(ph, ph.conj())
    G[0, 1] = complex(re[k], im[k])
    r, s = np.triu_indices(n, 1)
    ok = rng.normal(size=(40, n)) + 1j * rng.normal(size=(40, n))  # an ordinary point beside it
    C = ok.conj().T @ ok
    d = np.sqrt(np.diag(C).real)
    Cn = C / np.outer(d, d)
    coh = np.stack([G[r, s], Cn[r, s]]).astype(np.complex64)
    assert coh[0, 0] == np.complex64(complex(re[k], im[k]))
    ph_r, q_r, route = mb.emi(coh, precision="refine", return_route=True)
    ph64, q64 = mb.emi(coh, precision="fp64")
    assert route[0] == 1
    np.testing.assert_array_equal(ph_r[0].view(np.int32), ph64[0].view(np.int32))
    np.testing.assert_array_equal(q_r[:1].view(np.int32), q64[:1].view(np.int32))
    assert np.all(np.isfinite(ph_r[0]))


def test_kernel_timing_names_the_chain_kernels(cuda):
    from moraine_b200 import _lib
    cfg = CONFIGS["c2"].scaled(nlines=48, width=48)
    z = make_stack(cfg, device=cuda)
    ch = DsChain(48, 48, cfg.nimages, cfg.az_half_win, cfg.r_half_win, cfg.p_max, 1, device=cuda,
                 precision="fp64", emi_precision="refine")
    ch.run(z)
    lib = _lib.load()
    lib.mr_set_kernel_timing(1)
    ch.run(z)
    torch.cuda.synchronize()
    kt = _lib.kernel_timing()
    lib.mr_set_kernel_timing(0)
    for name in ("ks sort keys", "ks merge", "gram fp64", "emi sweep fp64", "emi reduce fp32", "emi refine tail"):
        assert name in kt and kt[name][0] > 0 and kt[name][1] >= 1, (name, kt)


def test_chain_mixed_route(cuda):
    cfg = CONFIGS["c3"].scaled(nlines=24, width=24, nimages=64)
    z = make_stack(cfg, device=cuda)
    ch = DsChain(24, 24, cfg.nimages, cfg.az_half_win, cfg.r_half_win, cfg.p_max, 1, device=cuda,
                 emi_precision="mixed")
    res = ch.run(z)
    ref = DsChain(24, 24, cfg.nimages, cfg.az_half_win, cfg.r_half_win, cfg.p_max, 1, device=cuda).run(z)
    assert res.route is not None and res.route.shape == (res.n_ds,)
    keep = res.route == 0
    assert keep.any()
    assert torch.equal(res.ph[keep], ref.ph[keep])


def test_emi_edges(cuda):
    # N = 2 and N = 3 with exact coherence, reference image other than 0
    for n in (2, 3, 5):
        phi = np.linspace(0, 1, n)
        g = 0.7 * np.exp(1j * (phi[:, None] - phi[None, :]))
        np.fill_diagonal(g, 1)
        r, s = np.triu_indices(n, 1)
        coh = g[r, s][None].astype(np.complex64)
        for ref in range(n):
            ph, q = mb.emi(coh, ref=ref)
            ph_r, q_r, _, _ = O.emi(coh, ref=ref)
            np.testing.assert_allclose(ph, ph_r, atol=1e-6)
            np.testing.assert_allclose(q, q_r, rtol=1e-6)
    empty = mb.emi(np.zeros((0, 6), np.complex64))
    assert empty[0].shape == (0, 4)
    with pytest.raises(ValueError):
        mb.emi(np.zeros((3, 7), np.complex64))


def test_temp_coh_variants(cuda):
    rng = np.random.default_rng(9)
    n = 12
    coh = (rng.standard_normal((300, 66)) + 1j * rng.standard_normal((300, 66))).astype(np.complex64)
    ph = (rng.standard_normal((300, n)) + 1j * rng.standard_normal((300, n))).astype(np.complex64)
    np.testing.assert_allclose(mb.temp_coh(coh, ph), O.temp_coh(coh, ph), atol=2e-6)
    unit = ph / np.abs(ph)
    np.testing.assert_allclose(mb.ds_temp_coh(coh, unit), O.ds_temp_coh(coh, unit), atol=2e-6)
    pairs = mb.TempNet.from_bandwidth(n, 2).image_pairs
    c2 = coh[:, :pairs.shape[0]]
    np.testing.assert_allclose(mb.temp_coh(c2, ph, pairs), O.temp_coh(c2, ph, pairs), atol=2e-6)
    ras = mb.temp_coh(coh.reshape(15, 20, 66), ph.reshape(15, 20, n))
    assert ras.shape == (15, 20)
    # inputs are not modified
    c0 = coh.copy()
    mb.temp_coh(coh, ph)
    np.testing.assert_array_equal(coh, c0)


def test_torch_in_torch_out(cuda, golden):
    g = golden("co_small.npz")
    c = torch.from_numpy(g["coh"]).to(cuda)
    ph, q = mb.emi(c)
    assert isinstance(ph, torch.Tensor) and ph.is_cuda and ph.dtype == torch.complex64
    t = mb.ds_temp_coh(c, ph)
    assert t.is_cuda and t.dtype == torch.float32


# ----------------------------------------------------------------------------- chain
def test_fused_helper_equals_separate_calls(cuda, golden):
    g = golden("chain_small.npz")
    idx = g["idx"]
    pc = np.unpackbits(g["is_shp_bits"]).astype(bool).reshape(48, 48, 11, 11)[tuple(idx.T)]
    ph_f, q_f, t_f = mb.emperical_co_emi_temp_coh_pc(g["rslc"], idx, pc, batch_size=100)
    coh = mb.emperical_co_pc(g["rslc"], idx, pc)
    ph, q = mb.emi(coh)
    t = mb.ds_temp_coh(coh, ph)
    np.testing.assert_array_equal(ph_f, ph)
    np.testing.assert_array_equal(q_f, q)
    np.testing.assert_array_equal(t_f, t)


def test_device_chain_vs_reference_fixture(cuda, golden):
    g = golden("chain_small.npz")
    azh, rh = (int(v) for v in g["win"])
    ch = DsChain(48, 48, 17, azh, rh, p_max=float(g["p_max"]), min_shp=int(g["min_shp"]), batch=100)
    res = ch.run(torch.from_numpy(g["rslc"]).to(cuda))
    np.testing.assert_array_equal(np.packbits(res.is_shp.cpu().numpy().astype(bool).reshape(-1)), g["is_shp_bits"])
    np.testing.assert_array_equal(res.shp_num.cpu().numpy(), g["shp_num"])
    np.testing.assert_array_equal(res.idx.cpu().numpy(), g["idx"])
    coh = O.emperical_co_pc(g["rslc"], g["idx"], np.unpackbits(g["is_shp_bits"]).astype(bool).reshape(
        48, 48, 11, 11)[tuple(g["idx"].T)])
    _, _, gap, cond = O.emi(coh.astype(np.complex64))
    tol = O.phase_tolerance(cond, gap, eps=EPS_GRAM32)
    err = np.abs(np.angle(res.ph.cpu().numpy() * np.conj(g["ph"]))).max(-1)
    assert np.all(err <= tol), (err / tol).max()
    well = tol < 1e-3
    assert np.abs(res.t_coh.cpu().numpy() - g["t_coh"])[well].max(initial=0) < 1e-3


@pytest.mark.parametrize("name", ["chain_c1_n50", "chain_c2_n100"])
@pytest.mark.parametrize("emi", ["fp64", "refine"])
def test_device_chain_vs_reference_at_image_counts(cuda, golden, name, emi):
    """The device chain against the reference's own chain at the benchmark image counts
    (N = 50 and N = 100): masks and counts bit-exact, FP64 coherence, phases within the
    reference's complex64 EMI bound, temporal coherence of the reference phases."""
    g = golden(f"{name}.npz")
    rslc = g["rslc"]
    nl, w, n = rslc.shape
    azh, rh = (int(v) for v in g["win"])
    ch = DsChain(nl, w, n, azh, rh, p_max=float(g["p_max"]), min_shp=int(g["min_shp"]), precision="fp64",
                 emi_precision=emi)
    res = ch.run(torch.from_numpy(rslc).to(cuda))
    np.testing.assert_array_equal(np.packbits(res.is_shp.cpu().numpy().astype(bool).reshape(-1)), g["is_shp_bits"])
    np.testing.assert_array_equal(res.shp_num.cpu().numpy(), g["shp_num"])
    k = g["idx"].shape[0]
    np.testing.assert_array_equal(res.idx.cpu().numpy()[:k], g["idx"])
    is_shp = np.unpackbits(g["is_shp_bits"]).astype(bool).reshape(nl, w, 2 * azh + 1, 2 * rh + 1)
    pc = is_shp[tuple(g["idx"].T)]
    coh = mb.emperical_co_pc(rslc, g["idx"], pc, precision="fp64")
    np.testing.assert_allclose(coh[:8], g["coh_head"], atol=2e-7)
    _, _, gap, cond = O.emi(coh)
    tol = O.phase_tolerance(cond, gap, eps=4 * EPS32)
    err = np.abs(np.angle(res.ph.cpu().numpy()[:k] * np.conj(g["ph"]))).max(-1)
    assert np.all(err <= tol), (err / tol).max()
    np.testing.assert_allclose(mb.ds_temp_coh(coh, g["ph"]), g["t_coh"], atol=5e-5)


@pytest.mark.parametrize("name,size", [("c0", 200), ("c1", 96), ("c2", 96)])
def test_device_chain_vs_oracle(cuda, name, size):
    cfg = CONFIGS[name].scaled(nlines=size, width=size)
    z = make_stack(cfg)
    ref = O.chain(z.numpy(), cfg.az_half_win, cfg.r_half_win, cfg.p_max, cfg.min_shp)
    res = DsChain(size, size, cfg.nimages, cfg.az_half_win, cfg.r_half_win, cfg.p_max, cfg.min_shp,
                  batch=4096).run(z.to(cuda))
    np.testing.assert_array_equal(res.is_shp.cpu().numpy().astype(bool), ref["is_shp"])
    np.testing.assert_array_equal(res.shp_num.cpu().numpy(), ref["shp_num"])
    np.testing.assert_array_equal(res.idx.cpu().numpy(), ref["idx"])
    assert res.n_ds == len(ref["idx"])
    if res.n_ds == 0:
        return
    # coherence in FP32 vs FP64: the phase error budget scales with cond / gap
    tol = O.phase_tolerance(ref["cond"], ref["gap"], eps=EPS_GRAM32)
    err = np.abs(np.angle(res.ph.cpu().numpy() * np.conj(ref["ph"]))).max(-1)
    assert np.all(err <= tol), (err / tol).max()
    well = tol < 1e-3
    assert np.abs(res.t_coh.cpu().numpy() - ref["t_coh"])[well].max(initial=0) < 1e-3


@pytest.mark.parametrize("ks_input", ["intensity", "amplitude"])
def test_chain_ks_input_vs_oracle(cuda, ks_input):
    """The chain ranks |z|^2 or |z| as asked: SHP mask, counts and DS points bit-exact with the
    oracle chain on the same KS input, and the amplitude mask equal to ks_test on rslc2amp."""
    cfg = CONFIGS["c1"].scaled(nlines=80, width=80)
    z = make_stack(cfg)
    # range neighbours share four dates up to a phase rotation: |z| ties more often than |z|^2
    z[:, 1::2, :4] = z[:, 0:-1:2, :4] * torch.tensor(np.exp(0.7j), dtype=torch.complex64)
    ref = O.chain(z.numpy(), cfg.az_half_win, cfg.r_half_win, cfg.p_max, cfg.min_shp, ks_input=ks_input)
    res = DsChain(80, 80, cfg.nimages, cfg.az_half_win, cfg.r_half_win, cfg.p_max, cfg.min_shp, batch=4096,
                  ks_input=ks_input).run(z.to(cuda))
    np.testing.assert_array_equal(res.is_shp.cpu().numpy().astype(bool), ref["is_shp"])
    np.testing.assert_array_equal(res.shp_num.cpu().numpy(), ref["shp_num"])
    np.testing.assert_array_equal(res.idx.cpu().numpy(), ref["idx"])
    if ks_input == "amplitude":
        p = mb.ks_test(mb.rslc2amp(z.to(cuda)), cfg.az_half_win, cfg.r_half_win)
        is_shp, shp_num = mb.select_shp(p, cfg.p_max)
        assert torch.equal(is_shp.to(torch.uint8), res.is_shp) and torch.equal(shp_num.to(torch.int32), res.shp_num)
    with pytest.raises(ValueError):
        DsChain(8, 8, 10, 1, 1, ks_input="power", device=cuda)


@pytest.mark.parametrize("gram,emi,ks_input", [("fp32", "fp32", "intensity"), ("fp64", "fp64", "intensity"),
                                               ("fp64", "mixed", "intensity"), ("fp64", "fp64", "amplitude")])
def test_ds_chain_c_abi_equals_python_chain(cuda, gram, emi, ks_input):
    """mr_ds_chain (one C call for the whole chain) gives the DsChain results bit for bit."""
    import ctypes
    from moraine_b200 import _dev, _lib
    cfg = CONFIGS["c1"].scaled(nlines=72, width=64, n_patches=6)
    z = make_stack(cfg, device=cuda)
    ref = DsChain(72, 64, cfg.nimages, cfg.az_half_win, cfg.r_half_win, cfg.p_max, cfg.min_shp, precision=gram,
                  emi_precision=emi, device=cuda, ks_input=ks_input).run(z)
    lib = _lib.load()
    npix, n, batch = 72 * 64, cfg.nimages, 1000  # several batches
    ws = _dev.workspace(lib.mr_ds_chain_workspace_bytes(72, 64, n, cfg.az_half_win, cfg.r_half_win, batch) + 256,
                        cuda)
    base = (ws.data_ptr() + 255) & ~255
    idx = torch.empty((npix, 2), dtype=torch.int32, device=cuda)
    ph = torch.empty((npix, n), dtype=torch.complex64, device=cuda)
    q = torch.empty((npix,), dtype=torch.float32, device=cuda)
    t = torch.empty((npix,), dtype=torch.float32, device=cuda)
    n_ds = ctypes.c_int64(-1)
    args = [z.data_ptr(), 72, 64, n, cfg.az_half_win, cfg.r_half_win, _lib.KS_INPUT[ks_input], cfg.p_max,
            cfg.min_shp, _lib.PREC[gram],
            _lib.PREC[emi], idx.data_ptr(), ph.data_ptr(), q.data_ptr(), t.data_ptr(), npix, ctypes.addressof(n_ds),
            batch, base, ws.numel() - 256, _dev.stream()]
    _lib.call("mr_ds_chain", *args)
    d = n_ds.value
    assert d == ref.n_ds > batch
    assert torch.equal(idx[:d], ref.idx)
    assert torch.equal(ph[:d].view(torch.float32), ref.ph.view(torch.float32))
    assert torch.equal(q[:d].view(torch.int32), ref.quality.view(torch.int32))
    assert torch.equal(t[:d].view(torch.int32), ref.t_coh.view(torch.int32))
    small = list(args)
    small[15] = d - 1  # max_ds below the DS count
    with pytest.raises(ValueError):
        _lib.call("mr_ds_chain", *small)
    small = list(args)
    small[19] = 1024  # workspace too small
    with pytest.raises(MemoryError):
        _lib.call("mr_ds_chain", *small)
    small = list(args)
    small[6] = 2  # neither intensity nor amplitude
    with pytest.raises(ValueError):
        _lib.call("mr_ds_chain", *small)


def test_maximum_sizes(cuda):
    """The build's limits: N = 512 images through KS (bit-exact), coherence and EMI; the
    largest window (4096 cells) through KS; one past each limit is refused."""
    rng = np.random.default_rng(11)
    n = 512
    z = (rng.standard_normal((10, 9, n)) + 1j * rng.standard_normal((10, 9, n))).astype(np.complex64)
    z *= np.exp(1j * np.linspace(0, 3, n))[None, None, :].astype(np.complex64)
    rmli = O.intensity(z)
    p = mb.ks_test(rmli, 2, 2)
    np.testing.assert_array_equal(p, O.ks_test(rmli, 2, 2))
    idx = np.array([[4, 4], [5, 3], [2, 6]], np.int32)
    pc = np.ones((3, 5, 5), bool)
    coh = mb.emperical_co_pc(z, idx, pc, precision="fp64")
    ref = O.emperical_co_pc(z, idx, pc)
    np.testing.assert_allclose(coh, ref, atol=2e-7, rtol=0)
    ph, q = mb.emi(coh)
    ph_r, q_r, gap, cond = O.emi(coh)
    err = np.abs(np.angle(ph * np.conj(ph_r))).max(-1)
    assert np.all(err <= O.phase_tolerance(cond, gap, eps=1e3 * EPS64, floor=3e-7))
    with pytest.raises(NotImplementedError):
        mb.ks_test(np.ones((4, 4, n + 1), np.float32), 1, 1)
    # largest window: 63 x 65 = 4095 cells on a small raster
    x = rng.exponential(size=(70, 70, 9)).astype(np.float32)
    np.testing.assert_array_equal(mb.ks_test(x, 31, 32), O.ks_test(x, 31, 32))
    with pytest.raises(NotImplementedError):
        mb.ks_test(x, 32, 32)  # 65 x 65 = 4225 cells


@pytest.mark.parametrize("prec,emi_prec", [("fp32", None), ("fp64", None), ("fp64", "refine")])
def test_chain_in_cuda_graph(cuda, prec, emi_prec):
    """The chain captured once in a CUDA graph and replayed on two stacks equals the plain chain
    (the refined EMI too: its routing and FP64 recomputation read the DS count on the device)."""
    cfg = CONFIGS["c1"].scaled(nlines=64, width=72, n_patches=6)
    kw = dict(precision=prec, emi_precision=emi_prec, batch=900, device=cuda)
    plain = DsChain(64, 72, cfg.nimages, cfg.az_half_win, cfg.r_half_win, cfg.p_max, cfg.min_shp, **kw)
    graph = DsChain(64, 72, cfg.nimages, cfg.az_half_win, cfg.r_half_win, cfg.p_max, cfg.min_shp, graph=True, **kw)
    for seed in (5, 6):
        z = make_stack(cfg.scaled(seed=seed), device=cuda)
        a, b = plain.run(z), graph.run(z)
        assert b.n_ds == a.n_ds > 900
        assert torch.equal(b.idx, a.idx)
        assert torch.equal(b.ph.view(torch.float32), a.ph.view(torch.float32))
        assert torch.equal(b.quality.view(torch.int32), a.quality.view(torch.int32))
        assert torch.equal(b.t_coh.view(torch.int32), a.t_coh.view(torch.int32))
    with pytest.raises(ValueError):
        DsChain(8, 8, 200, 1, 1, graph=True, device=cuda)
    with pytest.raises(ValueError):
        DsChain(8, 8, 20, 1, 1, precision="fp64", emi_precision="mixed", graph=True, device=cuda)
    with pytest.raises(ValueError):
        DsChain(8, 8, 20, 1, 1, precision="fp64", emi_precision="refine", refine_tol=1e-3, graph=True, device=cuda)


def test_ks_autotune_same_results(cuda):
    """Tuned and heuristic KS tile plans give bit-identical p, masks and counts."""
    import ctypes
    from moraine_b200 import _lib
    lib = _lib.load()
    cfg = CONFIGS["c1"].scaled(nlines=90, width=70)
    z = make_stack(cfg)
    rmli = torch.from_numpy(O.intensity(z.numpy())).to(cuda)
    out = []
    try:
        for tune in (0, 1):
            lib.mr_set_autotune(tune)
            out.append(_fused_select(rmli, cfg.az_half_win, cfg.r_half_win))
        th, tw, azc = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        assert lib.mr_ks_plan(cfg.nimages, cfg.az_half_win, cfg.r_half_win, ctypes.byref(th), ctypes.byref(tw),
                              ctypes.byref(azc)) == 0
        assert th.value * tw.value >= 1 and 1 <= azc.value <= cfg.az_win
    finally:
        lib.mr_set_autotune(1)
    for a, b in zip(out[0], out[1]):
        np.testing.assert_array_equal(a, b)
