"""Parity at full size: the 2000 x 2000 x 100 scene through the FP64 device chain.

The SHP masks and counts of the whole scene are compared bit for bit with the oracle's KS
selection (C, all host cores). The rest of the chain is too heavy for the oracle as a
whole, so the whole-scene result is also checked through properties that hold at any size
(KS symmetry, the centre always an SHP, counts equal to the masks, DS indices in row-major
order), and sampled DS points are checked against the oracle on the crop of their own
window, which holds everything their result depends on.
"""
import numpy as np
import pytest
import torch

import moraine_b200 as mb
from moraine_b200.chain import DsChain
from moraine_b200.synth import CONFIGS, make_stack
from oracle import oracle as O

pytestmark = pytest.mark.gpu

EPS64 = 1.2e-16


@pytest.fixture(scope="module")
def c2_full(cuda):
    cfg = CONFIGS["c2"]
    z = make_stack(cfg, device=cuda)
    chain = DsChain(cfg.nlines, cfg.width, cfg.nimages, cfg.az_half_win, cfg.r_half_win, cfg.p_max, cfg.min_shp,
                    precision="fp64", device=cuda)
    res = chain.run(z)
    torch.cuda.synchronize()
    return cfg, z, res


def test_fullsize_masks_bit_exact_vs_oracle(c2_full):
    cfg, z, res = c2_full
    rmli = O.intensity(z.cpu().numpy())
    is_shp, num = O.ks_select(rmli, cfg.az_half_win, cfg.r_half_win, cfg.p_max)
    np.testing.assert_array_equal(res.shp_num.cpu().numpy(), num)
    dev = res.is_shp.cpu().numpy().view(bool)
    assert np.array_equal(dev, is_shp), int(np.count_nonzero(dev != is_shp))


def test_fullsize_mask_properties(c2_full):
    cfg, z, res = c2_full
    m = res.is_shp
    azh, rh = cfg.az_half_win, cfg.r_half_win
    H, W = cfg.nlines, cfg.width
    assert bool((m[:, :, azh, rh] == 1).all())  # k = 0: p = 0 < p_max
    assert torch.equal(res.shp_num, m.sum((2, 3), dtype=torch.int32))
    # the two-sample KS statistic is symmetric: pixel x sees x + d as x + d sees x
    for da in range(-azh, azh + 1):
        for dr in range(-rh, rh + 1):
            a0, a1 = max(0, -da), H - max(0, da)
            r0, r1 = max(0, -dr), W - max(0, dr)
            fwd = m[a0:a1, r0:r1, azh + da, rh + dr]
            bwd = m[a0 + da:a1 + da, r0 + dr:r1 + dr, azh - da, rh - dr]
            assert torch.equal(fwd, bwd), (da, dr)
    # DS points: SHP count >= min_shp, row-major order, all of them
    idx = res.idx.long()
    lin = idx[:, 0] * W + idx[:, 1]
    assert res.n_ds == int((res.shp_num >= cfg.min_shp).sum())
    assert bool((lin[1:] > lin[:-1]).all())
    assert bool((res.shp_num[idx[:, 0], idx[:, 1]] >= cfg.min_shp).all())
    assert bool(torch.isfinite(res.quality).all()) and bool(((res.t_coh >= 0) & (res.t_coh <= 1 + 1e-6)).all())


def test_fullsize_sampled_points_vs_oracle(c2_full):
    cfg, z, res = c2_full
    azh, rh = cfg.az_half_win, cfg.r_half_win
    idx = res.idx.long().cpu()
    inner = ((idx[:, 0] >= azh) & (idx[:, 0] < cfg.nlines - azh) & (idx[:, 1] >= rh) & (idx[:, 1] < cfg.width - rh))
    cand = inner.nonzero().squeeze(1)
    g = torch.Generator().manual_seed(7)
    sel = cand[torch.randperm(cand.numel(), generator=g)[:48]]
    coh_dev, masks = [], []
    for k in sel.tolist():
        a, r = int(idx[k, 0]), int(idx[k, 1])
        crop = z[a - azh:a + azh + 1, r - rh:r + rh + 1].cpu().numpy()
        p = O.ks_test(O.intensity(crop), azh, rh)
        is_shp, _ = O.select_shp(p, cfg.p_max)
        centre = is_shp[azh, rh]
        np.testing.assert_array_equal(centre.astype(np.uint8), res.is_shp[a, r].cpu().numpy())  # bit-exact mask
        masks.append(centre)
        c_ref = O.emperical_co_pc(crop, np.array([[azh, rh]], np.int32), centre[None])
        c_dev = mb.emperical_co_pc(z, idx[k:k + 1].int().to(z.device), res.is_shp[a:a + 1, r].bool(),
                                   precision="fp64")
        np.testing.assert_allclose(c_dev.cpu().numpy()[0], c_ref[0], atol=2e-7, rtol=0)
        coh_dev.append(c_dev.cpu().numpy()[0])
    coh = np.stack(coh_dev)
    ph_r, q_r, gap, cond = O.emi(coh)
    ph = res.ph[sel.to(res.ph.device)].cpu().numpy()
    err = np.abs(np.angle(ph * np.conj(ph_r))).max(-1)
    tol = O.phase_tolerance(cond, gap, eps=1e3 * EPS64, floor=3e-7)
    assert np.all(err <= tol), (err / tol).max()
    t_ref = O.ds_temp_coh(coh, ph)
    np.testing.assert_allclose(res.t_coh[sel.to(res.t_coh.device)].cpu().numpy(), t_ref, atol=1e-6)
