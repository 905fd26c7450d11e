"""The seeded scene generator."""
import numpy as np
import torch

from moraine_b200.synth import CONFIGS, make_stack, rmli_of


def test_deterministic_and_shaped():
    cfg = CONFIGS["c0"].scaled(nlines=32, width=40)
    a = make_stack(cfg)
    b = make_stack(cfg)
    assert a.shape == (32, 40, 17) and a.dtype == torch.complex64
    assert torch.equal(a, b)
    c = make_stack(cfg.scaled(seed=5))
    assert not torch.equal(a, c)


def test_patch_statistics():
    cfg = CONFIGS["c0"].scaled(nlines=64, width=64, ps_frac=0.0)
    z, truth = make_stack(cfg, return_truth=True)
    lab = truth["labels"].numpy()
    inten = truth["intensity"].numpy()
    zz = z.numpy()
    for p in np.unique(lab):
        sel = lab == p
        if sel.sum() < 200:
            continue
        m = (np.abs(zz[sel]) ** 2).mean()
        assert abs(m / inten[p] - 1) < 0.15


def test_rmli_rounding():
    z = make_stack(CONFIGS["c0"].scaled(nlines=8, width=8))
    r = rmli_of(z).numpy()
    zn = z.numpy()
    re, im = zn.real.astype(np.float32), zn.imag.astype(np.float32)
    np.testing.assert_array_equal(r, (re * re) + (im * im))
