"""PS-side statistics (amplitude, amplitude dispersion, calibrated amplitude) against the reference."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.fixture(scope="module")
def g(golden):
    return golden("ps_small.npz")


def test_oracle_matches_reference(g):
    np.testing.assert_array_equal(O.rslc2amp(g["rslc"]), g["amp"])
    np.testing.assert_allclose(O.amp_disp(g["rslc"]), g["amp_disp"], rtol=1e-5, equal_nan=True)
    np.testing.assert_allclose(O.calamp(g["amp0"]), g["calamp"], rtol=1e-6, equal_nan=True)


@pytest.mark.gpu
def test_device_matches_reference(cuda, g):
    import moraine_b200 as mb
    amp = mb.rslc2amp(g["rslc"])
    assert amp.dtype == np.float32 and amp.shape == g["amp"].shape
    np.testing.assert_array_equal(amp.view(np.uint32), g["amp"].view(np.uint32))  # bit-exact |z|
    np.testing.assert_array_equal(mb.rslc2amp(g["rslc"][:, :, 0].copy()), g["amp"][:, :, 0])  # 2-D SLC
    ad = mb.amp_disp(g["rslc"])
    assert ad.dtype == np.float32 and ad.shape == g["amp_disp"].shape
    np.testing.assert_allclose(ad, g["amp_disp"], rtol=1e-5, equal_nan=True)
    np.testing.assert_array_equal(np.isnan(ad), np.isnan(g["amp_disp"]))
    np.testing.assert_allclose(mb.calamp(g["amp0"]), g["calamp"], rtol=1e-6, equal_nan=True)


@pytest.mark.gpu
def test_device_vs_oracle_larger(cuda):
    import moraine_b200 as mb
    from moraine_b200.synth import CONFIGS, make_stack
    z = make_stack(CONFIGS["c1"].scaled(nlines=96, width=80, n_patches=6)).numpy()
    np.testing.assert_array_equal(mb.rslc2amp(z), O.rslc2amp(z))
    np.testing.assert_allclose(mb.amp_disp(z), O.amp_disp(z), rtol=2e-6)
    a0 = O.rslc2amp(z[:, :, 0])
    np.testing.assert_allclose(mb.calamp(a0), O.calamp(a0), rtol=1e-6)
