"""GAMMA raster ingest: the oracle and the device decode against the reference's reader."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

TYPES = ("float", "fcomplex", "int", "double")


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view({4: np.uint32, 8: np.uint64, 16: np.uint64}[a.dtype.itemsize])


def _write(tmp_path, golden_gamma, dtype):
    f = tmp_path / f"img.{dtype}"
    golden_gamma[f"{dtype}_raw"].tofile(f)
    return f


@pytest.fixture(scope="module")
def golden_gamma(golden):
    return golden("gamma_small.npz")


@pytest.mark.parametrize("dtype", TYPES)
def test_oracle_matches_reference_reader(tmp_path, golden_gamma, dtype):
    f = _write(tmp_path, golden_gamma, dtype)
    width = int(golden_gamma["shape"][1])
    np.testing.assert_array_equal(_bits(O.read_gamma_image(f, width, dtype)), _bits(golden_gamma[f"{dtype}_all"]))
    np.testing.assert_array_equal(_bits(O.read_gamma_image(f, width, dtype, y0=3, ny=5)),
                                  _bits(golden_gamma[f"{dtype}_y3_n5"]))


def test_unsupported_dtype():
    from moraine_b200.gamma_ import read_gamma_image
    with pytest.raises(ValueError, match="Unsupported"):
        read_gamma_image("nonexistent", 10, "short")


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", TYPES)
def test_device_decode_bit_exact(cuda, tmp_path, golden_gamma, dtype):
    from moraine_b200.gamma_ import read_gamma_image
    f = _write(tmp_path, golden_gamma, dtype)
    width = int(golden_gamma["shape"][1])
    got = read_gamma_image(str(f), width, dtype).cpu().numpy()
    np.testing.assert_array_equal(_bits(got), _bits(golden_gamma[f"{dtype}_all"]))
    got = read_gamma_image(str(f), width, dtype, y0=3, ny=5).cpu().numpy()
    np.testing.assert_array_equal(_bits(got), _bits(golden_gamma[f"{dtype}_y3_n5"]))
    with pytest.raises(AssertionError):
        read_gamma_image(str(f), width, dtype, y0=50)
    with pytest.raises(AssertionError):
        read_gamma_image(str(f), width, dtype, y0=8, ny=5)


@pytest.mark.gpu
def test_pdata_and_stack(cuda, tmp_path):
    from moraine_b200.gamma_ import read_gamma_image, read_gamma_pdata, read_gamma_stack
    rng = np.random.default_rng(3)
    width, nl, nd = 37, 23, 5
    paths = []
    for d in range(nd):
        z = (rng.standard_normal((nl, width)) + 1j * rng.standard_normal((nl, width))).astype(np.complex64)
        z[d, :3] = 0  # no-data samples
        p = tmp_path / f"d{d}.rslc"
        z.astype(">c8").tofile(p)
        paths.append(str(p))
    st = read_gamma_stack(paths, width, "fcomplex", y0=2, ny=17)
    assert st.shape == (17, width, nd) and st.dtype == torch.complex64
    for d in range(nd):
        one = read_gamma_image(paths[d], width, "fcomplex", y0=2, ny=17)
        ref = O.read_gamma_image(paths[d], width, "fcomplex", y0=2, ny=17)
        np.testing.assert_array_equal(_bits(st[:, :, d].cpu().numpy().copy()), _bits(one.cpu().numpy()))
        np.testing.assert_array_equal(_bits(one.cpu().numpy()), _bits(ref))
    q = tmp_path / "pt.float"
    v = rng.standard_normal(1001).astype(np.float32)
    v[7] = 0
    v.astype(">f4").tofile(q)
    got = read_gamma_pdata(str(q), "float").cpu().numpy()
    np.testing.assert_array_equal(_bits(got), _bits(O.gamma_decode(v.astype(">f4").tobytes(), "float")))
    assert np.isnan(got[7])
