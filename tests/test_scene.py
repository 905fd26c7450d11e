"""Scenes in halo tiles: the tiling against the reference's own slices, the streaming loop
against a whole-scene run (CPU stand-in chain), and the device chain bit for bit (GPU)."""
import types

import numpy as np
import pytest
import torch

from moraine_b200.scene import ArraySource, GammaSource, SceneRunner, chunk_slices
from oracle import oracle as O


def test_chunk_slices_match_reference(golden):
    """moraine/chunk_.py chunkwise_slicing_mapping / all_chunk_slices_with_overlap on seven cases
    (whole-axis chunks, chunks beyond the scene, zero depth, depth beyond the chunk, 3-D)."""
    g = golden("chunk_small.npz")
    k = 0
    while f"case{k}" in g:
        shape, chunks, depths = (tuple(int(v) for v in r) for r in g[f"case{k}"])
        tiles = chunk_slices(shape, chunks, depths)
        got = {name: np.array([[list(ax) for ax in getattr(t, name)] for t in tiles]) for name in ("read", "own",
                                                                                                   "inner")}
        np.testing.assert_array_equal(got["read"], g[f"in{k}"])
        np.testing.assert_array_equal(got["read"], g[f"overlap{k}"])
        np.testing.assert_array_equal(got["own"], g[f"out{k}"])
        np.testing.assert_array_equal(got["inner"], g[f"map{k}"])
        k += 1
    assert k == 7
    with pytest.raises(ValueError):
        chunk_slices((10, 10), (0, 5), (1, 1))


class FakeChain:
    """A windowed stand-in for DsChain on the CPU. A neighbour counts when both series are free
    of NaN, it lies inside the stack and its mean amplitude is within half of the pixel's (NaN
    samples and pixels outside the stack never count, as in the KS test); pixels with at least
    min_shp such neighbours are DS points, their phase series is the sum of those neighbours'."""

    def __init__(self, ty, tx, n, azh, rh, min_shp):
        self.shape, self.azh, self.rh, self.min_shp = (ty, tx, n), azh, rh, min_shp
        self.device = torch.device("cpu")
        self.calls = 0

    def run(self, z, own=None):
        self.calls += 1
        z = z.numpy()
        ty, tx, n = z.shape
        azh, rh = self.azh, self.rh
        a = np.abs(z).astype(np.float64)
        valid = ~np.isnan(a).any(-1)
        m = np.where(valid, a.mean(-1), np.nan)
        zp = np.full((ty + 2 * azh, tx + 2 * rh, n), np.nan, np.complex128)
        zp[azh:azh + ty, rh:rh + tx] = z
        mp = np.full((ty + 2 * azh, tx + 2 * rh), np.nan)
        mp[azh:azh + ty, rh:rh + tx] = m
        cnt = np.zeros((ty, tx), np.int32)
        acc = np.zeros((ty, tx, n), np.complex128)
        for da in range(2 * azh + 1):
            for dr in range(2 * rh + 1):
                nm = mp[da:da + ty, dr:dr + tx]
                sim = (np.abs(m - nm) < 0.5 * m) & ~np.isnan(nm) & valid
                cnt += sim
                acc += np.where(sim[..., None], zp[da:da + ty, dr:dr + tx], 0)
        l0, l1, p0, p1 = own if own is not None else (0, ty, 0, tx)
        ds = np.zeros((ty, tx), bool)
        ds[l0:l1, p0:p1] = cnt[l0:l1, p0:p1] >= self.min_shp
        idx = np.stack(np.nonzero(ds), -1).astype(np.int32)
        ph = acc[ds].astype(np.complex64)
        t = torch.from_numpy
        return types.SimpleNamespace(n_ds=len(idx), idx=t(idx), ph=t(ph), quality=t(cnt[ds].astype(np.float32)),
                                     t_coh=t(m[ds].astype(np.float32)), shp_num=t(cnt))


def _scene(nl=37, w=29, n=6, seed=0):
    rng = np.random.default_rng(seed)
    z = (rng.standard_normal((nl, w, n)) + 1j * rng.standard_normal((nl, w, n))).astype(np.complex64)
    z *= (1 + 3 * (np.arange(nl)[:, None, None] > nl // 2)).astype(np.float32)  # two amplitude regions
    z[4, 5, 2] = np.nan
    z[20, :, 0] = np.nan
    return z


@pytest.mark.parametrize("chunks,azh,rh", [((7, 9), 2, 3), ((-1, 5), 2, 3), ((100, 100), 1, 1), ((2, 3), 3, 4),
                                           ((11, -1), 0, 2)])
def test_stream_equals_whole_scene(chunks, azh, rh):
    z = _scene()
    nl, w, n = z.shape
    ms = max(2, (2 * azh + 1) * (2 * rh + 1) // 3)
    whole = FakeChain(nl, w, n, azh, rh, ms).run(torch.from_numpy(z))
    runner = SceneRunner(z.shape, azh, rh, chunks=chunks, device="cpu",
                         chain_factory=lambda ty, tx, nn: FakeChain(ty, tx, nn, azh, rh, ms))
    res = runner.run(ArraySource(z))
    assert res.n_ds == whole.n_ds > 0
    assert runner.chain.calls == len(runner.tiles)
    np.testing.assert_array_equal(res.idx, whole.idx.numpy())
    np.testing.assert_array_equal(res.ph.view(np.uint32), whole.ph.numpy().view(np.uint32))
    np.testing.assert_array_equal(res.quality, whole.quality.numpy())
    np.testing.assert_array_equal(res.t_coh.view(np.uint32), whole.t_coh.numpy().view(np.uint32))
    np.testing.assert_array_equal(res.shp_num, whole.shp_num.numpy())
    assert res.stats["tiles"] == len(runner.tiles)


@pytest.mark.parametrize("chunks", [(7, 9), (5, -1), (100, 100)])
def test_sink_gets_chunk_rows_in_scene_order(chunks):
    """With a sink, each chunk row's results arrive in scene order and together equal the
    whole-scene run; nothing is gathered."""
    z = _scene()
    azh, rh, ms = 2, 3, 11
    whole = FakeChain(*z.shape, azh, rh, ms).run(torch.from_numpy(z))
    runner = SceneRunner(z.shape, azh, rh, chunks=chunks, device="cpu",
                         chain_factory=lambda ty, tx, n: FakeChain(ty, tx, n, azh, rh, ms))
    rows = []
    res = runner.run(ArraySource(z), sink=rows.append)
    assert res.idx is None and res.n_ds == whole.n_ds > 0
    assert rows[0].lines[0] == 0 and rows[-1].lines[1] == z.shape[0]
    assert all(a.lines[1] == b.lines[0] for a, b in zip(rows[:-1], rows[1:]))
    np.testing.assert_array_equal(np.concatenate([r.idx for r in rows]), whole.idx.numpy())
    np.testing.assert_array_equal(np.concatenate([r.ph for r in rows]).view(np.uint32),
                                  whole.ph.numpy().view(np.uint32))
    np.testing.assert_array_equal(np.concatenate([r.quality for r in rows]), whole.quality.numpy())
    np.testing.assert_array_equal(np.concatenate([r.shp_num for r in rows]), whole.shp_num.numpy())
    for r in rows:
        assert ((r.idx[:, 0] >= r.lines[0]) & (r.idx[:, 0] < r.lines[1])).all()


def _band_rank(rank, world, port, out_path):
    """One rank of a two-rank gloo run: its azimuth band (moraine_b200.shard) streamed in halo
    tiles, the DS points of the lines it owns gathered to rank 0 and compared with the whole
    scene."""
    import os

    import torch.distributed as dist

    from moraine_b200.shard import band_partition, owned, to_scene
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        z = _scene()
        azh, rh, ms = 2, 3, 11
        band = band_partition(z.shape[0], world, azh)[rank]
        zb = np.ascontiguousarray(z[band.read0:band.read1])
        runner = SceneRunner(zb.shape, azh, rh, chunks=(6, 10), device="cpu",
                             chain_factory=lambda ty, tx, n: FakeChain(ty, tx, n, azh, rh, ms))
        res = runner.run(ArraySource(zb))
        keep = owned(torch.from_numpy(res.idx), band).numpy()
        part = (to_scene(torch.from_numpy(res.idx[keep]), band).numpy(), res.ph[keep], res.quality[keep])
        parts = [None] * world
        dist.all_gather_object(parts, part)  # result collection only: no exchange on the data path
        if rank == 0:
            whole = FakeChain(*z.shape, azh, rh, ms).run(torch.from_numpy(z))
            np.testing.assert_array_equal(np.concatenate([q[0] for q in parts]), whole.idx.numpy())
            np.testing.assert_array_equal(np.concatenate([q[1] for q in parts]).view(np.uint32),
                                          whole.ph.numpy().view(np.uint32))
            np.testing.assert_array_equal(np.concatenate([q[2] for q in parts]), whole.quality.numpy())
            with open(out_path, "w") as f:
                f.write(f"ok {whole.n_ds}")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_stream_their_bands(tmp_path):
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    out = tmp_path / "ok.txt"
    mp.start_processes(_band_rank, args=(2, port, str(out)), nprocs=2, join=True, start_method="spawn")
    assert out.read_text().startswith("ok ")


def test_sources_check_shapes(tmp_path):
    z = _scene()
    with pytest.raises(ValueError):
        ArraySource(z[..., 0])
    with pytest.raises(ValueError):
        ArraySource(z.astype(np.complex128))
    runner = SceneRunner((10, 10, 6), 1, 1, device="cpu", chain_factory=lambda *a: FakeChain(*a, 1, 1, 3))
    with pytest.raises(ValueError):
        runner.run(ArraySource(z))
    a, b = tmp_path / "a.rslc", tmp_path / "b.rslc"
    z[:, :, 0].astype(">c8").tofile(a)
    z[:-1, :, 1].astype(">c8").tofile(b)
    with pytest.raises(ValueError):
        GammaSource([str(a), str(b)], z.shape[1])


def test_gamma_source_staging(tmp_path):
    """Tiles staged from GAMMA files (big-endian, padded with NaN) decode to the reference
    reader's lines and pixels."""
    z = _scene(nl=21, w=17, n=4, seed=3)
    z[2, 3, 1] = 1e-31  # below the no-data threshold
    paths = []
    for d in range(z.shape[2]):
        p = tmp_path / f"d{d}.rslc"
        z[:, :, d].astype(">c8").tofile(p)
        paths.append(str(p))
    src = GammaSource(paths, z.shape[1])
    assert src.shape == z.shape
    host = src.alloc_host(9, 8, pin=False)
    src.stage((1, 8), (10, 17), host)  # a 7 x 7 tile padded to 9 x 8
    raw = host.numpy()
    for d, p in enumerate(paths):
        got = O.gamma_decode(raw[d].tobytes(), "fcomplex").reshape(9, 8)
        ref = O.read_gamma_image(p, z.shape[1], "fcomplex", y0=1, ny=7)[:, 10:17]
        np.testing.assert_array_equal(got[:7, :7].view(np.uint64), np.ascontiguousarray(ref).view(np.uint64))
        assert np.isnan(got[7:]).all() and np.isnan(got[:7, 7:]).all()


# ----------------------------------------------------------------------------- device
def _whole_and_stack(cuda, ks_input="intensity", emi_precision=None):
    from moraine_b200.chain import DsChain
    from moraine_b200.synth import CONFIGS, make_stack
    cfg = CONFIGS["c1"].scaled(nlines=150, width=130, n_patches=8)
    z = make_stack(cfg).numpy()
    whole = DsChain(150, 130, cfg.nimages, cfg.az_half_win, cfg.r_half_win, cfg.p_max, cfg.min_shp,
                    precision="fp64", emi_precision=emi_precision, ks_input=ks_input,
                    device=cuda).run(torch.from_numpy(z).to(cuda))
    return cfg, z, whole


def _assert_same(res, whole):
    assert res.n_ds == whole.n_ds > 0
    np.testing.assert_array_equal(res.idx, whole.idx.cpu().numpy())
    np.testing.assert_array_equal(res.ph.view(np.uint32), whole.ph.cpu().numpy().view(np.uint32))
    np.testing.assert_array_equal(res.quality.view(np.uint32), whole.quality.cpu().numpy().view(np.uint32))
    np.testing.assert_array_equal(res.t_coh.view(np.uint32), whole.t_coh.cpu().numpy().view(np.uint32))
    np.testing.assert_array_equal(res.shp_num, whole.shp_num.cpu().numpy())


@pytest.mark.gpu
@pytest.mark.parametrize("chunks,ks_input,emi", [((40, 48), "intensity", None), ((64, -1), "amplitude", "mixed"),
                                                 ((13, 130), "intensity", None)])
def test_device_stream_equals_whole_scene(cuda, chunks, ks_input, emi):
    """Halo tiles (NaN-padded at the border, DS points from the chunk only) give the
    whole-scene chain's results bit for bit, in its order."""
    cfg, z, whole = _whole_and_stack(cuda, ks_input, emi)
    runner = SceneRunner(z.shape, cfg.az_half_win, cfg.r_half_win, chunks=chunks, p_max=cfg.p_max,
                         min_shp=cfg.min_shp, precision="fp64", emi_precision=emi, ks_input=ks_input, device=cuda)
    assert len(runner.tiles) > 1
    _assert_same(runner.run(ArraySource(z)), whole)
    rows = []
    runner.run(ArraySource(z), sink=rows.append)  # chunk rows handed over one by one
    from types import SimpleNamespace
    cat = SimpleNamespace(n_ds=sum(len(r.idx) for r in rows), shp_num=np.concatenate([r.shp_num for r in rows]),
                          **{k: np.concatenate([getattr(r, k) for r in rows]) for k in ("idx", "ph", "quality",
                                                                                          "t_coh")})
    _assert_same(cat, whole)


@pytest.mark.gpu
def test_device_stream_from_memmap_and_gamma(cuda, tmp_path):
    """The same scene streamed from a memory-mapped .npy file and from GAMMA files per date."""
    cfg, z, whole = _whole_and_stack(cuda)
    np.save(tmp_path / "stack.npy", z)
    mm = np.load(tmp_path / "stack.npy", mmap_mode="r")
    kw = dict(p_max=cfg.p_max, min_shp=cfg.min_shp, precision="fp64", device=cuda)
    runner = SceneRunner(z.shape, cfg.az_half_win, cfg.r_half_win, chunks=(50, 70), **kw)
    _assert_same(runner.run(ArraySource(mm)), whole)
    paths = []
    for d in range(z.shape[2]):
        p = tmp_path / f"d{d}.rslc"
        z[:, :, d].astype(">c8").tofile(p)
        paths.append(str(p))
    _assert_same(runner.run(GammaSource(paths, z.shape[1])), whole)


def test_chunk_slices_properties():
    """For any scene, chunk size and depth: the chunks tile the scene exactly, each tile reads
    its chunk plus the depth on both sides clipped to the scene, and ``inner`` locates the
    chunk inside what is read."""
    from hypothesis import given, settings
    from hypothesis import strategies as st

    @settings(max_examples=200, deadline=None)
    @given(st.integers(1, 60), st.integers(1, 60), st.integers(-1, 70), st.integers(-1, 70), st.integers(0, 12),
           st.integers(0, 12))
    def check(nl, w, cl, cw, dl, dw):
        if cl == 0 or cw == 0:
            return
        tiles = chunk_slices((nl, w), (cl, cw), (dl, dw))
        cover = np.zeros((nl, w), np.int32)
        for t in tiles:
            (o0, o1), (p0, p1) = t.own
            cover[o0:o1, p0:p1] += 1
            for (r0, r1), (a0, a1), (i0, i1), n, d in zip(t.read, t.own, t.inner, (nl, w), (dl, dw)):
                assert (r0, r1) == (max(a0 - d, 0), min(a1 + d, n))
                assert (i0, i1) == (a0 - r0, a1 - r0)
        assert (cover == 1).all()
        # row-major over the chunk grid: chunk rows in order, chunks left to right within a row
        keys = [(t.own[0][0], t.own[1][0]) for t in tiles]
        assert keys == sorted(keys)

    check()
