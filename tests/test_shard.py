"""Azimuth-band sharding: partition logic, a two-rank gloo run on the CPU, bands on one GPU."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from moraine_b200.shard import band_partition, owned, to_scene

AZH, RH, N, MIN_SHP = 3, 4, 12, 20


def _scene():
    from moraine_b200.synth import CONFIGS, make_stack
    cfg = CONFIGS["c0"].scaled(nlines=41, width=30, nimages=N, az_half_win=AZH, r_half_win=RH, n_patches=5, seed=21)
    return make_stack(cfg).numpy()


def _oracle_band(z):
    from oracle import oracle as O
    p = O.ks_test(O.intensity(z), AZH, RH, nthreads=1)
    is_shp, num = O.select_shp(p, 0.05)
    idx, pc = O.ds_candidates(is_shp, num, MIN_SHP)
    coh = O.emperical_co_pc(z, idx, pc, nthreads=1) if len(idx) else np.zeros((0, N * (N - 1) // 2))
    return idx, pc, coh


@pytest.mark.parametrize("nlines,world,h", [(41, 2, 3), (10, 3, 5), (7, 7, 2), (100, 8, 7), (5, 1, 3)])
def test_band_partition(nlines, world, h):
    bands = band_partition(nlines, world, h)
    assert len(bands) == world
    assert bands[0].own0 == 0 and bands[-1].own1 == nlines
    for a, b in zip(bands[:-1], bands[1:]):
        assert a.own1 == b.own0
    for b in bands:
        assert b.read0 == max(0, b.own0 - h) and b.read1 == min(nlines, b.own1 + h)
        assert b.read0 <= b.own0 <= b.own1 <= b.read1
    with pytest.raises(ValueError):
        band_partition(0, 2, 1)


def test_owned_and_to_scene():
    b = band_partition(20, 2, 3)[1]  # owns [10, 20), reads [7, 20)
    idx = torch.tensor([[0, 1], [2, 5], [3, 0], [12, 4]], dtype=torch.int32)
    m = owned(idx, b)
    assert m.tolist() == [False, False, True, True]
    assert to_scene(idx[m], b).tolist() == [[10, 0], [19, 4]]


def _rank_main(rank, world, port, out_path):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        z = _scene()
        band = band_partition(z.shape[0], world, AZH)[rank]
        idx, pc, coh = _oracle_band(np.ascontiguousarray(z[band.read0:band.read1]))
        keep = owned(torch.from_numpy(idx), band).numpy()
        part = (to_scene(torch.from_numpy(idx[keep]), band).numpy(), pc[keep], coh[keep])
        parts = [None] * world
        dist.all_gather_object(parts, part)  # result collection only: no exchange on the data path
        if rank == 0:
            idx_all = np.concatenate([p[0] for p in parts])
            pc_all = np.concatenate([p[1] for p in parts])
            coh_all = np.concatenate([p[2] for p in parts])
            ref_idx, ref_pc, ref_coh = _oracle_band(z)
            assert len(ref_idx) > 0
            np.testing.assert_array_equal(idx_all, ref_idx)
            np.testing.assert_array_equal(pc_all, ref_pc)
            np.testing.assert_array_equal(coh_all, ref_coh)
            with open(out_path, "w") as f:
                f.write(f"ok {len(ref_idx)}")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_equal_whole_scene(tmp_path):
    out = tmp_path / "ok.txt"
    mp.start_processes(_rank_main, args=(2, _free_port(), str(out)), nprocs=2, join=True, start_method="spawn")
    assert out.read_text().startswith("ok ")


@pytest.mark.gpu
def test_bands_on_device_equal_whole_scene(cuda):
    from moraine_b200.chain import DsChain
    from moraine_b200.shard import run_band
    z = torch.from_numpy(_scene()).to(cuda)

    def factory(nl, w, n):
        return DsChain(nl, w, n, AZH, RH, 0.05, MIN_SHP, device=cuda)

    whole = factory(*z.shape).run(z)
    parts = [run_band(factory, z[b.read0:b.read1].contiguous(), b) for b in band_partition(z.shape[0], 3, AZH)]
    idx = torch.cat([p[0] for p in parts])
    assert whole.n_ds > 0 and torch.equal(idx, whole.idx)
    for k, ref in ((1, whole.ph), (2, whole.quality), (3, whole.t_coh)):
        got = torch.cat([p[k] for p in parts])
        assert torch.equal(got.view(torch.int32) if got.dtype == torch.float32 else got.view(torch.float32),
                           ref.view(torch.int32) if ref.dtype == torch.float32 else ref.view(torch.float32))
