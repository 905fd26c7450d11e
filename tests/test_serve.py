"""Tile serving: admission, concurrency and result independence from the mix."""
import threading
import time

import numpy as np
import pytest
import torch

from moraine_b200.serve import DsServer, TileRequest, latency_summary


def _fake_runner(log, lock, hold=0.05):
    def run(req, slot):
        with lock:
            log.append(("start", req.request_id, slot))
        time.sleep(hold)
        with lock:
            log.append(("end", req.request_id, slot))
        n = int(req.rslc.shape[0])
        return {"n_ds": n, "idx": torch.zeros((n, 2), dtype=torch.int32), "ph": torch.zeros((n, 1)),
                "quality": torch.zeros(n), "t_coh": torch.zeros(n)}
    return run


def _req(i, rows=4):
    return TileRequest(rslc=torch.zeros((rows, 1, 1), dtype=torch.complex64), request_id=i)


def test_admission_respects_budget_and_slots():
    log, lock = [], threading.Lock()
    sizes = {i: s for i, s in enumerate([40, 30, 50, 20, 60, 10, 30, 70])}
    srv = DsServer(hbm_budget=100, slots=3, runner=_fake_runner(log, lock),
                   footprint_fn=lambda r: sizes[r.request_id])
    futs = [srv.submit(_req(i)) for i in sizes]
    res = [f.result(timeout=30) for f in futs]
    srv.close()
    assert [r.request_id for r in res] == list(sizes)
    assert srv.peak_used <= 100 and srv.used == 0
    assert srv.peak_active <= 3 and srv.active == 0
    # replay the log: at no time do running tiles exceed the budget or the slots
    running, used = set(), 0
    for ev, rid, _ in log:
        if ev == "start":
            running.add(rid)
            used += sizes[rid]
            assert used <= 100 and len(running) <= 3
        else:
            running.remove(rid)
            used -= sizes[rid]
    # arrival order of admission
    assert srv.admitted_order == list(sizes)


def test_tiles_overlap_when_they_fit():
    log, lock = [], threading.Lock()
    srv = DsServer(hbm_budget=1000, slots=4, runner=_fake_runner(log, lock, hold=0.2), footprint_fn=lambda r: 10)
    t0 = time.perf_counter()
    futs = [srv.submit(_req(i)) for i in range(4)]
    for f in futs:
        f.result(timeout=30)
    dt = time.perf_counter() - t0
    srv.close()
    assert srv.peak_active == 4
    assert dt < 0.6  # four 0.2 s tiles side by side, not one after another


def test_late_arrival_is_admitted_while_others_run():
    log, lock = [], threading.Lock()
    srv = DsServer(hbm_budget=1000, slots=2, runner=_fake_runner(log, lock, hold=0.3), footprint_fn=lambda r: 10)
    f0 = srv.submit(_req(0))
    time.sleep(0.1)
    f1 = srv.submit(_req(1))  # arrives while tile 0 is on the device
    r0, r1 = f0.result(timeout=30), f1.result(timeout=30)
    srv.close()
    assert r1.admitted < r0.done  # started before tile 0 finished
    starts = [e for e in log if e[0] == "start"]
    assert [e[1] for e in starts] == [0, 1]


def test_oversize_request_is_rejected_and_errors_propagate():
    def boom(req, slot):
        raise ValueError("bad tile")

    srv = DsServer(hbm_budget=50, slots=1, runner=boom, footprint_fn=lambda r: 10 * r.request_id)
    with pytest.raises(MemoryError):
        srv.submit(_req(6))
    f = srv.submit(_req(1))
    with pytest.raises(ValueError, match="bad tile"):
        f.result(timeout=30)
    assert srv.used == 0
    srv.close()
    with pytest.raises(RuntimeError):
        srv.submit(_req(1))


def test_latency_summary():
    class R:
        def __init__(self, a, d, n):
            self.arrival, self.done, self.n_ds = a, d, n

        @property
        def latency(self):
            return self.done - self.arrival

    rs = [R(0.0, 0.1 * (i + 1), 10) for i in range(100)]
    s = latency_summary(rs)
    assert s["requests"] == 100 and s["n_ds"] == 1000
    assert s["p50_ms"] == pytest.approx(np.percentile(np.arange(1, 101) * 100.0, 50))
    assert s["p99_ms"] == pytest.approx(np.percentile(np.arange(1, 101) * 100.0, 99))


# ------------------------------------------------------------------ on the GPU
MIX = [  # (size, nimages, az_half_win, r_half_win, seed)
    (96, 20, 5, 5, 11),
    (128, 50, 5, 10, 12),
    (64, 17, 7, 15, 13),
    (112, 30, 5, 5, 14),
    (80, 100, 5, 10, 15),
]


def _mix_requests():
    from moraine_b200.synth import CONFIGS, make_stack
    reqs = []
    for i, (s, n, azh, rh, seed) in enumerate(MIX):
        cfg = CONFIGS["c0"].scaled(nlines=s, width=s, nimages=n, az_half_win=azh, r_half_win=rh, seed=seed,
                                   n_patches=6)
        reqs.append(TileRequest(rslc=make_stack(cfg).pin_memory(), az_half_win=azh, r_half_win=rh, min_shp=20,
                                request_id=i))
    return reqs


@pytest.mark.gpu
def test_results_same_alone_and_in_mix(cuda):
    reqs = _mix_requests()
    with DsServer(hbm_budget=8e9, slots=1) as srv:  # one tile at a time
        alone = {r.request_id: r for r in (srv.submit(q).result(timeout=300) for q in reqs)}
    for q in reqs:
        q.arrival = None
    with DsServer(hbm_budget=8e9, slots=4) as srv:  # all in flight together
        futs = [srv.submit(q) for q in reqs]
        mixed = {r.request_id: r for r in (f.result(timeout=300) for f in futs)}
        assert srv.peak_active > 1
    for i in alone:
        a, m = alone[i], mixed[i]
        assert a.n_ds == m.n_ds and a.n_ds > 0
        assert torch.equal(a.idx, m.idx)
        # per-point arithmetic is identical in both runs: bit-equal results
        assert torch.equal(a.ph.view(torch.float32), m.ph.view(torch.float32))
        assert torch.equal(a.quality.view(torch.int32), m.quality.view(torch.int32))
        assert torch.equal(a.t_coh.view(torch.int32), m.t_coh.view(torch.int32))
    s = latency_summary(list(mixed.values()))
    assert s["requests"] == len(reqs) and s["p99_ms"] >= s["p50_ms"] > 0


def test_kept_slot_memory_is_charged_and_given_back():
    """With slots keeping their memory between tiles (the device chain's plans and cached
    blocks), each slot is charged what it keeps; a request that the kept memory blocks makes
    the idle slots give theirs back instead of waiting for ever."""
    log, lock = [], threading.Lock()
    sizes = {0: 60, 1: 40, 2: 70, 3: 30, 4: 90, 5: 10}
    srv = DsServer(hbm_budget=100, slots=2, runner=_fake_runner(log, lock, hold=0.05),
                   footprint_fn=lambda r: sizes[r.request_id], keep_slot_memory=True)
    futs = [srv.submit(_req(i)) for i in sizes]
    res = [f.result(timeout=30) for f in futs]
    srv.close()
    assert [r.request_id for r in res] == list(sizes)
    assert srv.peak_used <= 100
    assert 0 < srv.used <= 100 and srv.used == sum(srv._charge)  # kept after the last tiles
    assert srv.admitted_order == list(sizes)
