"""The bench contract on the host: the reference arm's JSON line at N = 1 and under torchrun
at N = 2 (rank 0 prints one line, the other rank exits 0 without work)."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

REPO = Path(__file__).resolve().parents[1]
TINY = ["--impl", "reference", "--steps", "1", "--warmup", "0", "--config", "c0", "--size", "64",
        "--cpu-sample", "48"]


def _lines(out: str) -> list[dict]:
    return [json.loads(ln) for ln in out.splitlines() if ln.startswith("{")]


def test_reference_arm_line():
    out = subprocess.run([sys.executable, str(REPO / "bench.py"), *TINY], capture_output=True, text=True,
                         timeout=600, cwd=REPO)
    assert out.returncode == 0, out.stderr[-2000:]
    (d,) = _lines(out.stdout)
    assert d["impl"] == "reference" and d["n_gpus"] == 1 and d["value"] > 0
    assert d["unit"] == "DS pixels/s" and d["higher_is_better"] is True and d["scaling"] == "weak"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "workload" in d["config"]


def test_reference_arm_under_torchrun_prints_once():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    out = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                          "--master-addr", "127.0.0.1", "--master-port", str(port), str(REPO / "bench.py"),
                          "--gpus", "2", *TINY], capture_output=True, text=True, timeout=600, cwd=REPO, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    (d,) = _lines(out.stdout)
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0


def test_ours_arm_rejects_zero_warmup():
    out = subprocess.run([sys.executable, str(REPO / "bench.py"), "--warmup", "0", "--steps", "1"],
                         capture_output=True, text=True, timeout=120, cwd=REPO)
    assert out.returncode == 2 and "--warmup must be at least 1" in out.stderr


def test_kernel_rooflines_traffic_and_work():
    """Per-kernel rooflines on the host: the algorithmic work per unit, and the DRAM traffic of
    a launch scaled from the one-kernel captures' bytes per unit."""
    import importlib.util
    from types import SimpleNamespace

    import pytest
    import torch

    spec = importlib.util.spec_from_file_location("bench_mod", REPO / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    cfg = SimpleNamespace(nimages=100, nlines=8, width=8, az_win=11, r_win=21)
    res = SimpleNamespace(idx=torch.tensor([[0, 0], [1, 1], [2, 2]], dtype=torch.int32),
                          shp_num=torch.full((8, 8), 50, dtype=torch.int32))
    kt = {"emi reduce fp32": (6.0, 3), "emi sweep fp64": (3.0, 3), "ks merge": (1.0, 1), "gram fp64": (2.0, 1),
          "emi refine tail": (1.5, 3)}
    out = bench.kernel_rooflines(cfg, kt, 3, res, {"hbm_gbs": 6547.2, "source": "measured"}, 64.0)
    per = bench.KERNEL_TRAFFIC_PER_UNIT
    assert out["emi reduce fp32"]["traffic"] == pytest.approx(per[("emi reduce fp32", 100)] * 3 / 3)
    assert out["ks merge"]["traffic"] == pytest.approx(per[("ks merge", 100)] * 64)
    assert out["gram fp64"]["traffic"] == pytest.approx(per[("gram fp64", 100)] * 3)
    red, swp = out["emi reduce fp32"], out["emi sweep fp64"]
    assert red["algorithmic_flops_per_unit"] == pytest.approx(4 * 100 ** 3 / 3)
    assert red["executed_flops_per_unit"] == pytest.approx(16 * 100 ** 3 / 3)
    assert swp["algorithmic_flops_per_unit"] == pytest.approx(4 * 100 ** 3 / 3) and swp["bound"] == "fp64-simt"
    assert out["emi refine tail"]["bound"] == "fp64-simt"
    # achieved = work of a launch / its mean duration (2 ms for one DS point per launch)
    assert red["achieved"] == pytest.approx(4 * 100 ** 3 / 3 / 2e-3 / 1e12)
