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
