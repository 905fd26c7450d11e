#!/usr/bin/env python
"""Benchmark of the distributed-scatterer chain (KS -> coherence -> EMI -> temporal coherence).

Metric: DS pixels per second through the whole chain on one synthetic stack (the
2000 x 2000 x 100 complex64 scene with an 11 x 21 window by default), i.e. the number of
DS points whose phase history and temporal coherence are produced, divided by the time
of one pass over the stack (intensity, KS test + SHP selection over every pixel, DS
extraction, coherence, EMI, temporal coherence).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun, one rank per GPU) every rank processes its own stack (tiles are
independent: no collective on the data path) and ``value`` is the sum over ranks,
timed as the max over ranks. ``--impl reference`` times the host restatement of the
reference algorithm (the oracle port) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "DS pixels/s (KS->coh->EMI->tcoh)"
# The reference's own CPU chain (its Numba functions) cannot run where the benchmark runs;
# this port stands in for it. Both timed on the same crops and 8 threads in the build
# container (ks_test -> select_shp -> emperical_co_pc -> emi -> ds_temp_coh):
REF_CALIBRATION = {"reference_over_port": {"c0 200x200x17": 1.73, "c2 160x160x100 crop": 1.30},
                   "note": "the reference's Numba chain is faster than this port by these factors"}
UNIT = "DS pixels/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", default="c2")
    ap.add_argument("--size", type=int, default=0, help="override nlines = width (smaller runs)")
    ap.add_argument("--precision", default="fp64", help="coherence Gram arithmetic: fp64, fp32, bf16x3, bf16")
    ap.add_argument("--emi-precision", default=None,
                    help="EMI arithmetic: fp64, fp32, mixed or refine (default: refine with an fp64 Gram - FP64 "
                         "inverse, FP32 reduction, FP64 refinement and check - else fp32)")
    ap.add_argument("--no-variants", action="store_true", help="skip the precision variants")
    ap.add_argument("--no-oracle", action="store_true", help="skip the check against the FP64 oracle")
    ap.add_argument("--other-configs", default="c1,c3", help="other benchmark scenes run once after the headline "
                                                             "('' for none)")
    ap.add_argument("--oracle-points", type=int, default=10240, help="DS points checked against the oracle")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample", type=int, default=160, help="side of the crop timed on the host")
    ap.add_argument("--stream-chunk", type=int, default=500,
                    help="lines per chunk of the scene streamed from host memory (0: no streaming run)")
    ap.add_argument("--serve-requests", type=int, default=16, help="tiles in the serving episode (0: none)")
    ap.add_argument("--serve-rate", type=float, default=8.0, help="Poisson arrival rate of tiles per second")
    ap.add_argument("--serve-slots", type=int, default=4, help="tiles in flight at once")
    ap.add_argument("--serve-full", action="store_true",
                    help="full serving workload: tiles up to 2048^2 and nimage up to 150 (default: up to 1024^2, 100)")
    args = ap.parse_args()
    if args.steps < 1:
        ap.error("--steps must be at least 1")
    if args.impl == "ours" and args.warmup < 1:
        ap.error("--warmup must be at least 1 (the DS count and the stage split come from a warm-up pass)")
    return args


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------- peaks
def measured_peaks() -> dict:
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        d["source"] = "measured"
        return d
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


DTYPE = {"fp32": "f32", "bf16": "bf16 Gram, f32 EMI", "bf16x3": "bf16x3 Gram, f32 EMI", "fp64": "f64"}
EMI_DTYPE = {"fp64": "f64", "fp32": "f32", "mixed": "f32 + f64 for cond > 1e4",
             "refine": "f64 inverse, f32 reduction, f64 refinement and check"}


def dtype_of(gram: str, emi: str) -> str:
    if (gram, emi) in (("fp64", "fp64"), ("fp32", "fp32")):
        return DTYPE[gram]
    return f"{DTYPE[gram].split(' Gram')[0]} Gram; EMI {EMI_DTYPE[emi]}"

# DRAM bytes per DS point of one mr_emi call (inverse + reduce + tail kernels), by (N, EMI
# arithmetic): dram__bytes_read.sum + dram__bytes_write.sum of the three kernels over one
# sub-batch, from ncu captures of the c2 scene model at N = 100 (FP64: 3.117 GB / 8,743
# points; FP32: 4.195 GB / 17,485 points); the traffic scales with the points processed
EMI_TRAFFIC_PER_POINT = {(100, "fp64"): 356_500, (100, "fp32"): 239_900}

# DRAM bytes per unit of one kernel (dram__bytes_read.sum + dram__bytes_write.sum of one launch
# / the units it processed), from one-kernel ncu captures on the 512 x 512 x 100 crop of the c2
# scene model (profiles/*_c2_512.md); the traffic of these kernels scales with the units, so a
# full-size launch gets units x bytes. Keyed by (kernel, N); DS points, pixels for the KS merge.
KERNEL_TRAFFIC_PER_UNIT = {
    ("emi reduce fp32", 100): (2.768748e9 + 1.384547e9) / 34_510,   # prof512_reduce_f32c
    ("emi refine tail", 100): (10.324045e9 + 31.297536e6) / 34_510,  # prof512_tail_refine_c
    ("emi sweep fp64", 100): (1.368710e9 + 1.348463e9) / 34_510,     # prof512_sweep2
    ("gram fp64", 100): (1.502556e9 + 2.682337e9) / 69_019,          # prof512_gram_b
    ("ks merge", 100): (109.437696e6 + 38.131456e6) / 262_144,       # prof512_ks_kept
}


def fp32_simt_peak(dev) -> float:
    """FP32 FMA-pipe reference rate in TFLOP/s: cuBLAS SGEMM 8192^3 with TF32 off, best of 5."""
    import torch  # noqa: PLC0415

    old = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        a = torch.randn(8192, 8192, device=dev)
        b = torch.randn(8192, 8192, device=dev)
        c = a @ b
        best = 0.0
        for _ in range(5):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b, out=c)
            e1.record()
            e1.synchronize()
            best = max(best, 2 * 8192 ** 3 / (e0.elapsed_time(e1) / 1e3) / 1e12)
        del a, b, c
        return best
    finally:
        torch.backends.cuda.matmul.allow_tf32 = old


def stage_rooflines(cfg, stage: dict, n_ds: int, res, peaks: dict, fp32: float, chain, precision: str) -> dict:
    """Achieved rate of every stage against the bound that limits it.

    Algorithmic work per unit (unit = pixel for the raster stages, DS point for the rest):
      ks_select   4N + W + 4 bytes per pixel (rmli in, mask and count out), W(2N-1) merge steps
      coherence   8 S Q + 3 S N flops per DS point (S = its SHP count, Q = N(N-1)/2)
      emi_tcoh    2.7 N^3 + 80 N^2 flops per DS point (Cholesky + inverse of |Gamma|, complex
                  factorisation of M, inverse-iteration solves)
    """
    n = cfg.nimages
    npix = cfg.nlines * cfg.width
    q = n * (n - 1) // 2
    hbm = peaks.get("hbm_gbs")
    out = {}
    if stage.get("ks_select"):
        ms = stage["ks_select"] + stage.get("intensity", 0.0)
        byts = npix * (4 * n + cfg.az_win * cfg.r_win + 4) + npix * n * 12
        gbs = byts / (ms / 1e3) / 1e9
        out["ks_select"] = {"kernel": "intensity_kernel + sort_keys_kernel + ks_merge_kernel", "bound": "hbm",
                            "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm, "traffic": None,
                            "ms": ms, "merge_steps_per_s": npix * cfg.az_win * cfg.r_win * (2 * n - 1) / (ms / 1e3),
                            "peak_source": peaks["source"]}
    if stage.get("coherence") and n_ds:
        ms = stage["coherence"]
        idx = res.idx.long()
        s = res.shp_num[idx[:, 0], idx[:, 1]].double()
        flops = float((8 * s * q + 3 * s * n).sum().item())
        tf = flops / (ms / 1e3) / 1e12
        tc = precision in ("bf16", "bf16x3")
        g64 = precision == "fp64"
        peak = peaks.get("bf16_tflops") if tc else (fp32 / 2 if g64 else fp32)
        out["coherence"] = {"kernel": "gram_tc_kernel" if tc else "gram_kernel", "bound": "tensor" if tc else
                            ("fp64-simt" if g64 else "fp32-simt"), "achieved": tf, "peak": peak, "unit": "TFLOP/s",
                            "frac": tf / peak, "traffic": None, "ms": ms,
                            "peak_source": peaks["source"] + " bf16" if tc else
                            "cuBLAS SGEMM in this run (FP32, TF32 off)" + (", halved for the FP64 pipe" if g64 else "")}
    if stage.get("emi_tcoh") and n_ds:
        ms = stage["emi_tcoh"]
        calls = -(-n_ds // chain.batch)
        flops = n_ds * (2.7 * n ** 3 + 80 * n ** 2)
        tf = flops / (ms / 1e3) / 1e12
        tpp = EMI_TRAFFIC_PER_POINT.get((n, chain.emi_precision))
        f64 = chain.emi_precision == "fp64" or n > 128
        peak = fp32 / 2 if f64 else fp32  # the FP64 pipe of B200 runs at half the FP32 rate
        out["emi_tcoh"] = {"kernel": "mr_emi: inverse_kernel + reduce_kernel + tail_kernel", "bound":
                           "fp64-simt" if f64 else "fp32-simt",
                           "achieved": tf, "peak": peak, "unit": "TFLOP/s", "frac": tf / peak,
                           "traffic": tpp * n_ds / calls if tpp else None, "ms": ms,
                           "launches": calls, "peak_source": "cuBLAS SGEMM in this run (FP32, TF32 off)"
                           + (", halved for the FP64 pipe" if f64 else ""),
                           "executed_flops_per_point": 2 * n ** 3 + 16 * n ** 3 / 3}
    return out


def kernel_rooflines(cfg, ktimes: dict, n_ds: int, res, peaks: dict, fp32: float) -> dict:
    """Every timed kernel's average launch against the pipe or memory bound that limits it.

    ``ktimes``: name -> (total ms, launches) from the library's event pairs. Algorithmic work
    per unit, and the bound:
      ks sort keys      pixel: 4N bytes in, 4K out (K = keys per pixel)          HBM
      ks merge          pixel: 4N + W + 4 bytes (keys in, mask and count out)     HBM (as asked;
                        its real limit is shared memory: the bank conflicts of its
                        data-dependent merge reads, W(2N-1) merge steps per pixel)
      gram fp32/fp64    DS point: 8 S Q + 3 S N flops (S its SHP count)          FP32 / FP64 pipe
      emi inverse/sweep DS point: N^3/3 + N^3 flops (factorisation and inverse of |Gamma|)
      emi reduce        DS point: 4N^3/3 flops (the complex factorisation of M)
      emi tail          DS point: 80 N^2 flops (solves, back-transformation)
    The EMI split follows the terms of the stage's 2.7 N^3 + 80 N^2 figure; the kernels
    execute more (2 N^3 for Gauss-Jordan, 16 N^3/3 for the Householder reduction), given as
    executed_flops_per_unit.
    """
    n = cfg.nimages
    npix = cfg.nlines * cfg.width
    q = n * (n - 1) // 2
    w = cfg.az_win * cfg.r_win
    hbm = peaks.get("hbm_gbs")
    s_sum = None
    if n_ds:
        idx = res.idx.long()
        s_sum = float(res.shp_num[idx[:, 0], idx[:, 1]].double().sum().item())
    out = {}
    for name, (ms, launches) in ktimes.items():
        if not launches or ms <= 0:
            continue
        per = ms / launches
        ent = {"kernel": name, "launches": launches, "ms_total": ms, "ms_per_launch": per, "traffic": None}
        tpu = KERNEL_TRAFFIC_PER_UNIT.get((name, n))
        if tpu:
            units = npix if name == "ks merge" else n_ds
            ent["traffic"] = tpu * units / launches
            ent["traffic_source"] = ("ncu DRAM bytes per unit on a 512 x 512 crop of the same scene model, "
                                     "scaled to the units of a launch")
        if name == "ks sort keys":
            byts = npix * (4 * n + 4 * ((n + 4) & ~3)) / launches
            ent.update(bound="hbm", unit="GB/s", achieved=byts / (per / 1e3) / 1e9, peak=hbm,
                       peak_source=peaks["source"])
        elif name == "ks merge":
            byts = npix * (4 * n + w + 4) / launches
            ent.update(bound="hbm", unit="GB/s", achieved=byts / (per / 1e3) / 1e9, peak=hbm,
                       peak_source=peaks["source"],
                       merge_steps_per_s=npix * w * (2 * n - 1) / (ms / 1e3))
        elif name.startswith("gram") and s_sum is not None and "tc" not in name:
            flops = (8 * q + 3 * n) * s_sum / launches
            peak = fp32 / 2 if name.endswith("fp64") else fp32
            ent.update(bound="fp64-simt" if name.endswith("fp64") else "fp32-simt", unit="TFLOP/s",
                       achieved=flops / (per / 1e3) / 1e12, peak=peak,
                       peak_source="cuBLAS SGEMM in this run (FP32, TF32 off)"
                       + (", halved for the FP64 pipe" if name.endswith("fp64") else ""))
        elif name.startswith("emi") and n_ds and "rerun" not in name:
            pts = n_ds / launches
            if "inverse" in name:  # pivoted Gauss-Jordan
                alg, exe = 4 * n ** 3 / 3, 2 * n ** 3
            elif "sweep" in name:  # symmetric sweep: the lower triangle only
                alg, exe = 4 * n ** 3 / 3, n ** 3
            elif "reduce" in name:
                alg, exe = 4 * n ** 3 / 3, 16 * n ** 3 / 3
            else:
                alg, exe = 80 * n ** 2, None
            # the refined tail's flops are its FP64 residuals and correction
            f64 = name.endswith("fp64") or "refine" in name
            peak = fp32 / 2 if f64 else fp32
            ent.update(bound="fp64-simt" if f64 else "fp32-simt", unit="TFLOP/s",
                       achieved=alg * pts / (per / 1e3) / 1e12, peak=peak,
                       peak_source="cuBLAS SGEMM in this run (FP32, TF32 off)"
                       + (", halved for the FP64 pipe" if f64 else ""),
                       algorithmic_flops_per_unit=alg, executed_flops_per_unit=exe, units_per_launch=pts)
        else:
            continue
        ent["frac"] = ent["achieved"] / ent["peak"] if ent.get("peak") else None
        out[name] = ent
    return out


# ----------------------------------------------------------------------------- precision
def precision_variants(cfg, rslc, ref, dev) -> dict:
    """Time and accuracy of the chain's arithmetic variants against the FP64 chain on the same
    stack.

    ``ref`` is the FP64 chain's result. For each variant: DS pixels/s of one pass (after a
    warm-up pass), the fraction of DS points whose phase history is within 1 mrad of the
    FP64 chain's, the largest and 99th-percentile phase error in rad, the largest
    temporal-coherence error, the share of points routed to FP64 (mixed and refined EMI),
    and the largest coherence error over the first 20,000 DS points (the Gram alone,
    against its FP64 accumulation).
    """
    import torch  # noqa: PLC0415

    import moraine_b200 as mb  # noqa: PLC0415
    from moraine_b200.chain import DsChain  # noqa: PLC0415

    ref_ph, ref_t = ref.ph.clone(), ref.t_coh.clone()
    idx = ref.idx[:20000]
    pc = ref.is_shp[idx[:, 0].long(), idx[:, 1].long()].view(torch.bool)
    coh64 = mb.emperical_co_pc(rslc, idx, pc, precision="fp64")
    out = {}
    for gram, emi in (("fp32", "fp32"), ("fp64", "fp64"), ("fp64", "fp32"), ("fp64", "refine"),
                      ("fp64", "mixed")):
        ch = DsChain(cfg.nlines, cfg.width, cfg.nimages, cfg.az_half_win, cfg.r_half_win, cfg.p_max, cfg.min_shp,
                     precision=gram, emi_precision=emi, device=dev)
        ch.run(rslc)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        r = ch.run(rslc)
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        err = (r.ph * ref_ph.conj()).angle().abs().amax(-1)
        fin = torch.isfinite(err)
        e = err[fin].sort().values
        co = mb.emperical_co_pc(rslc, idx, pc, precision=gram)
        out[f"gram {gram}, emi {emi}"] = {
            "ds_pixels_per_s": r.n_ds / (ms / 1e3), "ms_per_step": ms,
            "frac_within_1mrad": float((err <= 1e-3).float().mean()),
            "phase_err_max_rad": float(e[-1]) if e.numel() else None,
            "phase_err_p99_rad": float(e[int(0.99 * (e.numel() - 1))]) if e.numel() else None,
            "t_coh_err_max": float((r.t_coh - ref_t).abs()[fin].max()) if e.numel() else None,
            "coh_err_max_abs": float((co - coh64).abs().max()),
            "routed_to_fp64": float((r.route == 1).float().mean()) if r.route is not None else
            (1.0 if emi == "fp64" else 0.0),
            "nan_points": int((~fin).sum())}
        del ch, r
    return out


# ----------------------------------------------------------------------------- oracle check
def oracle_check(cfg, rslc, res, gram: str, n_points: int = 10240, nthreads: int = 0) -> dict:
    """The headline chain's results against the FP64 oracle on a seeded sample of DS points.

    For ``n_points`` DS points drawn evenly from the run: the oracle's coherence (C, FP64
    accumulation) against the device coherence, the oracle's EMI (numpy LAPACK FP64 on that
    coherence) against the device phases, and the oracle's temporal coherence of the oracle
    phases against the device value. Reported: the fraction of points within 1 mrad, the
    median, 99th percentile and largest phase error in rad, the largest coherence and
    temporal coherence errors.
    """
    from concurrent.futures import ThreadPoolExecutor  # noqa: PLC0415

    import torch  # noqa: PLC0415
    from threadpoolctl import threadpool_limits  # noqa: PLC0415

    import moraine_b200 as mb  # noqa: PLC0415
    from oracle import oracle as O  # noqa: PLC0415

    nthreads = nthreads or cpu_threads()
    n = min(n_points, res.n_ds)
    sel = np.unique(np.linspace(0, res.n_ds - 1, n).round().astype(np.int64))
    t = torch.from_numpy(sel).to(res.idx.device)
    idx = res.idx[t]
    pc = res.is_shp[idx[:, 0].long(), idx[:, 1].long()]
    coh_dev = mb.emperical_co_pc(rslc, idx, pc.view(torch.bool), precision=gram).cpu().numpy()
    ph_dev = res.ph[t].cpu().numpy()
    tc_dev = res.t_coh[t].cpu().numpy()
    idx_np, pc_np = idx.cpu().numpy(), pc.cpu().numpy().astype(bool)
    t0 = time.perf_counter()
    coh = O.emperical_co_pc(rslc.cpu().numpy(), idx_np, pc_np, nthreads=nthreads).astype(np.complex64)

    def emi_part(c):
        with threadpool_limits(limits=1):
            return O.emi(c)

    with ThreadPoolExecutor(nthreads) as ex:
        parts = list(ex.map(emi_part, [coh[i:i + 64] for i in range(0, len(coh), 64)]))
    ph = np.concatenate([p[0] for p in parts])
    tc = O.ds_temp_coh(coh, ph.astype(np.complex64), nthreads=nthreads)
    err = np.abs(np.angle(ph_dev * np.conj(ph))).max(-1)
    fin = np.isfinite(err)
    e = np.sort(err[fin])
    return {"points": int(len(sel)), "frac_within_1mrad": float((err[fin] <= 1e-3).mean()) if fin.any() else None,
            "phase_err_p99_rad": float(e[int(0.99 * (len(e) - 1))]) if len(e) else None,
            "phase_err_max_rad": float(e[-1]) if len(e) else None,
            "phase_err_median_rad": float(np.median(e)) if len(e) else None,
            "coh_err_max_abs": float(np.abs(coh_dev - coh).max()),
            "t_coh_err_max": float(np.abs(tc_dev - tc)[fin].max()) if fin.any() else None,
            "nan_points": int((~fin).sum()), "oracle_s": time.perf_counter() - t0,
            "oracle": "C FP64 Gram (stored complex64) + numpy LAPACK eigh/inv FP64 + C temporal coherence, "
                      "DS points drawn evenly over the run"}


# ----------------------------------------------------------------------------- other configs
def config_leg(name: str, dev, gram: str, emi: str, variants, steps: int = 2, oracle_points: int = 2048) -> dict:
    """One pass of the chain on another benchmark scene (its own size, window and image
    count), timed after a warm-up pass, and the accuracy of each arithmetic variant against
    the FP64 oracle on a sample of its DS points (coherence max-abs, phase error, temporal
    coherence error, share of points recomputed in FP64)."""
    import torch  # noqa: PLC0415

    from moraine_b200.chain import DsChain  # noqa: PLC0415
    from moraine_b200.synth import CONFIGS, make_stack  # noqa: PLC0415

    cfg = CONFIGS[name]
    z = make_stack(cfg, device=dev)
    out = {"workload": f"ds-chain {cfg.name} {cfg.nlines}x{cfg.width}x{cfg.nimages} complex64, window "
                       f"{cfg.az_win}x{cfg.r_win}, DS = SHP count >= {cfg.min_shp}", "variants": {}}
    if cfg.nimages > 128:
        out["note"] = ("nimages > 128: EMI runs the FP64 kernel for every EMI arithmetic, so only the Gram "
                       "arithmetic differs between variants; the tensor-core Gram supports nimages <= 128")
    for g, e in variants:
        ch = DsChain(cfg.nlines, cfg.width, cfg.nimages, cfg.az_half_win, cfg.r_half_win, cfg.p_max, cfg.min_shp,
                     precision=g, emi_precision=e, device=dev)
        r = ch.run(z)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            r = ch.run(z)
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        ent = {"ds_pixels_per_s": r.n_ds / (ms / 1e3), "ms_per_step": ms, "n_ds": r.n_ds,
               "routed_to_fp64": float((r.route == 1).float().mean()) if r.route is not None else
               (1.0 if e == "fp64" or cfg.nimages > 128 else 0.0)}
        if oracle_points:
            ent["oracle_check"] = oracle_check(cfg, z, r, g, n_points=oracle_points)
        out["variants"][f"gram {g}, emi {e}"] = ent
        log(f"{name} gram {g} emi {e}: {ent['ds_pixels_per_s']:.0f} DS px/s")
        del ch, r
        torch.cuda.empty_cache()
    if (gram, emi) in variants:
        out["headline"] = out["variants"][f"gram {gram}, emi {emi}"]["ds_pixels_per_s"]
    return out


# ----------------------------------------------------------------------------- streaming
def scene_stream(cfg, rslc, ref, chain, args) -> dict:
    """The scene streamed from a host array through SceneRunner in chunks of full lines with
    az_half_win halo lines: wall-clock DS px/s with the host reads, copies and results included,
    and whether the results equal the whole-scene chain's bit for bit."""
    import torch  # noqa: PLC0415

    from moraine_b200.scene import ArraySource, SceneRunner
    host = rslc.cpu().numpy()
    runner = SceneRunner(host.shape, cfg.az_half_win, cfg.r_half_win, chunks=(args.stream_chunk, -1),
                         p_max=cfg.p_max, min_shp=cfg.min_shp, precision=args.precision,
                         emi_precision=chain.emi_precision, device=rslc.device)
    src = ArraySource(host)
    runner.run(src, return_shp_num=False)  # warm-up
    out = runner.run(src, return_shp_num=False)
    same = (out.n_ds == ref.n_ds and np.array_equal(out.idx, ref.idx.cpu().numpy())
            and np.array_equal(out.t_coh.view(np.uint32), ref.t_coh.cpu().numpy().view(np.uint32)))
    st = out.stats
    log(f"scene stream: {len(runner.tiles)} tiles of {runner.tile_shape}, {st['wall_s'] * 1e3:.0f} ms, "
        f"same as whole scene: {same}")
    del runner
    torch.cuda.empty_cache()
    return {"value": out.n_ds / st["wall_s"], "unit": UNIT, "wall_ms": st["wall_s"] * 1e3,
            "chunks": [args.stream_chunk, -1], "tiles": st["tiles"], "tile_shape": list(st["tile_shape"]),
            "read_bytes": st["read_bytes"], "n_ds": out.n_ds, "same_as_whole_scene": bool(same),
            "path": "moraine_b200.scene.SceneRunner over a host numpy stack (wall clock, results on the host)"}


# ----------------------------------------------------------------------------- serving
def serving_episode(dev, args) -> dict:
    """p50/p99 tile latency of a Poisson stream of tiles through the request loop.

    The stream is served twice after a warm-up pass: with ``--serve-slots`` tiles in flight
    under a 150 GB admission budget and arrivals in real time (latency), and one tile at a
    time with every tile queued at once (the plain chain's throughput on the same tiles).
    """
    import torch  # noqa: PLC0415

    from moraine_b200.serve import DsServer, TileRequest, latency_summary  # noqa: PLC0415
    from moraine_b200.synth import SERVING_NIMAGES, SERVING_SIZES, make_stack, serving_stream  # noqa: PLC0415

    sizes = SERVING_SIZES if args.serve_full else SERVING_SIZES[:3]
    nimg = SERVING_NIMAGES if args.serve_full else SERVING_NIMAGES[:3]
    specs = serving_stream(args.serve_requests, args.serve_rate, sizes=sizes, nimages=nimg)
    stacks = {}
    for sp in specs:  # drawn on the device, served from pinned host memory
        stacks[sp.request_id] = make_stack(sp.scene(), device=dev).cpu().pin_memory()
    torch.cuda.synchronize()

    def run(slots: int, realtime: bool) -> list:
        srv = DsServer(hbm_budget=150e9, slots=slots, device=dev)
        t0 = time.perf_counter()
        futs = []
        for sp in specs:
            at = t0 + sp.arrival_s if realtime else t0
            while realtime and time.perf_counter() < at:
                time.sleep(min(0.002, max(0.0, at - time.perf_counter())))
            futs.append(srv.submit(TileRequest(rslc=stacks[sp.request_id], az_half_win=sp.az_half_win,
                                               r_half_win=sp.r_half_win, precision=args.precision,
                                               emi_precision=args.emi_precision, request_id=sp.request_id,
                                               arrival=at)))
        out = [f.result() for f in futs]
        srv.close()
        return out

    run(args.serve_slots, False)  # warm-up: kernels, plans, allocator
    served = latency_summary(run(args.serve_slots, True))
    plain = latency_summary(run(1, False))
    return {"p50_ms": served["p50_ms"], "p99_ms": served["p99_ms"], "mean_ms": served["mean_ms"],
            "max_ms": served["max_ms"], "requests": served["requests"], "n_ds": served["n_ds"],
            "ds_pixels_per_s": served["ds_pixels_per_s"], "span_s": served["span_s"],
            "one_at_a_time_ds_pixels_per_s": plain["ds_pixels_per_s"], "slots": args.serve_slots,
            "hbm_budget_gb": 150, "rate_per_s": args.serve_rate,
            "workload": f"{len(specs)} Poisson tiles, sizes {list(sizes)}^2, nimage {list(nimg)}, windows "
                        f"11x11/11x21/15x31, small-scene generator with one seed per tile, from pinned host "
                        f"memory; latency = arrival to results in host memory"}


# ----------------------------------------------------------------------------- CPU leg
def cpu_threads() -> int:
    """Host threads for the CPU legs: all cores this process may use, capped at 64."""
    return max(1, min(64, len(os.sched_getaffinity(0))))


def cpu_chain_rate(cfg, rslc_np, side: int, nthreads: int, budget_s: float = 25.0):
    """Oracle chain on a side x side crop of the stack; DS pixels per second on the host.

    KS, selection and DS extraction run over the whole crop; coherence, EMI and temporal
    coherence then run over the crop's DS points in chunks until ``budget_s`` is spent,
    and the rate counts only the points that were finished (the KS time is charged in
    full).
    """
    from concurrent.futures import ThreadPoolExecutor  # noqa: PLC0415

    from threadpoolctl import threadpool_limits  # noqa: PLC0415

    from oracle import oracle as O  # noqa: PLC0415

    crop = np.ascontiguousarray(rslc_np[:side, :side])
    t0 = time.perf_counter()
    rmli = O.intensity(crop)
    p = O.ks_test(rmli, cfg.az_half_win, cfg.r_half_win, nthreads=nthreads)
    is_shp, num = O.select_shp(p, cfg.p_max)
    idx, pc = O.ds_candidates(is_shp, num, cfg.min_shp)
    done = 0
    chunk = 64 * nthreads

    def emi_one(c):  # complex64 LAPACK, the reference CPU path's own arithmetic
        with threadpool_limits(limits=1):
            return O.emi_c64(c)[0]

    with ThreadPoolExecutor(nthreads) as ex:
        for s0 in range(0, len(idx), chunk):
            coh = O.emperical_co_pc(crop, idx[s0:s0 + chunk], pc[s0:s0 + chunk], nthreads=nthreads).astype(
                np.complex64)
            parts = list(ex.map(emi_one, [coh[i:i + 64] for i in range(0, len(coh), 64)]))
            ph = np.concatenate(parts)
            O.ds_temp_coh(coh, ph.astype(np.complex64), nthreads=nthreads)
            done += len(coh)
            if time.perf_counter() - t0 > budget_s:
                break
    dt = time.perf_counter() - t0
    return done / dt, dt, done, len(idx)


def log(msg: str) -> None:
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


# ----------------------------------------------------------------------------- main
def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    from moraine_b200.synth import CONFIGS  # noqa: PLC0415

    cfg = CONFIGS[args.config]
    if args.size:
        cfg = cfg.scaled(nlines=args.size, width=args.size,
                         n_patches=max(8, cfg.n_patches * args.size * args.size // (cfg.nlines * cfg.width)))
    workload = {"workload": f"ds-chain {cfg.name} {cfg.nlines}x{cfg.width}x{cfg.nimages} complex64, "
                            f"window {cfg.az_win}x{cfg.r_win}, p<{cfg.p_max}, DS = SHP count >= {cfg.min_shp}",
                "nlines": cfg.nlines, "width": cfg.width, "nimages": cfg.nimages,
                "window": [cfg.az_win, cfg.r_win], "precision": args.precision,
                "l2": "inputs larger than L2 (stack, masks and coherence batch each exceed 126 MB)"
                      if cfg.nlines * cfg.width * cfg.nimages * 8 > 126e6 else "small input (fits L2)",
                "parallelism": f"independent tiles x{args.gpus}"}

    if args.impl == "reference":
        if rank != 0:
            return
        import torch  # noqa: PLC0415
        from moraine_b200.synth import make_stack  # noqa: PLC0415

        nthreads = cpu_threads()
        side = min(args.cpu_sample, cfg.nlines)
        sub = cfg.scaled(nlines=side, width=side,
                         n_patches=max(4, cfg.n_patches * side * side // (cfg.nlines * cfg.width)))
        z = make_stack(sub).numpy()
        log(f"reference arm: {nthreads} host threads, {side}x{side} crop")
        cpu_chain_rate(cfg, z[:48, :48], 48, nthreads, budget_s=5.0)  # warm caches / thread pools
        rates, times, nds = [], [], []
        for _ in range(args.steps):
            r, dt, n, _ = cpu_chain_rate(cfg, z, side, nthreads, budget_s=max(5.0, 60.0 / max(1, args.steps)))
            rates.append(r)
            times.append(dt)
            nds.append(n)
            log(f"reference step: {n} DS points in {dt:.1f} s")
        value = float(np.sum(nds) / np.sum(times))
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "note": "one host process (rank 0) on the host cores; the value is not summed over ranks",
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(times)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port",
                             "sample": f"{side}x{side} crop of the scene model per step ({int(np.mean(nds))} DS "
                                       f"points), oracle chain: C/OpenMP KS, Gram and temp_coh, complex64 numpy LAPACK EMI as the "
                                       f"reference computes it",
                             "calibration": REF_CALIBRATION},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return

    import torch  # noqa: PLC0415
    import torch.distributed as dist  # noqa: PLC0415

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta  # noqa: PLC0415
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    from moraine_b200 import _lib  # noqa: PLC0415
    from moraine_b200.chain import DsChain  # noqa: PLC0415
    from moraine_b200.synth import make_stack  # noqa: PLC0415

    _lib.load()
    rcfg = cfg.scaled(seed=cfg.seed + 1000 * rank)
    log(f"rank {rank}: generating {cfg.nlines}x{cfg.width}x{cfg.nimages} stack")
    rslc = make_stack(rcfg, device=dev)
    torch.cuda.synchronize()
    log("stack ready")
    emi_prec = args.emi_precision or ("refine" if args.precision == "fp64" else None)
    args.emi_precision = emi_prec  # the serving episode and the streamed scene use the same EMI
    chain = DsChain(cfg.nlines, cfg.width, cfg.nimages, cfg.az_half_win, cfg.r_half_win, cfg.p_max, cfg.min_shp,
                    precision=args.precision, emi_precision=emi_prec, device=dev)
    workload["emi_precision"] = chain.emi_precision

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        res = chain.run(rslc)
        torch.cuda.synchronize()
        log(f"warm-up pass done ({res.n_ds} DS points)")
    n_ds = res.n_ds

    # per-stage split (separate pass with events, outside the timed region)
    # per-kernel device time (event pairs around every launch), also a separate pass
    lib0 = _lib.load()
    chain.timing = True
    lib0.mr_set_kernel_timing(1)
    stage = chain.run(rslc).stage_ms
    torch.cuda.synchronize()
    ktimes = _lib.kernel_timing()
    lib0.mr_set_kernel_timing(0)
    chain.timing = False

    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    lib = _lib.load()
    launches0 = lib.mr_kernel_launches()
    t0.record()
    for _ in range(args.steps):
        res = chain.run(rslc)
    t1.record()
    barrier()
    launches = int(lib.mr_kernel_launches() - launches0)
    clk = clocks.stop()
    ms = t0.elapsed_time(t1) / args.steps
    log(f"timed: {ms:.1f} ms per step")
    if world > 1:
        t = torch.tensor([ms, float(n_ds)], device=dev, dtype=torch.float64)
        tmax = t.clone()
        dist.all_reduce(tmax[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
        ms_max, ds_total = float(tmax[0]), float(t[1])
    else:
        ms_max, ds_total = ms, float(n_ds)
    value = ds_total / (ms_max / 1e3)

    # end to end through the public chain API from pinned host memory
    e2e = None
    if not args.no_e2e:
        host = torch.empty(rslc.shape, dtype=rslc.dtype, pin_memory=True)
        host.copy_(rslc)
        out_ph = torch.empty((chain.shape[0] * chain.shape[1], cfg.nimages), dtype=torch.complex64, pin_memory=True)
        out_q = torch.empty((chain.shape[0] * chain.shape[1],), dtype=torch.float32, pin_memory=True)
        out_t = torch.empty_like(out_q)
        out_idx = torch.empty((chain.shape[0] * chain.shape[1], 2), dtype=torch.int32, pin_memory=True)
        dev_in = torch.empty_like(rslc)
        d2h = 0

        def e2e_step():
            dev_in.copy_(host, non_blocking=True)
            r = chain.run(dev_in)
            n = r.n_ds
            out_ph[:n].copy_(r.ph, non_blocking=True)
            out_q[:n].copy_(r.quality, non_blocking=True)
            out_t[:n].copy_(r.t_coh, non_blocking=True)
            out_idx[:n].copy_(r.idx, non_blocking=True)
            return n * (cfg.nimages * 8 + 4 + 4 + 8)

        e2e_step()
        barrier()
        log("e2e warm-up done")
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            d2h = e2e_step()
        e1.record()
        barrier()
        ems = e0.elapsed_time(e1) / args.steps
        if world > 1:
            t = torch.tensor([ems], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t[0])
        e2e = {"value": ds_total / (ems / 1e3), "unit": UNIT, "ms_per_step": ems,
               "h2d_bytes_per_step": int(rslc.numel() * 8), "d2h_bytes_per_step": int(d2h + 8),
               "path": "moraine_b200.chain.DsChain.run on a pinned host stack, results copied back"}

    # the scene streamed from host memory in halo tiles (reads, copies and compute overlapped)
    stream = None
    if not args.no_variants and world == 1 and args.stream_chunk > 0:
        stream = scene_stream(cfg, rslc, res, chain, args)

    # precision variants on the same stack, against the headline's FP64 chain
    variants = None
    oracle = None
    # single-GPU reports (precision variants, oracle check, serving): only at N = 1, so that
    # ranks stay in step
    if not args.no_variants and world == 1 and args.precision == "fp64":
        ref = res
        if chain.emi_precision != "fp64":
            ref = DsChain(cfg.nlines, cfg.width, cfg.nimages, cfg.az_half_win, cfg.r_half_win, cfg.p_max,
                          cfg.min_shp, precision="fp64", emi_precision="fp64", device=dev).run(rslc)
        variants = precision_variants(cfg, rslc, ref, dev)
        del ref
        torch.cuda.empty_cache()
    if not args.no_oracle and world == 1:
        log("oracle check of the headline results")
        oracle = oracle_check(cfg, rslc, res, args.precision, n_points=args.oracle_points)
        log(f"oracle check: {oracle['frac_within_1mrad']} within 1 mrad, max {oracle['phase_err_max_rad']:.2e}")

    # rooflines: every stage against its bound; the headline is the dominant stage
    peaks = measured_peaks()
    fp32 = fp32_simt_peak(dev)
    log(f"FP32 SIMT reference rate: {fp32:.1f} TFLOP/s (cuBLAS SGEMM, TF32 off)")
    stage_roof = stage_rooflines(cfg, stage, n_ds, res, peaks, fp32, chain, args.precision)
    kernel_roof = kernel_rooflines(cfg, ktimes, n_ds, res, peaks, fp32)
    dom = max(kernel_roof, key=lambda k: kernel_roof[k]["ms_total"]) if kernel_roof else None
    roofline = dict(kernel_roof[dom]) if dom else None
    others = None
    if args.other_configs and world == 1 and not args.size:
        others = {}
        for name in [c for c in args.other_configs.split(",") if c]:
            log(f"config {name}")
            # at nimages > 128 mixed and refined EMI both run every point in FP64 (route 1);
            # they stay in the table so that it shows the route fraction per arithmetic
            var = [("fp32", "fp32"), ("fp64", "fp64"), ("fp64", "refine"), ("fp64", "mixed")]
            others[name] = config_leg(name, dev, args.precision, chain.emi_precision, var)
    latency = None
    if args.serve_requests > 0 and world == 1:
        log(f"serving episode: {args.serve_requests} tiles")
        latency = serving_episode(dev, args)
        log(f"serving: p50 {latency['p50_ms']:.1f} ms, p99 {latency['p99_ms']:.1f} ms")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        nthreads = cpu_threads()
        side = min(args.cpu_sample, cfg.nlines)
        sub = cfg.scaled(nlines=side, width=side,
                         n_patches=max(4, cfg.n_patches * side * side // (cfg.nlines * cfg.width)))
        z = make_stack(sub).numpy()
        log(f"cpu baseline: {nthreads} host threads")
        cpu_chain_rate(cfg, z[:48, :48], 48, nthreads, budget_s=5.0)
        r, dt, n, ntot = cpu_chain_rate(cfg, z, side, nthreads, budget_s=25.0)
        cpu = {"value": r, "unit": UNIT, "cores": nthreads, "kind": "port",
               "sample": f"{side}x{side} crop of the scene model: KS over the crop, then {n} of its {ntot} DS "
                         f"points through coherence, EMI and temporal coherence ({dt:.1f} s), oracle chain"}
        log("cpu baseline done")

    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": dtype_of(args.precision, chain.emi_precision), "data": "synthetic",
            "config": workload, "n_ds_per_gpu": n_ds, "stage_ms": stage, "roofline": roofline,
            "stage_roofline": stage_roof, "kernel_roofline": kernel_roof, "kernel_ms": ktimes,
            "precision_variants": variants, "oracle_check": oracle, "other_configs": others,
            "cpu_baseline": cpu, "e2e": e2e, "scene_stream": stream, "latency": latency, "clocks": clk, "gpu_launches": launches,
        }))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
