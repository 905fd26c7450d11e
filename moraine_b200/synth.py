"""Seeded synthetic SLC stacks for the distributed-scatterer chain.

The reference's own real stack (a 2500x1834x17 Sentinel-1 crop) is not shipped with
it, so every test and benchmark here runs on scenes drawn by this module instead:

* the image plane is cut into Voronoi patches; a fraction of the seed points can be
  clustered around other seeds so that some patches are only a few pixels wide;
* each patch has a log-uniform mean intensity, a temporal coherence model
  ``gamma(dt) = gamma0 * exp(-dt / tau) + gamma_inf`` (``gamma(0) = 1``) and a linear
  deformation rate, giving the Hermitian covariance
  ``C[m, n] = I * gamma(|t_m - t_n|) * exp(1j * (phi_m - phi_n))``;
* distributed pixels are circular-Gaussian draws ``z = L w`` through the Cholesky
  factor ``L`` of their patch's covariance;
* persistent scatterers (a fraction of pixels) have a constant amplitude of ``ps_amp``
  times the patch amplitude and a phase that follows the deformation plus Gaussian
  noise of phase coherence ``ps_gamma``.

All randomness comes from one ``torch.Generator`` seeded with ``seed`` on the device the
stack is drawn on, so a (config, seed, device) triple always gives the same stack.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, replace

import numpy as np
import torch

WAVELENGTH_MM = 56.0  # C-band, 5.6 cm
DAYS_PER_YEAR = 365.25


@dataclass(frozen=True)
class SceneConfig:
    name: str
    nlines: int
    width: int
    nimages: int
    dt_days: float = 12.0
    n_patches: int = 12
    clustered_frac: float = 0.0   # fraction of seeds placed 2-6 px from another seed
    gamma0: float = 0.6
    gamma_inf: float = 0.1
    tau_days: float = 48.0
    vmax_mm_yr: float = 30.0
    ps_frac: float = 0.02
    ps_amp: float = 20.0
    ps_gamma: float = 0.95
    az_half_win: int = 5
    r_half_win: int = 5
    p_max: float = 0.05
    min_shp: int = 50
    seed: int = 0

    @property
    def az_win(self) -> int:
        return 2 * self.az_half_win + 1

    @property
    def r_win(self) -> int:
        return 2 * self.r_half_win + 1

    @property
    def npairs(self) -> int:
        return self.nimages * (self.nimages - 1) // 2

    def scaled(self, **kw) -> "SceneConfig":
        return replace(self, **kw)


# The five workloads of the benchmark plan (sizes, windows and scene models).
CONFIGS = {
    # plain method at small size, runnable on the CPU path
    "c0": SceneConfig("c0", 200, 200, 17, dt_days=12, n_patches=12, gamma0=0.6, gamma_inf=0.1,
                      tau_days=48, vmax_mm_yr=30, ps_frac=0.02, az_half_win=5, r_half_win=5,
                      min_shp=50, seed=0),
    # plain method at scale: 1000x1000x50, 15x31 window, DS = SHP count >= 50
    "c1": SceneConfig("c1", 1000, 1000, 50, dt_days=12, n_patches=60, gamma0=0.6, gamma_inf=0.1,
                      tau_days=48, vmax_mm_yr=30, ps_frac=0.02, az_half_win=7, r_half_win=15,
                      min_shp=50, seed=1),
    # batching plus precision: 2000x2000x100, 11x21 window, 200 patches many of them tiny
    "c2": SceneConfig("c2", 2000, 2000, 100, dt_days=12, n_patches=200, clustered_frac=0.6,
                      gamma0=0.5, gamma_inf=0.05, tau_days=36, vmax_mm_yr=50, ps_frac=0.01,
                      az_half_win=5, r_half_win=10, min_shp=50, seed=2),
    # precision stress: long low-coherence stack, near-singular |Gamma|
    "c3": SceneConfig("c3", 256, 256, 200, dt_days=6, n_patches=12, gamma0=0.3, gamma_inf=0.02,
                      tau_days=24, vmax_mm_yr=30, ps_frac=0.02, az_half_win=7, r_half_win=15,
                      min_shp=50, seed=3),
}


def coherence_model(cfg: SceneConfig, dt_days: torch.Tensor) -> torch.Tensor:
    g = cfg.gamma0 * torch.exp(-dt_days.abs() / cfg.tau_days) + cfg.gamma_inf
    return torch.where(dt_days == 0, torch.ones_like(g), g)


def _voronoi_labels(cfg: SceneConfig, gen: torch.Generator, device) -> torch.Tensor:
    H, W, P = cfg.nlines, cfg.width, cfg.n_patches
    seeds = torch.rand((P, 2), generator=gen, device=device, dtype=torch.float64)
    seeds[:, 0] *= H
    seeds[:, 1] *= W
    n_cl = int(round(cfg.clustered_frac * P))
    if n_cl > 0:
        # place the last n_cl seeds a few pixels away from one of the free seeds
        n_free = P - n_cl
        host = torch.randint(0, n_free, (n_cl,), generator=gen, device=device)
        r = 2.0 + 4.0 * torch.rand((n_cl,), generator=gen, device=device, dtype=torch.float64)
        a = 2 * math.pi * torch.rand((n_cl,), generator=gen, device=device, dtype=torch.float64)
        seeds[n_free:, 0] = (seeds[host, 0] + r * torch.cos(a)).clamp(0, H - 1e-6)
        seeds[n_free:, 1] = (seeds[host, 1] + r * torch.sin(a)).clamp(0, W - 1e-6)
    labels = torch.empty((H, W), dtype=torch.int64, device=device)
    cols = torch.arange(W, device=device, dtype=torch.float64) + 0.5
    rows_per_chunk = max(1, (1 << 22) // max(1, W * P))
    for r0 in range(0, H, rows_per_chunk):
        r1 = min(H, r0 + rows_per_chunk)
        rows = torch.arange(r0, r1, device=device, dtype=torch.float64) + 0.5
        d = (rows[:, None, None] - seeds[None, None, :, 0]) ** 2 + \
            (cols[None, :, None] - seeds[None, None, :, 1]) ** 2
        labels[r0:r1] = d.argmin(dim=-1)
    return labels


def make_stack(cfg: SceneConfig, device="cpu", return_truth: bool = False):
    """Draw the complex64 SLC stack ``(nlines, width, nimages)`` of ``cfg``.

    With ``return_truth`` also returns a dict with the patch labels, the PS mask and the
    true phase history of every pixel's patch.
    """
    device = torch.device(device)
    gen = torch.Generator(device=device)
    gen.manual_seed(cfg.seed)
    H, W, N, P = cfg.nlines, cfg.width, cfg.nimages, cfg.n_patches
    labels = _voronoi_labels(cfg, gen, device)

    t = torch.arange(N, device=device, dtype=torch.float64) * cfg.dt_days
    intensity = 10.0 ** (torch.rand((P,), generator=gen, device=device, dtype=torch.float64) * 2 - 1)
    vel = torch.rand((P,), generator=gen, device=device, dtype=torch.float64) * cfg.vmax_mm_yr
    phase = -4 * math.pi / WAVELENGTH_MM * vel[:, None] * (t[None, :] / DAYS_PER_YEAR)  # (P, N)
    gam = coherence_model(cfg, t[:, None] - t[None, :])  # (N, N)
    eph = torch.exp(1j * phase)  # (P, N)
    C = intensity[:, None, None] * gam[None] * (eph[:, :, None] * eph[:, None, :].conj())
    L = torch.linalg.cholesky(C)  # (P, N, N) complex128

    flat = labels.reshape(-1)
    npix = H * W
    rslc = torch.empty((npix, N), dtype=torch.complex64, device=device)
    chunk = max(1, (1 << 24) // N)
    for s0 in range(0, npix, chunk):
        s1 = min(npix, s0 + chunk)
        n = s1 - s0
        w = torch.randn((n, N, 2), generator=gen, device=device, dtype=torch.float32) * math.sqrt(0.5)
        w = torch.view_as_complex(w).to(torch.complex128)
        lab = flat[s0:s1]
        z = torch.empty((n, N), dtype=torch.complex128, device=device)
        for p in torch.unique(lab).tolist():
            sel = (lab == p).nonzero(as_tuple=True)[0]
            z[sel] = w[sel] @ L[p].T
        rslc[s0:s1] = z.to(torch.complex64)

    ps_mask = torch.rand((npix,), generator=gen, device=device) < cfg.ps_frac
    n_ps = int(ps_mask.sum().item())
    if n_ps:
        sig = math.sqrt(-2.0 * math.log(cfg.ps_gamma))
        lab = flat[ps_mask]
        amp = cfg.ps_amp * torch.sqrt(intensity[lab])
        theta0 = 2 * math.pi * torch.rand((n_ps, 1), generator=gen, device=device, dtype=torch.float64)
        eps = sig * torch.randn((n_ps, N), generator=gen, device=device, dtype=torch.float64)
        rslc[ps_mask] = (amp[:, None] * torch.exp(1j * (phase[lab] + theta0 + eps))).to(torch.complex64)

    rslc = rslc.reshape(H, W, N)
    if return_truth:
        return rslc, {"labels": labels, "ps_mask": ps_mask.reshape(H, W), "phase": phase,
                      "intensity": intensity, "velocity": vel}
    return rslc


@dataclass(frozen=True)
class TileSpec:
    """One request of a serving stream: a tile drawn from the small-scene generator."""
    request_id: int
    size: int
    nimages: int
    az_half_win: int
    r_half_win: int
    seed: int
    arrival_s: float

    def scene(self) -> SceneConfig:
        # the small-scene model (12 patches per 200 x 200 pixels) at this tile's size
        patches = max(4, round(12 * self.size * self.size / (200 * 200)))
        return CONFIGS["c0"].scaled(nlines=self.size, width=self.size, nimages=self.nimages,
                                    az_half_win=self.az_half_win, r_half_win=self.r_half_win,
                                    n_patches=patches, seed=self.seed)


# Serving workload: tile sizes, nimage and windows drawn uniformly, Poisson arrivals.
SERVING_SIZES = (256, 512, 1024, 2048)
SERVING_NIMAGES = (20, 50, 100, 150)
SERVING_WINDOWS = ((5, 5), (5, 10), (7, 15))  # 11x11, 11x21, 15x31


def serving_stream(n_requests: int, rate_per_s: float, seed: int = 4, sizes=SERVING_SIZES,
                   nimages=SERVING_NIMAGES, windows=SERVING_WINDOWS) -> list[TileSpec]:
    """A Poisson stream of ``n_requests`` tile requests, each with its own generator seed."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_per_s, size=n_requests))
    t -= t[0]
    out = []
    for i in range(n_requests):
        azh, rh = windows[rng.integers(len(windows))]
        out.append(TileSpec(i, int(sizes[rng.integers(len(sizes))]), int(nimages[rng.integers(len(nimages))]),
                            int(azh), int(rh), int(seed * 100000 + i), float(t[i])))
    return out


def rmli_of(rslc: torch.Tensor) -> torch.Tensor:
    """Intensity ``re*re + im*im`` in float32 with every product and sum rounded once.

    This is the intensity the device chain computes (``|slc|**2`` written without a fused
    multiply-add), so a host reference fed with it sees the same KS ties and orderings.
    """
    re, im = rslc.real.contiguous(), rslc.imag.contiguous()
    return (re * re) + (im * im)
