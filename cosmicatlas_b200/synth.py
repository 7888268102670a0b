"""Seeded synthetic inputs with the shapes and distributions of the
benchmark configurations (no external data is used).

* ``clumped``: a fraction of particles uniform in the periodic box, the rest
  in isotropic Gaussian clumps with uniform centres, wrapped into [0, L).
* ``halo_masses``: log10(M) ~ N(mu, sigma) truncated to [lo, hi] by
  rejection.
* ``zeldovich_lattice``: a Gaussian random field with a power-law times
  Gaussian-cutoff spectrum normalised to a target cell variance, and a
  lattice of particles displaced by its Zel'dovich displacement.
"""
from __future__ import annotations

import numpy as np


def _wrap32(v: np.ndarray, box: float) -> np.ndarray:
    """Wraps float64 positions into [0, box) and rounds to float32, keeping
    the float32 value strictly below box."""
    v = np.mod(v, box)
    f = v.astype(np.float32)
    f[f >= np.float32(box)] = np.float32(0.0)
    return f


def clumped(n: int, box: float, n_clumps: int, sigma: float, clump_frac: float = 0.8, seed: int = 0):
    """Returns float32 x, y, z of n particles."""
    rng = np.random.default_rng(seed)
    n_cl = int(round(n * clump_frac))
    n_un = n - n_cl
    pos = np.empty((3, n), np.float32)
    pos[:, :n_un] = _wrap32(rng.uniform(0.0, box, size=(3, n_un)), box)
    if n_cl:
        centres = rng.uniform(0.0, box, size=(3, n_clumps))
        which = rng.integers(0, n_clumps, size=n_cl)
        # process in chunks to bound memory for tens of millions of particles
        step = 1 << 22
        for s in range(0, n_cl, step):
            e = min(n_cl, s + step)
            p = centres[:, which[s:e]] + rng.normal(0.0, sigma, size=(3, e - s))
            pos[:, n_un + s:n_un + e] = _wrap32(p, box)
    return pos[0].copy(), pos[1].copy(), pos[2].copy()


def clumped_torch(n: int, box: float, n_clumps: int, sigma: float, clump_frac: float = 0.8, seed: int = 0,
                  device: str = "cuda"):
    """The clumped process of ``clumped`` drawn with torch on `device` (a
    different random stream than the numpy version, same distribution):
    returns float32 tensors x, y, z wrapped into [0, box)."""
    import torch
    g = torch.Generator(device=device).manual_seed(seed)
    n_cl = int(round(n * clump_frac))
    n_un = n - n_cl
    pos = torch.empty((3, n), dtype=torch.float64, device=device)
    pos[:, :n_un] = torch.rand((3, n_un), generator=g, device=device, dtype=torch.float64) * box
    if n_cl:
        centres = torch.rand((3, n_clumps), generator=g, device=device, dtype=torch.float64) * box
        which = torch.randint(0, n_clumps, (n_cl,), generator=g, device=device)
        pos[:, n_un:] = centres[:, which] + sigma * torch.randn((3, n_cl), generator=g, device=device,
                                                               dtype=torch.float64)
    f = torch.remainder(pos, box).to(torch.float32)
    f[f >= box] = 0.0
    return f[0].contiguous(), f[1].contiguous(), f[2].contiguous()


def halo_masses(n: int, mu: float = 12.5, sigma: float = 0.5, lo: float = 11.0, hi: float = 15.0, seed: int = 0):
    rng = np.random.default_rng(seed)
    out = np.empty(n, np.float64)
    filled = 0
    while filled < n:
        x = rng.normal(mu, sigma, size=max(1024, int((n - filled) * 1.1)))
        x = x[(x >= lo) & (x <= hi)]
        k = min(len(x), n - filled)
        out[filled:filled + k] = x[:k]
        filled += k
    return (10.0 ** out).astype(np.float32)


def config_c1(seed: int = 1):
    """2,000,000 particles, L = 1000, 20% uniform + 80% in 20,000 clumps of
    sigma = 2, unit weights; CIC onto 128^3 FP64, 64 bins, T-web R = 8."""
    x, y, z = clumped(2_000_000, 1000.0, 20_000, 2.0, 0.8, seed)
    return dict(x=x, y=y, z=z, w=None, n=128, box=1000.0, nbins=64, R=8.0, lth=0.0)


def config_c2(seed: int = 2, n_particles: int = 16_777_216):
    """16,777,216 particles, L = 1000, 200,000 clumps of sigma = 1.5, halo-like
    masses; NGP/CIC/TSC onto 256^3 FP32, 128 bins."""
    x, y, z = clumped(n_particles, 1000.0, 200_000, 1.5, 0.8, seed)
    w = halo_masses(n_particles, seed=seed + 1000)
    return dict(x=x, y=y, z=z, w=w, n=256, box=1000.0, nbins=128)


def config_c5_job(job: int, n_particles: int = 262_144):
    """One calibration-batch job: 262,144 particles, L = 500, clump fraction
    U[0.5, 0.9], sigma U[1, 4]; CIC onto 64^3, 32 bins, T-web R = 8."""
    rng = np.random.default_rng(5 + job)
    frac = rng.uniform(0.5, 0.9)
    sig = rng.uniform(1.0, 4.0)
    x, y, z = clumped(n_particles, 500.0, 2_000, sig, frac, seed=100_000 + job)
    return dict(x=x, y=y, z=z, w=None, n=64, box=500.0, nbins=32, R=8.0, lth=0.0)


def zeldovich_lattice(ng: int, box: float, amp_sigma: float = 1.0, kcut: float = 0.5, slope: float = -1.5,
                      seed: int = 3, device: str | None = None):
    """Gaussian random field on ng^3 with P(k) ~ k^slope exp(-(k/kcut)^2),
    scaled to unit cell variance (times amp_sigma), and particles on the
    lattice (i + 1/2) d displaced by psi_k = i k delta_k / k^2.  Uses torch
    (on `device`) for the FFTs.  Returns float32 x, y, z (torch tensors on
    `device` when given, else numpy) and delta."""
    import torch
    dev = torch.device(device or "cpu")
    g = torch.Generator(device=dev).manual_seed(seed)
    kf = 2.0 * np.pi / box
    white = torch.randn((ng, ng, ng), generator=g, device=dev, dtype=torch.float64)
    wk = torch.fft.rfftn(white)
    fx = torch.fft.fftfreq(ng, d=1.0 / ng, device=dev, dtype=torch.float64) * kf
    fz = torch.fft.rfftfreq(ng, d=1.0 / ng, device=dev, dtype=torch.float64) * kf
    k2 = fx[:, None, None] ** 2 + fx[None, :, None] ** 2 + fz[None, None, :] ** 2
    k = torch.sqrt(k2)
    pk = torch.where(k2 > 0, k.clamp_min(1e-30) ** slope * torch.exp(-(k / kcut) ** 2), torch.zeros_like(k))
    dk = wk * torch.sqrt(pk)
    delta = torch.fft.irfftn(dk, s=(ng, ng, ng))
    scale = amp_sigma / delta.std()
    dk = dk * scale
    delta = delta * scale
    d = box / ng
    lat = (torch.arange(ng, device=dev, dtype=torch.float64) + 0.5) * d
    ik2 = torch.where(k2 > 0, 1.0 / k2, torch.zeros_like(k2))
    out = []
    for a, f in enumerate((fx[:, None, None], fx[None, :, None], fz[None, None, :])):
        psi = torch.fft.irfftn(1j * f * ik2 * dk, s=(ng, ng, ng))
        shape = [1, 1, 1]
        shape[a] = ng
        pos = torch.remainder(psi + lat.view(shape), box).to(torch.float32).reshape(-1)
        pos[pos >= box] = 0.0
        out.append(pos)
        del psi
    if device is None:
        return out[0].numpy(), out[1].numpy(), out[2].numpy(), delta.numpy()
    return out[0], out[1], out[2], delta
