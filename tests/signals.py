"""Seeded synthetic inputs with the shapes of the workloads (no public
dataset is involved; these stand in for the reference's input kinds)."""
import numpy as np


def gaussian(N, seed, dtype=np.complex128):
    r = np.random.default_rng(seed)
    return (r.standard_normal(N) + 1j * r.standard_normal(N)).astype(dtype)


def gaussian_plus_tones(N, seed, ntones=64, dtype=np.complex128):
    """i.i.d. complex Gaussian plus `ntones` pure tones at random bin +
    fractional offsets, amplitudes log-uniform in [1e-6, 1]."""
    r = np.random.default_rng(seed)
    x = r.standard_normal(N) + 1j * r.standard_normal(N)
    n = np.arange(N, dtype=np.float64)
    for _ in range(ntones):
        f = r.integers(0, N) + r.random()
        a = 10.0 ** r.uniform(-6, 0)
        ph = r.uniform(0, 2 * np.pi)
        x += a * np.exp(1j * (2 * np.pi * ((f * n) % N) / N + ph))
    return x.astype(dtype)


def band_limited(N, seed, frac=0.05, dtype=np.complex128):
    """Gaussian noise whose spectrum is confined to a random band of frac*N bins."""
    r = np.random.default_rng(seed)
    W = max(1, int(frac * N))
    k0 = int(r.integers(0, N))
    X = np.zeros(N, np.complex128)
    idx = (k0 + np.arange(W)) % N
    X[idx] = r.standard_normal(W) + 1j * r.standard_normal(W)
    return np.fft.ifft(X).astype(dtype) * np.sqrt(N)


def gaussian_plus_tones_torch(N, seed, device="cuda"):
    """gaussian_plus_tones built on the GPU in FP64 (same recipe, torch RNG)."""
    import math
    import torch
    g = torch.Generator(device=device).manual_seed(seed)
    x = torch.complex(torch.randn(N, generator=g, device=device, dtype=torch.float64),
                      torch.randn(N, generator=g, device=device, dtype=torch.float64))
    n = torch.arange(N, device=device, dtype=torch.int64)
    r = np.random.default_rng(seed)
    for _ in range(64):
        k0 = int(r.integers(0, N))
        frac = float(r.random())
        amp = 10.0 ** r.uniform(-6, 0)
        ph0 = float(r.uniform(0, 2 * math.pi))
        ph = (torch.remainder(n * k0, N).to(torch.float64) + frac * n.to(torch.float64)) * (2 * math.pi / N) + ph0
        x += amp * torch.polar(torch.ones_like(ph), ph)
    return x
