"""Seeded synthetic SIFT-like descriptors (the reference's real data, tests/ApiTests.cpp:42, is
private and absent; no public dataset is used).

Each descriptor is 128-D uint8 = 4x4 spatial bins x 8 orientations.  A descriptor picks one of
``n_components`` mixture means (uniform weights, or Zipf(s) weights over the component rank),
draws every element from a Gamma(shape 0.5) distribution whose mean is that element of the
mixture mean, then follows the SIFT normalisation: L2-normalise, clip each element at 0.2,
renormalise, scale by 512, clamp to 255 and round.

Sampling runs in torch on the requested device (CUDA for bench-size inputs; the CPU for small
test cases).  The same (seed, device) always gives the same descriptors.
"""
from __future__ import annotations

import torch

SHAPE = 0.5


def mixture_means(n_components: int, seed: int, device: str | torch.device = "cpu") -> torch.Tensor:
    """[n_components, 128] float32 positive means: per spatial bin a random orientation profile."""
    g = torch.Generator(device="cpu").manual_seed(seed)
    bins = torch.rand((n_components, 16, 1), generator=g) * 1.5 + 0.25      # bin energy
    orient = torch.rand((n_components, 16, 8), generator=g) ** 3             # peaky orientation histograms
    means = (bins * orient).reshape(n_components, 128) + 0.02
    return means.to(device=device, dtype=torch.float32)


def component_weights(n_components: int, zipf: float | None) -> torch.Tensor:
    if zipf is None:
        return torch.full((n_components,), 1.0 / n_components, dtype=torch.float64)
    r = torch.arange(1, n_components + 1, dtype=torch.float64)
    w = r.pow(-zipf)
    return w / w.sum()


@torch.no_grad()
def sift_like(n: int, seed: int, n_components: int = 256, zipf: float | None = None,
              means_seed: int = 0, device: str | torch.device = "cpu", chunk: int = 1 << 21) -> torch.Tensor:
    """[n, 128] uint8 descriptors on ``device``."""
    device = torch.device(device)
    means = mixture_means(n_components, means_seed, device)
    w = component_weights(n_components, zipf).to(device)
    out = torch.empty((n, 128), dtype=torch.uint8, device=device)
    g = torch.Generator(device=device).manual_seed(seed)
    for beg in range(0, n, chunk):
        m = min(chunk, n - beg)
        comp = torch.multinomial(w, m, replacement=True, generator=g)
        mu = means[comp]                                                  # [m, 128]
        alpha = torch.full_like(mu, SHAPE)
        # Gamma(shape, scale) with scale = mean / shape; torch draws Gamma(shape, 1).
        gam = _standard_gamma(alpha, g) * (mu / SHAPE)
        v = gam / gam.norm(dim=1, keepdim=True).clamp_min(1e-12)
        v = v.clamp_max(0.2)
        v = v / v.norm(dim=1, keepdim=True).clamp_min(1e-12)
        out[beg: beg + m] = (v * 512.0).clamp_max(255.0).round().to(torch.uint8)
    return out


def _standard_gamma(alpha: torch.Tensor, g: torch.Generator) -> torch.Tensor:
    # torch._standard_gamma has no generator argument; draw Gamma(alpha) for alpha < 1 as
    # Gamma(alpha + 1) * U^(1/alpha) (Marsaglia & Tsang's boost), with Gamma(alpha + 1) from the
    # Marsaglia-Tsang squeeze method, all from the seeded generator.
    a1 = alpha + 1.0
    d = a1 - 1.0 / 3.0
    c = 1.0 / torch.sqrt(9.0 * d)
    res = torch.empty_like(alpha)
    todo = torch.ones_like(alpha, dtype=torch.bool)
    for _ in range(64):
        if not bool(todo.any()):
            break
        x = torch.randn(alpha.shape, generator=g, device=alpha.device, dtype=alpha.dtype)
        u = torch.rand(alpha.shape, generator=g, device=alpha.device, dtype=alpha.dtype)
        v = (1.0 + c * x) ** 3
        ok = (v > 0) & (torch.log(u.clamp_min(1e-30)) < 0.5 * x * x + d - d * v + d * torch.log(v.clamp_min(1e-30)))
        take = ok & todo
        res = torch.where(take, d * v, res)
        todo = todo & ~ok
    res = torch.where(todo, d, res)  # vanishingly rare: fall back to the mode
    u = torch.rand(alpha.shape, generator=g, device=alpha.device, dtype=alpha.dtype)
    return res * u.clamp_min(1e-30).pow(1.0 / alpha)


def log_uniform_counts(n_images: int, lo: int, hi: int, seed: int) -> torch.Tensor:
    """Per-image descriptor counts, log-uniform in [lo, hi]."""
    g = torch.Generator().manual_seed(seed)
    u = torch.rand(n_images, generator=g, dtype=torch.float64)
    import math

    return torch.exp(math.log(lo) + u * (math.log(hi) - math.log(lo))).round().to(torch.int64)
