"""The seeded synthetic SIFT-like data that stands in for the reference's private image data:
deterministic per seed, uint8, SIFT-normalised, and with the mixture and image-size
distributions the workloads are defined by."""
import math

import numpy as np
import torch

from rapidbow_b200.synth import component_weights, log_uniform_counts, sift_like


def test_same_seed_same_descriptors_other_seed_other_descriptors():
    a = sift_like(3000, seed=5)
    assert a.dtype == torch.uint8 and tuple(a.shape) == (3000, 128)
    assert torch.equal(a, sift_like(3000, seed=5))
    assert not torch.equal(a, sift_like(3000, seed=6))


def test_sift_normalisation():
    x = sift_like(20000, seed=9).numpy().astype(np.float64)
    norms = np.linalg.norm(x, axis=1)
    # L2-normalised, clipped at 0.2, renormalised, scaled by 512, clamped to 255 and rounded:
    # the clamp can only lower a norm, rounding moves it by at most half a unit per element
    rounding = 0.5 * math.sqrt(128)
    assert x.min() >= 0 and x.max() <= 255
    assert np.all(norms <= 512.0 + rounding)
    assert abs(np.median(norms) - 512.0) < rounding
    assert np.all(norms > 0)


def test_component_weights():
    u = component_weights(256, None).double()
    assert torch.allclose(u.sum(), torch.tensor(1.0, dtype=torch.float64), atol=1e-6)
    assert torch.allclose(u, torch.full_like(u, 1 / 256), atol=1e-6)
    z = component_weights(4096, 1.1).double()
    assert torch.allclose(z.sum(), torch.tensor(1.0, dtype=torch.float64), atol=1e-5)
    assert torch.all(z[1:] <= z[:-1])
    assert abs(float(z[0] / z[9]) - 10 ** 1.1) < 1e-3 * 10 ** 1.1


def test_log_uniform_image_sizes():
    c = log_uniform_counts(20000, 500, 4000, seed=3).numpy()
    assert c.min() >= 500 and c.max() <= 4000
    logs = np.log(c)
    assert abs(logs.mean() - (math.log(500) + math.log(4000)) / 2) < 0.02
    assert torch.equal(log_uniform_counts(100, 300, 8000, seed=1), log_uniform_counts(100, 300, 8000, seed=1))
