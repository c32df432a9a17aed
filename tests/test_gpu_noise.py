"""estimate_noise on the GPU vs the reference's maps and the FP64 oracle."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from conftest import load_noise_golden, noise_golden_names
from patch_denoising_b200.space_time import estimate_noise

pytestmark = pytest.mark.gpu

# FP64 moments of the same float32 samples the reference saw as float64: only
# the summation order differs from NumPy's.
RTOL = 1e-10


@pytest.mark.parametrize("name", noise_golden_names())
def test_noise_map_matches_reference(name):
    x, b, ref, covered = load_noise_golden(name)
    ours = estimate_noise(x, b)
    assert ours.dtype == np.float64 and ours.shape == x.shape[:-1]
    np.testing.assert_allclose(ours[covered], ref[covered], rtol=RTOL, atol=0)
    assert np.all(ours[~covered] == 0)


@pytest.mark.parametrize("block", [1, 2, 3, 5])
def test_noise_map_matches_oracle(block):
    rng = np.random.default_rng(block)
    x = (3.0 + rng.normal(scale=0.7, size=(14, 12, 9, 33))).astype(np.float32)
    np.testing.assert_allclose(estimate_noise(x, block), oracle.estimate_noise(x, block), rtol=RTOL, atol=1e-300)


def test_noise_map_large_volume_properties():
    """Full-size map: a constant-std field gives that std at every block centre."""
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn((96, 96, 48, 100), device="cuda", generator=g) * 2.5
    m = estimate_noise(x, 3)
    assert m.is_cuda and m.dtype == torch.float64
    inner = m[1:-1, 1:-1, 1:-1]
    assert abs(float(inner.mean()) - 2.5) < 0.01
    assert float(m[0].abs().max()) == 0.0 and float(m[:, :, -1].abs().max()) == 0.0


def test_noise_map_rejects_short_axes():
    with pytest.raises(IndexError):
        estimate_noise(np.zeros((3, 8, 8, 5), dtype=np.float32), 3)


@pytest.mark.parametrize("block_dim", [5, 10])
@pytest.mark.parametrize("seed", range(3))
def test_noise_estimation_reference_case(block_dim, seed):
    """The reference's noise-estimation case (a 200 x 200 x 100 white-noise
    sequence, blocks 5 and 10): the map averages to the sequence's std. (The
    reference leaves this check commented out as flaky: its border voxels are
    uninitialised; here they are 0 and the check uses the block centres.)"""
    x = np.random.default_rng(seed).normal(size=(200, 200, 100)).astype(np.float32)
    m = estimate_noise(x, block_dim)
    cov = oracle.estimate_noise_covered(x.shape[:-1], block_dim)
    assert abs(float(m[cov].mean()) - float(x.std())) <= 0.1 * float(x.std())
    assert np.all(m[~cov] == 0)
