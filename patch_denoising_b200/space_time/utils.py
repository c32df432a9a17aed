"""Host utilities of the space-time path."""

from __future__ import annotations

import numpy as np
import torch

from .. import _engine


def marchenko_pastur_median(beta, eps=1e-7):
    """Median of the Marchenko-Pastur law of aspect ratio ``beta`` in [0, 1].

    Same 5-point dichotomy as the reference (space_time/utils.py:149-204), on the
    closed-form CDF instead of numerical quadrature; computed in libpd_b200.so.
    """
    return _engine.mp_median(beta, eps)


def estimate_noise(noise_sequence, block_size=1):
    """Noise map of a noise-only sequence (space_time/utils.py:207-242).

    ``noise_sequence`` has shape (spatial..., T) with 1 to 3 spatial axes. For
    every block of ``block_size`` voxels per spatial axis (all positions), the
    voxel ``block_size // 2`` past the block's corner gets the population
    standard deviation of the block's samples over all frames. Returns float64
    of the spatial shape: a NumPy array for a NumPy input, a CUDA tensor for a
    tensor input. Voxels that are no block's centre are 0 (the reference leaves
    them uninitialised). Runs in libpd_b200.so (FP64 moments of float32 or
    complex64 data); an axis not longer than ``block_size`` raises IndexError,
    as the reference's patch-location helper does.
    """
    if not torch.cuda.is_available():
        raise RuntimeError("patch_denoising_b200 needs a CUDA device (sm_100a); no CPU fallback exists")
    b = int(block_size)
    shape = tuple(noise_sequence.shape)
    if b < 1:
        raise ValueError("block_size must be at least 1")
    for v in shape[:-1]:
        if v - b <= 0:
            raise IndexError("index -1 is out of bounds for axis 0 with size 0")
    is_torch = isinstance(noise_sequence, torch.Tensor)
    if is_torch and noise_sequence.is_cuda:
        device = noise_sequence.device
    else:
        device = torch.device("cuda", torch.cuda.current_device())
    x = _engine.to_device(noise_sequence, device, _engine.compute_dtype(noise_sequence.dtype)).contiguous()
    out = _engine.estimate_noise(x, b)
    if is_torch:
        return out
    return out.cpu().numpy().astype(np.float64)
