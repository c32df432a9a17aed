"""Seeded synthetic 4D ``(x, y, z, t)`` volumes with a known low-rank structure.

The benchmark volumes are spatial Gaussian blobs times temporal sinusoids plus
i.i.d. noise: ``sum_k A_k(x) c_k(t) + n``, with ``A_k`` a blob of amplitude
``amplitude`` and spatial standard deviation ``sigma_space`` voxels at a random
centre, and ``c_k(t) = sin(2 pi t / P_k + phi_k)`` with ``P_k ~ U[8, 30]`` frames.
Complex volumes multiply each component by a smooth random phase map
``exp(i phi_k(x))`` and add circular complex noise (``noise`` per component).
These stand in for fMRI data; no dataset is needed.
"""

from __future__ import annotations

import numpy as np


def lowrank_volume(
    shape,
    rank,
    *,
    amplitude=100.0,
    sigma_space=4.0,
    periods=(8.0, 30.0),
    noise=5.0,
    complex_valued=False,
    seed=0,
    dtype=None,
    noise_map=None,
):
    """Return ``(noisy, clean)`` arrays of ``shape`` (last axis = time).

    ``noise_map`` (spatial shape) multiplies the noise standard deviation voxelwise.
    """
    rng = np.random.default_rng(seed)
    spatial = shape[:-1]
    n_t = shape[-1]
    grids = np.meshgrid(*[np.arange(s, dtype=np.float64) for s in spatial], indexing="ij")
    t = np.arange(n_t, dtype=np.float64)
    cdtype = np.complex128 if complex_valued else np.float64
    clean = np.zeros(shape, dtype=cdtype)
    for _ in range(rank):
        centre = [rng.uniform(0, s - 1) for s in spatial]
        r2 = sum((g - c) ** 2 for g, c in zip(grids, centre))
        blob = amplitude * np.exp(-0.5 * r2 / sigma_space**2)
        period = rng.uniform(*periods)
        phase = rng.uniform(0, 2 * np.pi)
        course = np.sin(2 * np.pi * t / period + phase)
        comp = blob[..., None] * course
        if complex_valued:
            slope = rng.normal(0, 0.2, size=len(spatial))
            offset = rng.uniform(0, 2 * np.pi)
            phi = offset + sum(s * g for s, g in zip(slope, grids))
            comp = comp * np.exp(1j * phi)[..., None]
        clean += comp
    sd = noise if noise_map is None else noise * np.asarray(noise_map)[..., None]
    nz = rng.standard_normal(shape) * sd
    if complex_valued:
        nz = nz + 1j * rng.standard_normal(shape) * sd
    noisy = clean + nz
    if dtype is None:
        dtype = np.complex64 if complex_valued else np.float32
    return noisy.astype(dtype), clean.astype(dtype)


def ellipsoid_mask(spatial_shape, fill=0.55, seed=0):
    """Boolean ellipsoid centred in the volume covering about ``fill`` of the voxels."""
    rng = np.random.default_rng(seed)
    grids = np.meshgrid(*[np.arange(s, dtype=np.float64) for s in spatial_shape], indexing="ij")
    centre = [(s - 1) / 2 + rng.uniform(-1, 1) for s in spatial_shape]
    axes = np.array([s / 2.0 for s in spatial_shape])
    # scale so that the ellipsoid volume is ``fill`` of the box
    unit = np.pi / 6 if len(spatial_shape) == 3 else np.pi / 4
    scale = (fill / unit) ** (1.0 / len(spatial_shape))
    r2 = sum(((g - c) / (a * scale)) ** 2 for g, c, a in zip(grids, centre, axes))
    return r2 <= 1.0


def radial_noise_map(spatial_shape, base=3.0, extra=2.0):
    """``sigma(x) = base + extra * r / r_max``, ``r`` the distance to the volume centre."""
    grids = np.meshgrid(*[np.arange(s, dtype=np.float64) for s in spatial_shape], indexing="ij")
    centre = [(s - 1) / 2 for s in spatial_shape]
    r = np.sqrt(sum((g - c) ** 2 for g, c in zip(grids, centre)))
    return base + extra * r / r.max()


def lowrank_volume_torch(shape, rank, *, amplitude=100.0, sigma_space=4.0, periods=(8.0, 30.0), noise=5.0,
                         noise_map=None, seed=0, device="cuda"):
    """``lowrank_volume``'s construction (real), generated on the device with a
    seeded torch generator: for volumes of gigabytes, where host generation is
    slow. The same law, other random draws. Returns the float32 noisy volume."""
    import torch

    gen = torch.Generator(device=device).manual_seed(seed)
    spatial = shape[:-1]
    grids = torch.meshgrid(*[torch.arange(s, dtype=torch.float32, device=device) for s in spatial], indexing="ij")
    t = torch.arange(shape[-1], dtype=torch.float32, device=device)
    out = torch.zeros(shape, dtype=torch.float32, device=device)
    for _ in range(rank):
        u = torch.rand(len(spatial) + 2, generator=gen, device=device)
        centre = [float(u[i]) * (s - 1) for i, s in enumerate(spatial)]
        r2 = sum((g - c) ** 2 for g, c in zip(grids, centre))
        blob = amplitude * torch.exp(-0.5 * r2 / sigma_space**2)
        period = periods[0] + float(u[-2]) * (periods[1] - periods[0])
        course = torch.sin(2 * np.pi * t / period + 2 * np.pi * float(u[-1]))
        out += blob[..., None] * course
    sd = torch.full(spatial, float(noise), device=device) if noise_map is None else \
        float(noise) * torch.as_tensor(noise_map, dtype=torch.float32, device=device)
    out += torch.randn(shape, generator=gen, device=device) * sd[..., None]
    return out
