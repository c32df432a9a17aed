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


# --------------------------------------------------------------------------- #
# Single-patch helpers of the reference module (space_time/utils.py:8-146).    #
# The denoisers never call these: their per-patch work is fused in the         #
# library's kernels. They are here so code written against the reference's    #
# utils keeps working; the decompositions run on the GPU through torch.linalg  #
# (cuSOLVER) in the input's precision, as the reference runs LAPACK in it.     #
# --------------------------------------------------------------------------- #
def get_patch_locs(p_shape, p_ovl, v_shape):
    """Top-left corners of all patches (space_time/utils.py:8-55), int32 (n_patches, ndim)."""
    if len(v_shape) != len(p_shape) or len(v_shape) != len(p_ovl):
        raise ValueError(f"Dimension mismatch between the arguments. {p_shape}{p_ovl}, {v_shape}")
    ranges = []
    for v_s, p_s, p_o in zip(v_shape, p_shape, p_ovl):
        if p_o >= p_s:
            raise ValueError("Overlap should be a non-negative integer smaller than patch_size")
        last = v_s - p_s
        r = np.arange(0, last, p_s - p_o, dtype=np.int32)
        if r[-1] < last:  # an empty range raises IndexError, as in the reference
            r = np.append(r, np.int32(last))
        ranges.append(r)
    grids = np.meshgrid(*ranges, indexing="ij")
    return np.stack([g.reshape(-1) for g in grids], axis=1).astype(np.int32)


def _device_array(a):
    """(tensor on the current CUDA device, was-numpy flag)."""
    if not torch.cuda.is_available():
        raise RuntimeError("patch_denoising_b200 needs a CUDA device (sm_100a); no CPU fallback exists")
    if isinstance(a, torch.Tensor):
        return a.to("cuda"), False
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda"), True


def _back(t, host):
    return t.cpu().numpy() if host else t


def svd_analysis(input_data):
    """Centred thin SVD: ``X = U @ (S * Vt) + M`` (space_time/utils.py:58-78)."""
    x, host = _device_array(input_data)
    mean = x.mean(dim=0)
    u, s, vt = torch.linalg.svd(x - mean, full_matrices=False)
    return _back(u, host), _back(s, host), _back(vt, host), _back(mean, host)


def svd_synthesis(u_vec, s_vals, v_vec, mean, idx):
    """``U[:, :idx] @ (S[:idx] * V[:idx]) + M`` (space_time/utils.py:81-99)."""
    u, host = _device_array(u_vec)
    s, _ = _device_array(s_vals)
    v, _ = _device_array(v_vec)
    m, _ = _device_array(mean)
    out = (u[:, :idx] @ (s[:idx, None].to(u.dtype) * v[:idx, :])) + m
    return _back(out, host)


def eig_analysis(input_data, max_eig_val=10):
    """Centred patch and the top ``max_eig_val`` eigenpairs of A^H A / (M - 1), ascending
    (space_time/utils.py:102-137)."""
    x, host = _device_array(input_data)
    mean = x.mean(dim=0)
    a = x - mean
    n_rows, n_cols = a.shape
    if not 0 < max_eig_val <= n_cols:
        raise ValueError("subset_by_index is out of range")
    vals, vecs = torch.linalg.eigh(a.conj().T @ a / (n_rows - 1))
    return _back(a, host), _back(vals[n_cols - max_eig_val:], host), _back(vecs[:, n_cols - max_eig_val:], host), \
        _back(mean, host)


def eig_synthesis(data_centered, eig_vec, mean, max_val):
    """``(A @ W) @ W^H + M`` with all but the last ``max_val`` columns of W zeroed in
    place, as the reference does (space_time/utils.py:140-146)."""
    eig_vec[:, :-max_val] = 0
    a, host = _device_array(data_centered)
    w, _ = _device_array(eig_vec)
    m, _ = _device_array(mean)
    return _back(((a @ w) @ w.conj().T) + m, host)
