"""Functional entry points (drop-in for ``patch_denoise.denoise``, denoise.py:15-347)."""

from __future__ import annotations

from .space_time.lowrank import (
    AdaptiveDenoiser,
    HybridPCADenoiser,
    MPPCADenoiser,
    NordicDenoiser,
    OptimalSVDDenoiser,
    RawSVDDenoiser,
)


def mp_pca(input_data, patch_shape, patch_overlap, mask=None, mask_threshold=50, recombination="weighted",
           threshold_scale=1.0, progbar=None, *, precision="fp32"):
    """Marchenko-Pastur PCA denoising (denoise.py:15-62)."""
    den = MPPCADenoiser(patch_shape, patch_overlap, recombination=recombination,
                        threshold_scale=threshold_scale, precision=precision)
    return den.denoise(input_data, mask=mask, mask_threshold=mask_threshold)


def hybrid_pca(input_data, patch_shape, patch_overlap, mask=None, mask_threshold=50, noise_std=1.0,
               recombination="weighted", progbar=None, *, precision="fp32"):
    """Hybrid-PCA denoising (denoise.py:66-112)."""
    den = HybridPCADenoiser(patch_shape, patch_overlap, recombination=recombination, precision=precision)
    return den.denoise(input_data, mask=mask, mask_threshold=mask_threshold, noise_std=noise_std, progbar=progbar)


def raw_svt(input_data, patch_shape, patch_overlap, mask_threshold=50, mask=None, threshold=1.0,
            recombination="weighted", progbar=None, *, precision="fp32"):
    """Raw singular-value hard thresholding (denoise.py:116-163)."""
    den = RawSVDDenoiser(patch_shape, patch_overlap, recombination=recombination, threshold_value=threshold,
                         precision=precision)
    return den.denoise(input_data, mask=mask, mask_threshold=mask_threshold, threshold_scale=1.0, progbar=progbar)


def nordic(input_data, patch_shape, patch_overlap, mask_threshold=50, mask=None, noise_std=1.0,
           recombination="weighted", n_iter_threshold=10, progbar=None, *, precision="fp32"):
    """NORDIC denoising (denoise.py:167-221)."""
    den = NordicDenoiser(patch_shape, patch_overlap, recombination=recombination, precision=precision)
    return den.denoise(input_data, mask=mask, mask_threshold=mask_threshold, noise_std=noise_std,
                       n_iter_threshold=n_iter_threshold, progbar=progbar)


def optimal_thresholding(input_data, patch_shape, patch_overlap, mask=None, mask_threshold=50, loss="fro",
                         noise_std=None, recombination="weighted", eps_marshenko_pastur=1e-7, progbar=None, *,
                         precision="fp32"):
    """Optimal singular-value shrinkage (denoise.py:225-281)."""
    den = OptimalSVDDenoiser(patch_shape, patch_overlap, recombination=recombination, loss=loss,
                             precision=precision)
    return den.denoise(input_data, mask=mask, noise_std=noise_std, mask_threshold=mask_threshold,
                       eps_marshenko_pastur=eps_marshenko_pastur, progbar=progbar)


def adaptive_thresholding(input_data, patch_shape, patch_overlap, mask=None, mask_threshold=50,
                          recombination="weighted", method="SURE", nbsim=500, tau0=None, gamma0=None,
                          noise_std=1.0, progbar=None, *, precision="fp32"):
    """Adaptive trace-norm shrinkage, SURE / GSURE / QUT (denoise.py:285-347)."""
    den = AdaptiveDenoiser(patch_shape, patch_overlap, recombination=recombination, method=method, nbsim=nbsim,
                           precision=precision)
    return den.denoise(input_data, mask, mask_threshold, tau0, noise_std, gamma0, progbar=progbar)
