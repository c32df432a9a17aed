"""The reference's own acceptance checks (its tests/test_denoiser.py strategy),
run through this package on the reference's phantom fixture: every method and
recombination (the adaptive SURE / GSURE / QUT shrinkage included) must lower
the residual noise level, and NORDIC must reject a non-numeric noise level."""

from __future__ import annotations

import pathlib

import numpy as np
import pytest

from patch_denoising_b200 import (
    adaptive_thresholding,
    hybrid_pca,
    mp_pca,
    nordic,
    optimal_thresholding,
    raw_svt,
)

pytestmark = pytest.mark.gpu

_Z = np.load(pathlib.Path(__file__).parent / "golden" / "phantom" / "phantom.npz")
PHANTOM, NOISY, G_MAP = _Z["phantom"], _Z["noisy"], _Z["g_map"]
RECOMBINATIONS = ["weighted", "average", "center"]


def _noise_level(x):
    return float(np.sqrt(np.nanmean(np.nanvar(x - PHANTOM, axis=-1))))


def _lowers_noise(result):
    denoised = np.asarray(result[0], dtype=np.float64)
    assert _noise_level(denoised) < _noise_level(NOISY)


@pytest.mark.parametrize("recombination", RECOMBINATIONS)
def test_mp_pca_lowers_noise(recombination):
    _lowers_noise(mp_pca(NOISY, patch_shape=6, patch_overlap=5, threshold_scale=2.3, recombination=recombination))


@pytest.mark.parametrize("recombination", RECOMBINATIONS)
def test_hybrid_pca_lowers_noise(recombination):
    _lowers_noise(hybrid_pca(NOISY, patch_shape=6, patch_overlap=5, noise_std=1.0, recombination=recombination))


@pytest.mark.parametrize("recombination", RECOMBINATIONS)
def test_nordic_lowers_noise(recombination):
    _lowers_noise(nordic(NOISY, patch_shape=6, patch_overlap=5, noise_std=1.0, recombination=recombination))


@pytest.mark.parametrize("recombination", RECOMBINATIONS)
def test_raw_svt_lowers_noise(recombination):
    _lowers_noise(raw_svt(NOISY, patch_shape=6, patch_overlap=5, threshold=10, recombination=recombination))


@pytest.mark.parametrize("loss", ["fro", "nuc", "ope"])
@pytest.mark.parametrize("recombination", RECOMBINATIONS)
def test_optimal_lowers_noise(recombination, loss):
    _lowers_noise(optimal_thresholding(NOISY, patch_shape=6, patch_overlap=5, recombination=recombination,
                                       loss=loss))


@pytest.mark.parametrize("loss", ["fro", "nuc", "ope"])
@pytest.mark.parametrize("recombination", RECOMBINATIONS)
def test_optimal_with_noise_prior_lowers_noise(recombination, loss):
    _lowers_noise(optimal_thresholding(NOISY, patch_shape=10, patch_overlap=9, noise_std=1.414 * G_MAP,
                                       recombination=recombination, loss=loss))


def test_nordic_rejects_a_non_numeric_noise_level():
    with pytest.raises(ValueError):
        nordic(NOISY, patch_shape=6, patch_overlap=5, noise_std="not_a_float_or_array")


@pytest.mark.parametrize("recombination", ["weighted", "average"])
@pytest.mark.parametrize(
    "method, gamma", [("qut", None), ("gsure", np.linspace(1, 5, 10)), ("sure", np.linspace(1, 5, 10))]
)
def test_adaptive_lowers_noise(recombination, method, gamma):
    """The reference's adaptive check: patch 10, no overlap, noise map 2 g, nbsim 500."""
    np.random.seed(3)
    _lowers_noise(adaptive_thresholding(NOISY, patch_shape=10, patch_overlap=0, recombination=recombination,
                                        method=method, noise_std=2 * G_MAP, gamma0=gamma, nbsim=500))


@pytest.mark.parametrize("gamma", [None, 2.0])
def test_adaptive_sure_needs_a_gamma_list(gamma):
    """As the reference's loop over gamma0: a missing or scalar gamma0 is a TypeError."""
    with pytest.raises(TypeError):
        adaptive_thresholding(NOISY, patch_shape=10, patch_overlap=0, method="SURE", noise_std=2 * G_MAP,
                              gamma0=gamma)
