"""Batched calls over volumes of uneven shape (pd_denoise_batch) against
per-volume calls, and the autotuner."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from parity import compare, rel_l2
from patch_denoising_b200 import HybridPCADenoiser, MPPCADenoiser, OptimalSVDDenoiser, RawSVDDenoiser
from patch_denoising_b200.batch import CANDIDATES, autotune, denoise_batch
from patch_denoising_b200.synthetic import ellipsoid_mask, lowrank_volume

pytestmark = pytest.mark.gpu

SHAPES = [(26, 22, 16, 60), (18, 20, 14, 100), (30, 24, 12, 40), (16, 16, 16, 130)]


def _volumes(cplx=False):
    vols, masks, sigmas = [], [], []
    for i, sh in enumerate(SHAPES):
        sigma = 2.0 + i
        x, _ = lowrank_volume(sh, 3 + i, noise=sigma, seed=100 + i, complex_valued=cplx)
        vols.append(x)
        masks.append(ellipsoid_mask(sh[:-1], fill=0.55, seed=i))
        sigmas.append(sigma)
    return vols, masks, sigmas


def _single(method, x, mask, sigma):
    if method == "mp-pca":
        return MPPCADenoiser(7, 4, 1.0).denoise(x, mask=mask, mask_threshold=50)
    if method == "hybrid-pca":
        return HybridPCADenoiser(7, 4).denoise(x, mask=mask, mask_threshold=50, noise_std=sigma)
    if method == "raw":
        return RawSVDDenoiser(7, 4, threshold_value=60.0).denoise(x, mask=mask, mask_threshold=50)
    return OptimalSVDDenoiser(7, 4, loss="fro").denoise(x, mask=mask, mask_threshold=50)


@pytest.mark.parametrize("method", ["optimal", "mp-pca", "hybrid-pca", "raw"])
@pytest.mark.parametrize("cplx", [False, True])
def test_batch_matches_per_volume_calls(method, cplx):
    vols, masks, sigmas = _volumes(cplx)
    kw = dict(threshold_value=60.0) if method == "raw" else {}
    if method == "hybrid-pca":
        kw["noise_std"] = sigmas
    res = denoise_batch(vols, method, 7, 4, "weighted", masks, 50, tuning=None, **kw)
    for x, m, sg, (out, w, nm, rm) in zip(vols, masks, sigmas, res):
        o1, w1, n1, r1 = _single(method, x, m, sg)
        out, w, rm = out.cpu().numpy(), w.cpu().numpy(), rm.cpu().numpy()
        np.testing.assert_array_equal(np.isnan(out), np.isnan(o1))
        np.testing.assert_array_equal(rm, r1)
        assert rel_l2(out.astype(np.complex128), o1.astype(np.complex128)) <= 1e-6
        assert rel_l2(w.astype(np.float64), w1.astype(np.float64)) <= 1e-6


def test_batch_against_the_oracle():
    """One batch, each volume held to the FP64 oracle (optimal shrinkage, T <= M)."""
    vols, masks, _ = _volumes()
    res = denoise_batch(vols, "optimal", 7, 4, "weighted", masks, 50, tuning=None)
    for x, m, (out, w, nm, rm) in zip(vols, masks, res):
        call = dict(method="optimal", patch_shape=7, patch_overlap=4, recombination="weighted", loss="fro", mask=m,
                    mask_threshold=50)
        rep = {}
        compare(call, x, report=rep)  # the single-volume path against the oracle
        o1, _, _, _ = _single("optimal", x, m, None)
        assert rel_l2(out.cpu().numpy().astype(np.float64), o1.astype(np.float64)) <= 1e-6


def test_autotuner_picks_a_candidate_and_caches_it():
    vols, masks, _ = _volumes()
    res, tn = denoise_batch(vols, "mp-pca", 7, 4, "weighted", masks, 50, return_tuning=True)
    assert tn in CANDIDATES
    res2, tn2 = denoise_batch(vols, "mp-pca", 7, 4, "weighted", masks, 50, return_tuning=True)
    assert tn2 == tn  # the cached choice
    for (a, *_), (b, *_) in zip(res, res2):
        fa = torch.isfinite(a)
        assert torch.equal(fa, torch.isfinite(b))
        assert float(torch.linalg.vector_norm(a[fa] - b[fa]) / torch.linalg.vector_norm(b[fa])) <= 1e-6
