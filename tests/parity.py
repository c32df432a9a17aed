"""Helpers shared by the GPU parity tests: run the CUDA path and the oracle, compare."""

from __future__ import annotations

import os

import numpy as np

import oracle
from patch_denoising_b200.space_time import (
    HybridPCADenoiser,
    MPPCADenoiser,
    NordicDenoiser,
    OptimalSVDDenoiser,
    RawSVDDenoiser,
)

# Decision margins below these (relative) are near-threshold ties: the rank may
# differ from the FP64 oracle there, and the oracle then replays our rank. The
# mixed band is 5x the largest relative eigenvalue error of the split-bf16 Gram
# measured on the parity volumes (1.9e-3; tests/test_mixed_tie_bound.py).
TIE_TOL = {"fp32": 2e-3, "mixed": 1e-2}
# (test id, precision, ties, largest tie margin) of every compare() call, printed
# in the terminal summary
TIE_LOG = []
# rel-L2 bounds against the FP64 oracle: 1e-5 for plain FP32, 1e-4 for the mixed path
OUT_TOL = {"fp32": 1e-5, "mixed": 1e-4}


def run_ours(call, x, precision="fp32", nordic_max_sval=None):
    """Denoise x (float32/complex64 numpy) with the CUDA path described by ``call``."""
    c = dict(call)
    method = c.pop("method")
    patch, overlap = c.pop("patch_shape"), c.pop("patch_overlap")
    rec = c.pop("recombination")
    mask = c.pop("mask", None)
    mt = c.pop("mask_threshold", 50)
    if method == "mp-pca":
        den = MPPCADenoiser(patch, overlap, c.get("threshold_scale", 1.0), recombination=rec, precision=precision)
        res = den.denoise(x, mask=mask, mask_threshold=mt)
    elif method == "hybrid-pca":
        den = HybridPCADenoiser(patch, overlap, recombination=rec, precision=precision)
        res = den.denoise(x, mask=mask, mask_threshold=mt, noise_std=c.get("noise_std", 1.0))
    elif method == "raw":
        den = RawSVDDenoiser(patch, overlap, threshold_value=c["threshold_value"], recombination=rec,
                             precision=precision)
        res = den.denoise(x, mask=mask, mask_threshold=mt)
    elif method == "nordic":
        den = NordicDenoiser(patch, overlap, recombination=rec, precision=precision)
        res = den.denoise(x, mask=mask, mask_threshold=mt, noise_std=c.get("noise_std", 1.0),
                          mc_max_sval=nordic_max_sval)
    elif method == "optimal":
        den = OptimalSVDDenoiser(patch, overlap, loss=c["loss"], recombination=rec, precision=precision)
        res = den.denoise(x, mask=mask, mask_threshold=mt, noise_std=c.get("noise_std"))
    else:
        raise ValueError(method)
    return res, den


def run_oracle(call, x, rank_override=None, threshold=None):
    c = dict(call)
    method = c.pop("method")
    c.pop("seed", None)
    x64 = x.astype(np.complex128 if np.iscomplexobj(x) else np.float64)
    if threshold is not None:
        c["threshold"] = threshold
    return oracle.denoise(method, x64, c.pop("patch_shape"), c.pop("patch_overlap"), rank_override=rank_override,
                          **c)


def rel_l2(a, b):
    ok = np.isfinite(b)
    num = np.linalg.norm((a - b)[ok])
    den = np.linalg.norm(b[ok])
    return float(num / den) if den > 0 else float(num)


def compare(call, x, precision="fp32", nordic_max_sval=None, report=None):
    """Run both paths and assert parity; returns a dict of the measured errors."""
    (out, weights, noise_map, rank_map), den = run_ours(call, x, precision, nordic_max_sval)
    thr = None
    if call["method"] == "nordic":
        thr = float(call.get("noise_std", 1.0)) * den.mc_max_sval_
    ref = run_oracle(call, x, threshold=thr)
    np.testing.assert_array_equal(den.patch_index_, ref["patches"])
    ours_rank = np.asarray(den.patch_rank_, dtype=np.int64)
    diff = np.nonzero(ours_rank != ref["patch_rank"])[0]
    ties = {}
    for j in diff:
        assert ref["patch_margin"][j] < TIE_TOL[precision], (
            f"rank differs at patch {ref['patches'][j]} (ours {ours_rank[j]}, oracle {ref['patch_rank'][j]}) "
            f"with decision margin {ref['patch_margin'][j]:.3g}"
        )
        ties[int(ref["patches"][j])] = int(ours_rank[j])
    if ties:
        ref = run_oracle(call, x, rank_override=ties, threshold=thr)
    TIE_LOG.append((os.environ.get("PYTEST_CURRENT_TEST", "?").split(" ")[0], precision, len(ties),
                    max((float(ref["patch_margin"][j]) for j in diff), default=0.0)))
    gold = ref["out"]
    np.testing.assert_array_equal(np.isnan(out), np.isnan(gold))
    err_out = rel_l2(out.astype(gold.dtype), gold)
    err_w = rel_l2(weights.astype(np.float64), ref["weights"].astype(np.float64))
    np.testing.assert_array_equal(rank_map, ref["rank_map"])
    err_noise = rel_l2(noise_map.astype(np.float64), ref["noise_map"].astype(np.float64))
    fin = np.isfinite(ref["patch_noise"])
    np.testing.assert_array_equal(np.isfinite(den.patch_noise_), fin)
    result = dict(out=err_out, weights=err_w, noise_map=err_noise, ties=len(ties), patches=len(ref["patches"]))
    if report is not None:
        report.update(result)
    assert err_out <= OUT_TOL[precision], result
    assert err_w <= 1e-6, result
    assert err_noise <= 10 * OUT_TOL[precision], result
    return result
