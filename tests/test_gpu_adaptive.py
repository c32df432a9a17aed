"""GPU parity of the adaptive trace-norm shrinkage (AdaptiveDenoiser) against the
FP64 oracle on the reference-generated fixtures' inputs.

The reference minimises the SURE / GSURE cost with scipy's BFGS from a
finite-difference slope; that slope is dominated by the float32 rounding of the
cost's divergence sum (its sign flips against a float64 evaluation), so BFGS
stops at its start point in most patches and its tau is not a function of the
data that another implementation can reproduce (the oracle's "bfgs" mode
replays it bit for bit against the fixtures on the CPU). The library minimises
the same cost in float64 by a line search and Brent's method; the oracle's
"search" mode does the same on FP64 singular values, and the GPU is held to it.
A singular value within ``ADAPTIVE_TIE`` (relative) of tau may fall on either
side; the oracle then replays our rank. QUT: the oracle takes the GPU's
Monte-Carlo quantile (``qut_level_``) so both use the same tau.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from conftest import adaptive_golden_names, load_adaptive_golden
from parity import rel_l2
from patch_denoising_b200 import _engine
from patch_denoising_b200.space_time import AdaptiveDenoiser

pytestmark = pytest.mark.gpu

# singular values carry half the relative error of the split-bf16 Gram's
# eigenvalues (at most 1.9e-3 on the parity volumes, test_mixed_tie_bound.py):
# the mixed band is 1e-2, as the other rules'
ADAPTIVE_TIE = {"fp32": 5e-3, "mixed": 1e-2}
# rel-L2 bounds against the FP64 oracle (float32 LAPACK singular values move
# the search's result by ~1e-7; the Gram route's spectrum is less accurate)
ADAPTIVE_TOL = {"fp32": 1e-4, "mixed": 1e-3}


def _ours(x, call, precision):
    den = AdaptiveDenoiser(call["patch_shape"], call["patch_overlap"], method=call["adaptive_method"],
                           recombination=call["recombination"], nbsim=call["nbsim"], precision=precision)
    res = den.denoise(x, tau0=call["tau0"], noise_std=call["noise_std"], gamma0=call["gamma0"])
    return res, den


def _oracle(x, call, qlevel, override=None):
    c = dict(call)
    c.pop("seed", None)
    x64 = x.astype(np.complex128 if np.iscomplexobj(x) else np.float64)
    return oracle.denoise(c.pop("method"), x64, c.pop("patch_shape"), c.pop("patch_overlap"), qut_level=qlevel,
                          rank_override=override, optimizer="search", **c)


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
@pytest.mark.parametrize("name", adaptive_golden_names())
def test_adaptive_matches_the_oracle(name, precision):
    arrays, call = load_adaptive_golden(name)
    _check(arrays["input"], call, precision, name)


@pytest.mark.parametrize("method,gamma0", [("sure", [1.0, 2.0, 3.0]), ("gsure", [1.0, 2.0]), ("qut", None),
                                           ("qut", 2.0)])
def test_adaptive_rank_deficient_patches(method, gamma0):
    """Patches with fewer voxels than frames (M = 27 < T = 40): the centred
    Casorati matrix has a zero singular value, whose cost terms vanish (the
    reference's SVD returns a tiny one there), so the cost stays finite."""
    from patch_denoising_b200.synthetic import lowrank_volume

    x, _ = lowrank_volume((12, 11, 9, 40), 3, amplitude=30.0, noise=2.0, seed=77)
    call = dict(method="adaptive", patch_shape=3, patch_overlap=1, recombination="weighted",
                adaptive_method=method, noise_std=2.0, nbsim=200, gamma0=gamma0, tau0=None)
    if method == "gsure":
        # GSURE = rss / (1 - div / (M T))^2 falls towards 0 as tau drops below
        # every singular value, so where a patch's search stops (a local
        # minimum or the bound on log tau) is not a continuous function of the
        # spectrum; check that the cost stayed finite (every patch kept a
        # finite, well-formed result) rather than patch-by-patch parity
        np.random.seed(11)
        (out, weights, _, _), den = _ours(x, call, "fp32")
        ref = _oracle(x, call, den.qut_level_)
        np.testing.assert_array_equal(np.isfinite(out), np.isfinite(ref["out"]))
        assert np.all(np.asarray(den.patch_rank_) >= 0)
        return
    _check(x, call, "fp32", f"rank-deficient {method}")


@pytest.mark.parametrize("cplx,frames,recombination", [(True, 200, "weighted"), (False, 120, "average"),
                                                        (True, 72, "average"), (False, 300, "weighted")])
def test_adaptive_mixed_tensor_core_synthesis(cplx, frames, recombination):
    """The mixed path synthesises adaptive patches on the tensor cores: 11^3-voxel
    patches (five 256-voxel tiles and a partial one) and frame counts whose real
    widths (2 x 200, 120, 2 x 72, 300) leave partial 128-column and 64-wide K
    tiles. Held to the FP64 oracle like the fixtures."""
    from patch_denoising_b200.synthetic import lowrank_volume

    x, _ = lowrank_volume((17, 17, 11, frames), 5, amplitude=25.0, noise=2.0, complex_valued=cplx, seed=91)
    x = x.astype(np.complex64 if cplx else np.float32)
    call = dict(method="adaptive", patch_shape=11, patch_overlap=5, recombination=recombination,
                adaptive_method="sure", noise_std=2.0, nbsim=100, gamma0=[1.0, 2.0], tau0=None)
    _check(x, call, "mixed", f"tensor-core synthesis c={cplx} T={frames}")


def _check(x, call, precision, name):
    np.random.seed(11)
    (out, weights, _, rank_map), den = _ours(x, call, precision)
    qlevel = den.qut_level_
    ref = _oracle(x, call, qlevel)
    np.testing.assert_array_equal(den.patch_index_, ref["patches"])
    ours_rank = np.asarray(den.patch_rank_, dtype=np.int64)
    ties = {}
    for j in np.nonzero(ours_rank != ref["patch_rank"])[0]:
        assert ref["patch_margin"][j] < ADAPTIVE_TIE[precision], (
            f"rank differs at patch {ref['patches'][j]}: ours {ours_rank[j]}, oracle {ref['patch_rank'][j]}, "
            f"margin {ref['patch_margin'][j]:.3g}"
        )
        ties[int(ref["patches"][j])] = int(ours_rank[j])
    if ties:
        ref = _oracle(x, call, qlevel, ties)
    gold = ref["out"]
    np.testing.assert_array_equal(np.isnan(out), np.isnan(gold))
    err = rel_l2(out.astype(gold.dtype), gold)
    err_w = rel_l2(weights.astype(np.float64), ref["weights"].astype(np.float64))
    np.testing.assert_array_equal(rank_map, ref["rank_map"])
    print(f"{name} {precision}: rel-L2 {err:.2e}, weights {err_w:.2e}, ties {len(ties)} of {len(ref['patches'])}")
    assert err <= ADAPTIVE_TOL[precision]
    assert err_w <= 1e-6
    assert np.all(np.isnan(den.patch_noise_))  # the reference returns no noise estimate


def test_qut_level_statistics():
    """The per-call QUT quantile against the oracle's draws (same law, other generator)."""
    ours = _engine.adaptive_qut_level(64, 20, 400, seed=5, device=torch.device("cuda", 0))
    ref = oracle.qut_level((64, 20), 400, np.random.RandomState(1))
    assert abs(ours - ref) / ref < 0.02
    again = _engine.adaptive_qut_level(64, 20, 400, seed=5, device=torch.device("cuda", 0))
    assert again == ours
