"""Pin the CPU oracle to the reference's own outputs (tests/golden/*.npz)."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import (
    adaptive_golden_names,
    golden_names,
    load_adaptive_golden,
    load_golden,
    load_noise_golden,
    noise_golden_names,
)


def _oracle_for(arrays, call):
    call = dict(call)
    method = call.pop("method")
    seed = call.pop("seed", None)
    x = arrays["input"]
    x = x.astype(np.complex128 if np.iscomplexobj(x) else np.float64)
    if seed is not None:
        call["nordic_rng"] = np.random.RandomState(seed)
    return oracle.denoise(
        method, x, call.pop("patch_shape"), call.pop("patch_overlap"), **call
    )


@pytest.mark.parametrize("name", golden_names())
def test_oracle_matches_reference(name):
    arrays, call = load_golden(name)
    res = _oracle_for(arrays, call)
    # integer / index work: exact
    np.testing.assert_array_equal(res["patches"], arrays["patches"])
    np.testing.assert_array_equal(res["patch_rank"], arrays["patch_rank"])
    np.testing.assert_allclose(res["patch_noise"], arrays["patch_noise"], rtol=1e-9, equal_nan=True)
    if "threshold" in arrays:
        assert res["threshold"] == pytest.approx(float(arrays["threshold"]), rel=1e-12)
    if "mp_median" in arrays:
        assert res["mp_median"] == float(arrays["mp_median"])
    # weights are float32 sums of the same float values in the same order
    np.testing.assert_array_equal(res["weights"], arrays["weights"])
    gold = arrays["out"]
    out = res["out"].astype(gold.dtype)
    np.testing.assert_array_equal(np.isnan(out), np.isnan(gold))
    ok = ~np.isnan(gold)
    scale = np.max(np.abs(gold[ok])) if ok.any() else 1.0
    np.testing.assert_allclose(out[ok], gold[ok], rtol=1e-6, atol=1e-6 * scale)


@pytest.mark.parametrize("name", noise_golden_names())
def test_oracle_noise_map_matches_reference(name):
    x, b, ref, covered = load_noise_golden(name)
    ours = oracle.estimate_noise(x, b)
    np.testing.assert_array_equal(oracle.estimate_noise_covered(x.shape[:-1], b), covered)
    np.testing.assert_allclose(ours[covered], ref[covered], rtol=1e-13, atol=0)
    assert np.all(ours[~covered] == 0)


def test_oracle_noise_map_rejects_short_axes():
    with pytest.raises(IndexError):
        oracle.estimate_noise(np.zeros((3, 8, 8, 5)), 3)


@pytest.mark.parametrize("name", adaptive_golden_names())
def test_oracle_adaptive_matches_reference(name):
    """The adaptive restatement (scipy BFGS as the reference, the QUT draws replayed
    from NumPy's seeded global generator) against the reference's own outputs."""
    arrays, call = load_adaptive_golden(name)
    call = dict(call)
    seed = call.pop("seed", None)
    x = arrays["input"]
    x = x.astype(np.complex128 if np.iscomplexobj(x) else np.float64)
    if seed is not None:
        np.random.seed(seed)
    res = oracle.denoise(call.pop("method"), x, call.pop("patch_shape"), call.pop("patch_overlap"), **call)
    np.testing.assert_array_equal(res["patches"], arrays["patches"])
    np.testing.assert_array_equal(res["patch_rank"], arrays["patch_rank"])
    np.testing.assert_array_equal(res["weights"], arrays["weights"])
    gold = arrays["out"]
    out = res["out"].astype(gold.dtype)
    np.testing.assert_array_equal(np.isnan(out), np.isnan(gold))
    ok = ~np.isnan(gold)
    np.testing.assert_allclose(out[ok], gold[ok], rtol=1e-6, atol=1e-6 * np.max(np.abs(gold[ok])))


def test_adaptive_search_reaches_a_lower_cost_than_the_reference_bfgs():
    """Per patch of the SURE / GSURE fixtures, the library's minimisation (the
    oracle's search mode) against the (gamma, tau) the reference's BFGS selects,
    both costs evaluated in float64: lower almost everywhere (BFGS mostly stops at
    its start point), never higher by more than a percent."""
    from oracle import oracle as O
    from scipy.optimize import minimize

    lower = total = 0
    for name in adaptive_golden_names():
        arrays, call = load_adaptive_golden(name)
        if call["adaptive_method"] == "qut":
            continue
        x = arrays["input"].astype(np.complex128 if np.iscomplexobj(arrays["input"]) else np.float64)
        p_s, p_o = O.patch_params(x.shape, call["patch_shape"], call["patch_overlap"])
        ps, step, grid = O.grid_geometry(x.shape, p_s, p_o)
        prior = O._prior_patches(call["noise_std"], x.shape)
        gs = call["adaptive_method"] == "gsure"
        for i in O.select_patches(O._broadcast_mask(None, x.shape), ps, step, grid, 50):
            sl = O._patch_slices(i, ps, step, grid)
            xp = x[sl].reshape(int(np.prod(p_s[:-1])), -1)
            s = O.svd_analysis(xp)[1].astype(np.float64)
            sig = np.sqrt(np.mean(prior[sl]))
            s2 = s**2
            si = np.array([np.sum(1.0 / (s2[k] - np.delete(s2, k))) for k in range(len(s))])
            x0 = np.log(np.median(s)) if call["tau0"] is None else call["tau0"]
            ref_best, ref64, ours = np.inf, None, np.inf
            for g in call["gamma0"]:
                xb = minimize(lambda t: O.sure_atn_cost(xp.shape, call["adaptive_method"], s, g, sig, t), x0).x[0]  # noqa: B023
                cb = O.sure_atn_cost(xp.shape, call["adaptive_method"], s, g, sig, xb)
                if cb < ref_best:
                    ref_best, ref64 = cb, O.atn_cost64(s, si, xp.shape, xb, g, sig, gs)
                xs = O.line_search_min(lambda t: O.atn_cost64(s, si, xp.shape, t, g, sig, gs),  # noqa: B023
                                       x0, np.log(s[-1]) - 10, np.log(s[0]) + 10)
                ours = min(ours, O.atn_cost64(s, si, xp.shape, xs, g, sig, gs))
            total += 1
            lower += ours <= ref64
            assert ours <= ref64 + 1e-2 * abs(ref64), (name, i, ours, ref64)
    assert lower >= 0.95 * total, (lower, total)
