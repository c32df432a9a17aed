"""Pin the CPU oracle to the reference's own outputs (tests/golden/*.npz)."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import golden_names, load_golden


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
