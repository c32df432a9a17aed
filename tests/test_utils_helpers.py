"""The reference module's single-patch helpers (space_time/utils.py:8-146)."""

from __future__ import annotations

from itertools import product

import numpy as np
import pytest

import oracle
from patch_denoising_b200.space_time import (
    eig_analysis,
    eig_synthesis,
    get_patch_locs,
    svd_analysis,
    svd_synthesis,
)


@pytest.mark.parametrize("p_shape, p_ovl, v_shape", [((3, 3, 3), (1, 1, 1), (8, 7, 9)),
                                                     ((5, 5), (0, 4), (11, 9)), ((2,), (1,), (5,))])
def test_patch_locs_match_the_oracle(p_shape, p_ovl, v_shape):
    ours = get_patch_locs(p_shape, p_ovl, v_shape)
    assert ours.dtype == np.int32
    np.testing.assert_array_equal(ours, oracle.patch_locs(p_shape, p_ovl, v_shape))


def test_patch_locs_errors():
    with pytest.raises(ValueError):
        get_patch_locs((3, 3), (3, 1), (8, 8))
    with pytest.raises(ValueError):
        get_patch_locs((3, 3), (1, 1), (8, 8, 8))
    with pytest.raises(IndexError):
        get_patch_locs((8, 3), (1, 1), (8, 8))


CASES = [dict(cplx=c, shape=s, sigma=g) for c, s, g in product([False, True], [(100, 50), (100, 10)], [0.1, 1, 10])]


def _matrix(case):
    rng = np.random.RandomState(42)
    m, n = case["shape"]
    x = rng.randn(m, n) * case["sigma"]
    if case["cplx"]:
        x = x + 1j * rng.randn(m, n) * case["sigma"]
    return x


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_svd_helpers(case):
    x = _matrix(case)
    u, s, vt, mean = svd_analysis(x)
    ref = oracle.svd_analysis(x)
    np.testing.assert_allclose(s, ref[1], rtol=1e-10)
    np.testing.assert_allclose(mean, ref[3], rtol=1e-12)
    full = svd_synthesis(u, s, vt, mean, idx=len(s))
    # the reference's round-trip check, and exactness in float64
    assert np.sqrt(np.mean(np.abs(x - full) ** 2)) <= np.std(x) / 10
    np.testing.assert_allclose(full, x, atol=1e-10 * np.abs(x).max())
    k = 3
    np.testing.assert_allclose(svd_synthesis(u, s, vt, mean, k), oracle.svd_synthesis(*ref, k),
                               atol=1e-9 * np.abs(x).max())


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_eig_helpers(case):
    x = _matrix(case)
    a, d, w, mean = eig_analysis(x)
    ra, rd, rw, rmean = oracle.eig_analysis(x)
    np.testing.assert_allclose(d, rd, rtol=1e-9)
    np.testing.assert_allclose(a, ra, atol=1e-12 * np.abs(x).max())
    n = x.shape[1]
    new = eig_synthesis(a, w.copy(), mean, max_val=len(mean))
    # the reference's round-trip check
    assert np.sqrt(np.mean(np.abs(x - new) ** 2)) <= np.std(x)
    ref_new = oracle.eig_synthesis(ra, rw.copy(), rmean, 4)
    np.testing.assert_allclose(eig_synthesis(a, w.copy(), mean, 4), ref_new, atol=1e-8 * np.abs(x).max())
    if n >= 10:
        ww = w.copy()
        eig_synthesis(a, ww, mean, 4)
        assert np.all(ww[:, :-4] == 0)  # zeroed in place, as the reference does
