"""The mixed path's tie band, derived from its eigenvalue error.

The chosen (mixed) path forms each patch Gram from split bf16 operands:
x = hi + lo with hi = bf16(x), lo = bf16(x - hi), and
G = hi·hiᵀ + hi·loᵀ + lo·hiᵀ accumulated in FP32. This test emulates that
split exactly (round-to-nearest-even bf16 in NumPy, exact products) on the
volumes the GPU parity tests use, and measures the largest relative error of
any eigenvalue above 1e-6·λ_max against the FP64 Gram of the same centred
float32 patch. A decision quantity is a sum or a square of eigenvalue
functions, so its relative error stays within a small multiple of that; the
mixed tie band ``TIE_TOL["mixed"]`` must be at least 5× the measured error.
"""

from __future__ import annotations

import numpy as np
import pytest

from parity import TIE_TOL
from patch_denoising_b200.synthetic import lowrank_volume


def bf16(a):
    """Round float32 to bfloat16 (nearest, ties to even), returned as float32."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def split_gram(xc):
    """Hermitian Gram of split-bf16 operands; complex data goes through the
    interleaved real embedding, as on the device."""
    if np.iscomplexobj(xc):
        r = np.empty((xc.shape[0], 2 * xc.shape[1]), np.float32)
        r[:, 0::2], r[:, 1::2] = xc.real, xc.imag
    else:
        r = xc.astype(np.float32)
    hi = bf16(r)
    lo = bf16(r - hi)
    h, l = hi.astype(np.float64), lo.astype(np.float64)
    g = h.T @ h + h.T @ l + l.T @ h
    if np.iscomplexobj(xc):
        return (g[0::2, 0::2] + g[1::2, 1::2]) + 1j * (g[0::2, 1::2] - g[1::2, 0::2])
    return g


def max_eig_error(x, p, step):
    worst = 0.0
    X, Y, Z, T = x.shape
    wide = np.complex128 if np.iscomplexobj(x) else np.float64
    for i in range(0, X - p + 1, step):
        for j in range(0, Y - p + 1, step):
            for k in range(0, Z - p + 1, step):
                pt = x[i:i + p, j:j + p, k:k + p].reshape(-1, T)
                xc = (pt - pt.mean(0)).astype(x.dtype)
                e = np.linalg.eigvalsh(xc.astype(wide).conj().T @ xc.astype(wide))
                em = np.linalg.eigvalsh(split_gram(xc))
                ok = e > 1e-6 * e.max()
                worst = max(worst, float((np.abs(em - e)[ok] / e[ok]).max()))
    return worst


CASES = [
    ("MP-PCA 32x32x24x60, patch 5", dict(shape=(32, 32, 24, 60), rank=4, seed=1), 5, 3, np.float32),
    ("NORDIC complex 28x28x17x200, patch 11", dict(shape=(28, 28, 17, 200), rank=6, complex_valued=True,
                                                   noise=3.0, seed=2), 11, 6, np.complex64),
    ("hybrid 24x24x14x300, patch 11", dict(shape=(24, 24, 14, 300), rank=8, noise=3.0, seed=4), 11, 3, np.float32),
]


@pytest.mark.parametrize("name,kw,patch,step,dtype", CASES, ids=[c[0] for c in CASES])
def test_mixed_tie_band_covers_the_split_gram_error(name, kw, patch, step, dtype):
    kw = dict(kw)
    x, _ = lowrank_volume(kw.pop("shape"), kw.pop("rank"), **kw)
    err = max_eig_error(x.astype(dtype), patch, step)
    print(f"{name}: max relative eigenvalue error of the split-bf16 Gram {err:.3g}")
    assert 5 * err <= TIE_TOL["mixed"]
