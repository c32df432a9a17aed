"""Host utilities of the space-time path."""

from __future__ import annotations

from .. import _engine


def marchenko_pastur_median(beta, eps=1e-7):
    """Median of the Marchenko-Pastur law of aspect ratio ``beta`` in [0, 1].

    Same 5-point dichotomy as the reference (space_time/utils.py:149-204), on the
    closed-form CDF instead of numerical quadrature; computed in libpd_b200.so.
    """
    return _engine.mp_median(beta, eps)
