"""CPU oracle for the space-time low-rank denoising path. TEST INFRASTRUCTURE ONLY.

Nothing in the product package imports this. Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use it, and only
as the checker / the timed CPU reference arm.
"""

from .oracle import (  # noqa: F401
    METHODS,
    atn_shrink,
    denoise,
    eig_analysis,
    eig_synthesis,
    estimate_noise,
    estimate_noise_covered,
    grid_geometry,
    marchenko_pastur_median,
    nordic_threshold,
    patch_locs,
    patch_params,
    qut_level,
    select_patches,
    sure_atn_cost,
    svd_analysis,
    svd_synthesis,
)
