"""Space-time denoisers (drop-in for ``patch_denoise.space_time``)."""

from .base import BaseSpaceTimeDenoiser, PatchedArray
from .diff import LowRankDenoiseFunction, LowRankDenoiseLayer, lowrank_denoise, mc_sure, sure_tune_threshold
from .lowrank import (
    AdaptiveDenoiser,
    HybridPCADenoiser,
    MPPCADenoiser,
    NordicDenoiser,
    OptimalSVDDenoiser,
    RawSVDDenoiser,
)
from .utils import (
    eig_analysis,
    eig_synthesis,
    estimate_noise,
    get_patch_locs,
    marchenko_pastur_median,
    svd_analysis,
    svd_synthesis,
)

__all__ = [
    "BaseSpaceTimeDenoiser",
    "PatchedArray",
    "MPPCADenoiser",
    "HybridPCADenoiser",
    "RawSVDDenoiser",
    "NordicDenoiser",
    "OptimalSVDDenoiser",
    "AdaptiveDenoiser",
    "marchenko_pastur_median",
    "estimate_noise",
    "get_patch_locs",
    "svd_analysis",
    "svd_synthesis",
    "eig_analysis",
    "eig_synthesis",
    "LowRankDenoiseFunction",
    "LowRankDenoiseLayer",
    "lowrank_denoise",
    "mc_sure",
    "sure_tune_threshold",
]
