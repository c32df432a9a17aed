"""Space-time denoisers (drop-in for ``patch_denoise.space_time``)."""

from .base import BaseSpaceTimeDenoiser, PatchedArray
from .lowrank import (
    AdaptiveDenoiser,
    HybridPCADenoiser,
    MPPCADenoiser,
    NordicDenoiser,
    OptimalSVDDenoiser,
    RawSVDDenoiser,
)
from .utils import estimate_noise, marchenko_pastur_median

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
]
