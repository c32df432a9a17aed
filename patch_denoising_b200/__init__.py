"""B200-native (sm_100a) space-time low-rank denoising.

Drop-in for the space-time path of paquiteau/patch-denoising: the same denoiser
classes, functional API and method registry, with the per-patch work running in
hand-written CUDA kernels (``libpd_b200.so``, C ABI in
``include/patch_denoise_b200.h``).
"""

__version__ = "0.1.0"

from .denoise import (  # noqa: E402
    adaptive_thresholding,
    hybrid_pca,
    mp_pca,
    nordic,
    optimal_thresholding,
    raw_svt,
)
from .space_time import (  # noqa: E402
    HybridPCADenoiser,
    MPPCADenoiser,
    NordicDenoiser,
    OptimalSVDDenoiser,
    RawSVDDenoiser,
)

__all__ = [
    "mp_pca",
    "hybrid_pca",
    "raw_svt",
    "nordic",
    "optimal_thresholding",
    "adaptive_thresholding",
    "MPPCADenoiser",
    "HybridPCADenoiser",
    "RawSVDDenoiser",
    "NordicDenoiser",
    "OptimalSVDDenoiser",
]
