"""``main_gpu`` with the signature of the reference GPU driver (gpu/main.py:186-250).

It runs the same B200 kernels as the denoiser classes, so its results follow the
CPU reference path (mean over voxels, theta = 1/(2+maxidx)), not the divergent
conventions of the reference's torch modules.
"""

from __future__ import annotations

from ..space_time.lowrank import MPPCADenoiser, OptimalSVDDenoiser


def main_gpu(args, input_data, mask, noise_map, batch_size=32, compile=False, **kwargs):
    """Denoise ``input_data`` as ``args.method`` describes; returns ``(out, weights, None)``."""
    method = args.method
    if method is not None and "optimal" in method:
        den = OptimalSVDDenoiser(args.patch_shape, args.patch_overlap, loss=method.split("-")[-1],
                                 recombination=args.recombination)
        out, weights, _, _ = den.denoise(input_data, mask=mask, mask_threshold=args.mask_threshold,
                                         noise_std=noise_map if method == "optimal-fro-noise" else None)
    elif method in ("mppca", "mp-pca"):
        den = MPPCADenoiser(args.patch_shape, args.patch_overlap,
                            threshold_scale=float(kwargs.get("threshold_scale", 1.0)),
                            recombination=args.recombination)
        out, weights, _, _ = den.denoise(input_data, mask=mask, mask_threshold=args.mask_threshold)
    else:
        raise ValueError(f"method {method} is not supported on GPU. ")
    return out, weights, None
