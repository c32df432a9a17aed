"""Low-rank denoisers (drop-in for ``patch_denoise.space_time.lowrank``).

Same constructors, ``denoise`` signatures and errors as the reference classes;
the per-patch work runs in libpd_b200.so.
"""

from __future__ import annotations

import numpy as np

from .. import _engine, _lib
from .base import BaseSpaceTimeDenoiser, _is_float_scalar


class MPPCADenoiser(BaseSpaceTimeDenoiser):
    """Marchenko-Pastur PCA thresholding (space_time/lowrank.py:28-63).

    ``threshold_scale`` multiplies the threshold on the eigenvalues.
    """

    _method = "mp-pca"

    def __init__(self, patch_shape, patch_overlap, threshold_scale, **kwargs):
        super().__init__(patch_shape, patch_overlap, **kwargs)
        self.input_denoising_kwargs["threshold_scale"] = threshold_scale

    def _method_args(self, data_shape, p_s, device):
        return {"threshold_scale": float(self.input_denoising_kwargs["threshold_scale"])}


class HybridPCADenoiser(BaseSpaceTimeDenoiser):
    """Hybrid-PCA thresholding with a noise prior (space_time/lowrank.py:67-119)."""

    _method = "hybrid-pca"

    def denoise(self, input_data, mask=None, mask_threshold=50, noise_std=1.0, progbar=None):
        """Denoise with a noise standard deviation (float or spatial map)."""
        self.input_denoising_kwargs["noise_std"] = noise_std
        return self._denoise(input_data, mask, mask_threshold, progbar)

    def _method_args(self, data_shape, p_s, device):
        ns = self.input_denoising_kwargs["noise_std"]
        return {"noise_std": self._spatial_map(ns, data_shape, device)}


class RawSVDDenoiser(BaseSpaceTimeDenoiser):
    """Hard singular-value thresholding (space_time/lowrank.py:123-184)."""

    _method = "raw"

    def __init__(self, patch_shape, patch_overlap, threshold_value=1.0, recombination="weighted", **kwargs):
        self._threshold_val = threshold_value
        super().__init__(patch_shape, patch_overlap, recombination, **kwargs)

    def denoise(self, input_data, mask=None, mask_threshold=50, threshold_scale=1.0, progbar=None):
        """Denoise with threshold ``threshold_value * threshold_scale``."""
        self._threshold = self._threshold_val * threshold_scale
        return self._denoise(input_data, mask, mask_threshold, progbar)

    def _method_args(self, data_shape, p_s, device):
        return {"threshold": float(self._threshold)}


class NordicDenoiser(RawSVDDenoiser):
    """NORDIC: hard thresholding at a Monte-Carlo noise level (space_time/lowrank.py:188-246).

    The level is ``noise_std * mean_n sigma_max(G_n)`` over ``n_iter_threshold``
    standard Gaussian draws ``G_n`` of ``prod(patch_shape incl. time) x T``,
    computed on the GPU (counter-based generator seeded from NumPy's global
    generator, so ``np.random.seed`` makes a call reproducible, as in the
    reference). The threshold never leaves the device (no host round trip in
    the call); ``mc_max_sval_`` reads the level back on first access. ``mc_max_sval`` (extension) supplies the
    level directly.
    """

    _method = "nordic"

    def denoise(self, input_data, mask=None, mask_threshold=50, noise_std=1.0, n_iter_threshold=10,
                progbar=None, mc_max_sval=None):
        """Denoise with the NORDIC threshold."""
        if isinstance(noise_std, np.ndarray):
            noise_std = np.mean(noise_std)
        if not _is_float_scalar(noise_std):
            raise ValueError(
                "For NORDIC the noise level must be either an"
                " array or a float specifying the std in the volume."
            )
        shape = tuple(input_data.shape)
        patch_shape, _ = self._get_patch_param(shape)
        self._nordic = None
        self._level = None
        if mc_max_sval is None:
            seed = int(np.random.randint(0, 2**62))
            self._nordic = {"noise_std": float(noise_std), "rows": int(np.prod(patch_shape)),
                            "n_iter": int(n_iter_threshold), "seed": seed}
            self._threshold = 0.0
            self._mc_max_sval = None
        else:
            self._mc_max_sval = float(mc_max_sval)
            self._threshold = float(noise_std) * float(mc_max_sval)
        return self._denoise(input_data, mask, mask_threshold, progbar)

    @property
    def mc_max_sval_(self):
        """Mean largest singular value of the Monte-Carlo draws of the last call."""
        if self._mc_max_sval is None and self._level is not None:
            self._mc_max_sval = float(self._level[0].item())
        return self._mc_max_sval

    def _method_args(self, data_shape, p_s, device):
        return {"threshold": float(self._threshold), "nordic": self._nordic}

    def _take_result(self, res):
        self._level = res.level


class OptimalSVDDenoiser(BaseSpaceTimeDenoiser):
    """Gavish-Donoho optimal shrinkage (space_time/lowrank.py:284-407).

    ``loss`` is "fro", "nuc" or "ope".
    """

    _method = "optimal"
    _LOSSES = ("fro", "nuc", "ope")

    def __init__(self, patch_shape, patch_overlap, loss="fro", recombination="weighted", **kwargs):
        super().__init__(patch_shape, patch_overlap, recombination=recombination, **kwargs)
        if loss not in self._LOSSES:
            raise KeyError(loss)
        self.loss = loss

    def denoise(self, input_data, mask=None, mask_threshold=50, noise_std=None, eps_marshenko_pastur=1e-7,
                progbar=None):
        """Denoise by optimal shrinkage; ``noise_std`` (float or map) replaces the MP estimate."""
        shape = tuple(input_data.shape)
        p_s, _ = self._get_patch_param(shape)
        beta = p_s[-1] / np.prod(p_s[:-1]) if len(p_s) == len(shape) else shape[-1] / np.prod(p_s)
        self.input_denoising_kwargs["mp_median"] = _engine.mp_median(beta, eps_marshenko_pastur)
        self.input_denoising_kwargs["noise_std"] = noise_std
        return self._denoise(input_data, mask, mask_threshold, progbar)

    def _method_args(self, data_shape, p_s, device):
        ns = self.input_denoising_kwargs["noise_std"]
        return {
            "loss": self.loss,
            "mp_med": float(self.input_denoising_kwargs["mp_median"]),
            "noise_std": None if ns is None else self._spatial_map(ns, data_shape, device),
        }


class AdaptiveDenoiser(BaseSpaceTimeDenoiser):
    """Adaptive trace-norm shrinkage d = s max(1 - (tau/s)^gamma, 0) (space_time/lowrank.py:536-636).

    ``method`` "sure" / "gsure": for every candidate in ``gamma0`` (an iterable,
    as in the reference) log tau minimises the SURE / GSURE cost from ``tau0``
    (default log of the median singular value); the lowest cost wins. "qut":
    tau = stdest x the (1 - 1/sqrt(log max(M, T)))-quantile of the largest
    singular value of ``nbsim`` Gaussian M x T draws (one set per call, seeded
    from NumPy's global generator, ``qut_level_``; ``qut_level`` supplies it);
    gamma is ``gamma0`` when it is a float, else minimises the cost. stdest is
    sqrt(mean noise_std^2) over the patch. The cost minimisation runs on the
    device (bracketing line search + Brent) in place of scipy's BFGS.
    """

    _method = "adaptive"
    _SUPPORTED_METHOD = ["sure", "qut", "gsure"]

    def __init__(self, patch_shape, patch_overlap, method="SURE", recombination="weighted", nbsim=500, *,
                 precision="fp32"):
        super().__init__(patch_shape, patch_overlap, recombination, precision=precision)
        if method.lower() not in self._SUPPORTED_METHOD:
            raise ValueError(f"Unsupported method: '{method}', use any of {self._SUPPORTED_METHOD}")
        self.input_denoising_kwargs["method"] = method.lower()
        self.input_denoising_kwargs["nbsim"] = nbsim
        self.qut_level_ = None

    def denoise(self, input_data, mask=None, mask_threshold=50, tau0=None, noise_std=None, gamma0=None,
                progbar=None, qut_level=None):
        """Denoise with adaptive shrinkage; ``noise_std`` (float or spatial map) is required."""
        method = self.input_denoising_kwargs["method"]
        if noise_std is None:  # the reference squares it
            raise TypeError("unsupported operand type(s) for ** or pow(): 'NoneType' and 'int'")
        self.input_denoising_kwargs["gamma0"] = gamma0
        self.input_denoising_kwargs["tau0"] = tau0
        self.input_denoising_kwargs["noise_std"] = noise_std
        ad = {"mode": method}
        if method == "qut":
            ad["gamma"] = [float(gamma0)] if isinstance(gamma0, (float, np.floating)) else []
            self._qut_seed = None if qut_level is not None else int(np.random.randint(0, 2**62))
            self.qut_level_ = None if qut_level is None else float(qut_level)
        else:
            gam = [float(g) for g in gamma0]  # TypeError for None or a scalar, as the reference's loop
            if not gam:
                raise UnboundLocalError("no candidate gamma: gamma0 is empty")
            if len(gam) > _lib.ADAPTIVE_MAX_GAMMA:
                raise NotImplementedError(f"at most {_lib.ADAPTIVE_MAX_GAMMA} candidate gammas")
            ad["gamma"] = gam
            ad["tau0"] = None if tau0 is None else float(np.asarray(tau0).reshape(-1)[0])
        self._adaptive = ad
        return self._denoise(input_data, mask, mask_threshold, progbar)

    def _method_args(self, data_shape, p_s, device):
        ad = dict(self._adaptive)
        if ad["mode"] == "qut":
            if self.qut_level_ is None:
                rows, cols = int(np.prod(p_s[:-1])), int(p_s[-1])
                self.qut_level_ = _engine.adaptive_qut_level(rows, cols, int(self.input_denoising_kwargs["nbsim"]),
                                                             self._qut_seed, device, self.precision)
            ad["qut_level"] = self.qut_level_
        ns = self.input_denoising_kwargs["noise_std"]
        return {"noise_std": self._spatial_map(ns, data_shape, device), "adaptive": ad}
