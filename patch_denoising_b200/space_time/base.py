"""Space-time patch denoiser base class (drop-in for ``patch_denoise.space_time.base``).

``BaseSpaceTimeDenoiser.denoise`` keeps the reference signature and return tuple
(space_time/base.py:177-270); the per-patch loop runs on the GPU through
``libpd_b200.so``. ``PatchedArray`` is the reference's strided patch view
(base.py:13-150), kept for callers that use it directly.
"""

from __future__ import annotations

import abc
import logging

import numpy as np
import torch

from .. import _engine

RECOMBINATIONS = ("weighted", "average", "center")


class PatchedArray:
    """Strided sliding view of an array by patches (space_time/base.py:13-150).

    ``grid = (shape - patch) // step + 1`` per axis (1 where the patch covers the
    axis); the patch is clamped to the array; there is no trailing partial patch.
    """

    def __init__(self, array, patch_shape, patch_overlap, dtype=None, padding_mode="edge", **kwargs):
        if isinstance(array, tuple):
            array = np.zeros(array, dtype=dtype)
        self._arr = array
        ps = np.asarray(patch_shape)
        self._po = patch_overlap
        step = ps - np.asarray(patch_overlap)
        if np.any(step < 0):
            raise ValueError("overlap should be smaller than patch on every dimension.")
        if ps.size != array.ndim or step.size != array.ndim:
            raise ValueError(
                "self._ps and step must have the same number of dimensions as the input self._array."
            )
        self._ps = np.minimum(ps, array.shape)
        grid = []
        strides = []
        for n, p, s, st in zip(array.shape, self._ps, step, array.strides):
            covered = p < n
            grid.append(int((n - p) // s + 1) if covered and s > 0 else 1)
            strides.append(st * s if covered else 0)
        self._grid_shape = tuple(grid)
        self.sliding_view = np.lib.stride_tricks.as_strided(
            array, shape=self._grid_shape + tuple(int(p) for p in self._ps),
            strides=tuple(strides) + array.strides,
        )

    @property
    def n_patches(self) -> int:
        """Number of patches."""
        return int(np.prod(self._grid_shape))

    def get_patch(self, idx):
        """Patch at linear index ``idx``."""
        return self.sliding_view[np.unravel_index(idx, self._grid_shape)]

    def idx2slice(self, idx):
        """Slices of the patch at linear index ``idx``."""
        g = np.unravel_index(idx, self._grid_shape)
        return tuple(slice(gi * (p - o), gi * (p - o) + p) for gi, p, o in zip(g, self._ps, self._po))

    def add2patch(self, idx, value):
        """Add ``value`` to the patch, in place."""
        patch = self.get_patch(idx)
        patch += value

    def __getattr__(self, name):
        return getattr(self._arr, name)


# the methods the CUDA patch loop implements (the per-patch hooks of space_time/lowrank.py)
_SUPPORTED_METHODS = ("mp-pca", "hybrid-pca", "raw", "nordic", "optimal", "adaptive")


def _is_float_scalar(x):
    return isinstance(x, (float, np.floating))


class BaseSpaceTimeDenoiser(abc.ABC):
    """Base class of the patch-based low-rank denoisers for dynamic data.

    Parameters
    ----------
    patch_shape: int or tuple
        Spatial patch shape (the time axis is appended), or the full shape.
    patch_overlap: int or tuple
        Overlap of neighbouring patches, same convention.
    recombination: str
        "weighted", "average" or "center".
    precision: str, keyword only
        "fp32" (plain FP32 kernels) or "mixed" (tensor-core Gram + FP32
        refinement). An extension of this package.
    """

    _method = None

    def __init__(self, patch_shape, patch_overlap, recombination="weighted", *, precision="fp32"):
        self.p_shape = patch_shape
        self.p_ovl = patch_overlap
        if recombination not in RECOMBINATIONS:
            raise ValueError("recombination must be one of 'weighted', 'average', 'center'")
        if precision not in ("fp32", "mixed"):
            raise ValueError("precision must be 'fp32' or 'mixed'")
        self.recombination = recombination
        self.precision = precision
        self.input_denoising_kwargs = dict()
        overridden = type(self)._patch_processing is not BaseSpaceTimeDenoiser._patch_processing
        if overridden or self._method not in _SUPPORTED_METHODS:
            raise NotImplementedError(
                f"{type(self).__name__}: a custom per-patch _patch_processing is not supported; the patch loop "
                f"runs on the GPU for the built-in methods only ({', '.join(_SUPPORTED_METHODS)}). Subclass "
                "MPPCADenoiser, HybridPCADenoiser, RawSVDDenoiser, NordicDenoiser, OptimalSVDDenoiser or "
                "AdaptiveDenoiser instead."
            )

    def denoise(self, input_data, mask=None, mask_threshold=50, progbar=None):
        """Denoise ``input_data`` (last axis = time) according to ``mask``.

        Returns ``(denoised, weights, noise_map, rank_map)``: NumPy arrays for a
        NumPy input, CUDA tensors for a tensor input.
        """
        return self._denoise(input_data, mask, mask_threshold, progbar)

    # ------------------------------------------------------------------ internals
    def _method_args(self, data_shape, p_s, device):
        """Per-method arguments of ``_engine.run`` (overridden by subclasses)."""
        return {}

    def _take_result(self, res):
        """Hook for subclasses that keep more of the device result."""

    def _denoise(self, input_data, mask, mask_threshold, progbar):
        if not torch.cuda.is_available():
            raise RuntimeError("patch_denoising_b200 needs a CUDA device (sm_100a); no CPU fallback exists")
        is_torch = isinstance(input_data, torch.Tensor)
        shape = tuple(input_data.shape)
        p_s, p_o = self._get_patch_param(shape)
        if is_torch and input_data.is_cuda:
            device = input_data.device
        else:
            device = torch.device("cuda", torch.cuda.current_device())
        in_dtype = input_data.dtype
        args = self._method_args(shape, p_s, device)
        if not is_torch and mask is None:
            # large host volumes stream: upload, patch ranges and download overlap
            xh = np.ascontiguousarray(input_data)
            if xh.dtype != np.dtype(_engine._NP[_engine.compute_dtype(in_dtype)]):
                xh = xh.astype(_engine._NP[_engine.compute_dtype(in_dtype)])
            with torch.cuda.device(device):
                streamed = _engine.run_host(self._method, xh, p_s, p_o, self.recombination, mask_threshold,
                                            precision=self.precision, device=device, **args)
            if streamed is not None:
                (out, weights, noise_map, rank_map), res = streamed
                self.patch_index_ = res.patch_index.cpu().numpy()
                self.patch_rank_ = res.patch_rank.cpu().numpy()
                self.patch_noise_ = res.patch_noise.cpu().numpy()
                self._take_result(res)
                if np.dtype(in_dtype) != out.dtype:
                    out = out.astype(in_dtype)
                return out, weights, noise_map, rank_map
        x = _engine.to_device(input_data, device, _engine.compute_dtype(in_dtype))
        m = self._device_mask(mask, shape, device)
        with torch.cuda.device(device):
            res = _engine.run(self._method, x, p_s, p_o, self.recombination, m, mask_threshold,
                              precision=self.precision, **args)
        self.patch_index_ = res.patch_index
        self.patch_rank_ = res.patch_rank
        self.patch_noise_ = res.patch_noise
        self._take_result(res)
        if progbar is not None and progbar is not False:
            progbar.reset(total=int(res.patch_index.numel()))
            progbar.update(int(res.patch_index.numel()))
        if is_torch:
            out = res.out
            if in_dtype in (torch.float64, torch.complex128):
                out = out.to(in_dtype)
            return out, res.weights, res.noise_map, res.rank_map
        # one time window (a patch spans every frame): the maps are constant
        # along frames, so only their spatial part is copied back
        # (the noise map of "center" recombination sits at the centre frame only,
        # and a 4D mask zeroes it frame by frame)
        one_window = p_s[-1] >= shape[-1]
        nm_flat = one_window and self.recombination != "center" and (m is None or m.dim() < len(shape))
        nm_d = res.noise_map[..., 0] if nm_flat else res.noise_map
        rm_d = res.rank_map[..., 0] if one_window else res.rank_map
        out, weights, noise_map, rank_map, pidx, prank, pnoise = _engine.to_host(
            [res.out, res.weights, nm_d, rm_d, res.patch_index, res.patch_rank, res.patch_noise])
        if nm_flat:
            noise_map = _engine.spread_over_frames(noise_map, shape)
        if one_window:
            rank_map = _engine.spread_over_frames(rank_map, shape)
        if np.dtype(in_dtype) != out.dtype:
            out = out.astype(in_dtype)
        self.patch_index_, self.patch_rank_, self.patch_noise_ = pidx, prank, pnoise
        return out, weights, noise_map, rank_map

    @staticmethod
    def _device_mask(mask, data_shape, device):
        """Mask normalisation of space_time/base.py:202-211, as uint8 on the device."""
        if mask is None:
            return None
        mshape = tuple(mask.shape)
        if mshape != tuple(data_shape) and mshape != tuple(data_shape[:-1]):
            raise ValueError(f"Mask shape {mshape} is incompatible with input {tuple(data_shape)}.")
        if isinstance(mask, torch.Tensor):
            return (mask != 0).to(device=device, dtype=torch.uint8).contiguous()
        return torch.from_numpy(np.ascontiguousarray(np.asarray(mask) != 0).view(np.uint8)).to(device)

    @staticmethod
    def _spatial_map(noise_std, data_shape, device):
        """``noise_std`` (float or spatial array) as a float64 device map."""
        spatial = tuple(data_shape[:-1])
        if _is_float_scalar(noise_std):
            arr = np.full(spatial, float(noise_std), dtype=np.float64)
        elif isinstance(noise_std, torch.Tensor):
            return torch.broadcast_to(noise_std.to(device=device, dtype=torch.float64), spatial).contiguous()
        elif isinstance(noise_std, np.ndarray):
            arr = np.array(np.broadcast_to(np.asarray(noise_std, dtype=np.float64), spatial))
        else:
            raise TypeError(f"noise_std must be a float or an array, not {type(noise_std).__name__}")
        return torch.from_numpy(np.ascontiguousarray(arr)).to(device)

    def _patch_processing(self, patch, patch_idx=None, **kwargs):
        """Per-patch plug-in of the reference (base.py:352-357).

        Here the whole patch loop runs inside libpd_b200.so; subclasses select the
        method through ``_method`` instead of overriding this hook.
        """
        raise NotImplementedError("per-patch processing runs on the GPU inside libpd_b200.so")

    def _get_patch_param(self, data_shape):
        """Patch shape and overlap as full tuples (space_time/base.py:359-384)."""
        pp = [None, None]
        for i, attr in enumerate(["p_shape", "p_ovl"]):
            p = getattr(self, attr)
            if isinstance(p, list):
                p = tuple(p)
            elif isinstance(p, (int, np.integer)):
                p = (p,) * (len(data_shape) - 1)
            if len(p) == len(data_shape) - 1:
                p = (*p, data_shape[-1])
            pp[i] = tuple(int(v) for v in p)
        if np.prod(pp[0][:-1]) < data_shape[-1]:
            logging.warning(
                f"the number of voxel in patch ({np.prod(pp[0])}) is smaller than the"
                f" last dimension ({data_shape[-1]}), this makes an ill-conditioned"
                "matrix for SVD.",
                stacklevel=2,
            )
        return tuple(pp)
