"""Differentiable low-rank patch denoising (an extension: the reference has no gradients).

``lowrank_denoise`` is a ``torch.autograd.Function`` over the whole path of
``BaseSpaceTimeDenoiser.denoise`` (space_time/base.py:177-270): patch extraction,
centring, spectral shrinkage of each Casorati matrix, synthesis, recombination
and normalisation. Two shrinkages are offered:

* ``shrink="soft"``: singular-value soft thresholding s~ = max(s - tau_p, 0)
  with tau_p = threshold_scale * stdest_p * (sqrt(M) + sqrt(T)), stdest_p the
  patch's root-mean-square noise_std and sqrt(M) + sqrt(T) the top edge of the
  singular values of an M x T noise matrix of unit variance (Marchenko-Pastur).
  This is the adaptive trace-norm shrinkage of AdaptiveDenoiser
  (space_time/lowrank.py:459-461) at gamma = 1 with a fixed tau, and the
  forward runs on that kernel. The output is continuous in threshold_scale, so
  its gradient is defined.
* ``shrink="hard"``: the MP-PCA rule (space_time/lowrank.py:42-63): the top
  components selected by the rule are kept unchanged. The selection is
  piecewise constant in the input and in threshold_scale, so the input
  gradient is that of the projection onto the kept components and the
  threshold gradient is zero.

The backward (``pd_lowrank_backward``) recomputes each patch's factorisation
instead of storing it. The recombination weights theta (constant for
"average", 1 / (2 + rank) for "weighted") are treated as constants: they change
only where a rank changes. Real float32 data, M > T and T <= 128.

``sure_tune_threshold`` tunes threshold_scale by gradient descent on a
Monte-Carlo SURE estimate of the mean-squared error (Ramani, Blu & Unser, IEEE
TIP 2008), whose gradient flows through this backward.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from .. import _engine, _lib
from .base import BaseSpaceTimeDenoiser

_SHRINK = {"soft": 0, "hard": 1}


def _vp(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def patch_geometry(data_shape, patch_shape, patch_overlap):
    """Full (time-appended) patch shape and overlap, as BaseSpaceTimeDenoiser._get_patch_param."""
    nd = len(data_shape)
    out = []
    for p in (patch_shape, patch_overlap):
        if isinstance(p, list):
            p = tuple(p)
        elif isinstance(p, (int, np.integer)):
            p = (int(p),) * (nd - 1)
        if len(p) == nd - 1:
            p = (*p, data_shape[-1])
        out.append(tuple(int(v) for v in p))
    return tuple(out)


class LowRankDenoiseFunction(torch.autograd.Function):
    """(x, threshold_scale) -> denoised volume; see the module docstring."""

    @staticmethod
    def forward(ctx, x, threshold_scale, cfg):
        p_s, p_o = cfg["p_s"], cfg["p_o"]
        g = _engine.geometry(tuple(x.shape), p_s, p_o)
        M, T = int(g.rows), int(g.cols)
        scale = float(threshold_scale)
        edge = math.sqrt(M) + math.sqrt(T)
        with torch.cuda.device(x.device):
            if cfg["shrink"] == "soft":
                ad = {"mode": "qut", "gamma": [1.0], "qut_level": scale * edge}
                res = _engine.run("adaptive", x, p_s, p_o, cfg["recombination"], None, 50,
                                  noise_std=cfg["noise_map"], adaptive=ad)
            else:
                res = _engine.run("mp-pca", x, p_s, p_o, cfg["recombination"], None, 50, threshold_scale=scale)
        ctx.save_for_backward(x, res.weights, res.patch_index, res.patch_rank)
        ctx.cfg = cfg
        ctx.level = scale * edge
        ctx.edge = edge
        ctx.scale_dtype = threshold_scale.dtype
        return res.out

    @staticmethod
    def backward(ctx, gout):
        x, weights, plist, prank = ctx.saved_tensors
        cfg = ctx.cfg
        lib = _lib.load()
        dev = x.device
        g = _engine.geometry(tuple(x.shape), cfg["p_s"], cfg["p_o"])
        gp = ctypes.byref(g)
        n_sel = int(plist.numel())
        gin = torch.zeros_like(x)
        dlevel = torch.zeros(max(n_sel, 1), dtype=torch.float64, device=dev)
        need = ctypes.c_size_t()
        _lib.check(lib.pd_lowrank_backward_workspace_size(gp, n_sel, ctypes.byref(need)))
        ws = torch.empty(max(need.value, 1), dtype=torch.uint8, device=dev)
        gout = gout.to(torch.float32).contiguous()
        with torch.cuda.device(dev):
            stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
            _lib.check(lib.pd_lowrank_backward(
                gp, _lib.RECOMBINATION[cfg["recombination"]], _SHRINK[cfg["shrink"]], _vp(x),
                _vp(cfg["noise_map"]), float(ctx.level), _vp(plist), n_sel, _vp(prank), _vp(weights), _vp(gout),
                _vp(gin), _vp(dlevel), _vp(ws), need.value, stream))
            if n_sel:
                _engine._queue_error_check([ws], dev)
        grad_x = gin if ctx.needs_input_grad[0] else None
        grad_s = None
        if ctx.needs_input_grad[1]:
            grad_s = (dlevel[:n_sel].sum() * ctx.edge).to(ctx.scale_dtype)
        return grad_x, grad_s, None


def lowrank_denoise(x, patch_shape, patch_overlap, threshold_scale=1.0, noise_std=None, *, shrink="soft",
                    recombination="average"):
    """Differentiable denoising of a real (X, Y, Z, T) CUDA tensor.

    ``threshold_scale``: float or 0-d tensor (a leaf with ``requires_grad`` to
    learn it). ``noise_std``: float or spatial map (required for "soft").
    Returns the denoised volume (float32; NaN where no patch covers a voxel,
    as in the reference).
    """
    if shrink not in _SHRINK:
        raise ValueError("shrink must be 'soft' or 'hard'")
    if recombination not in ("weighted", "average"):
        raise ValueError("the differentiable path needs 'weighted' or 'average' recombination")
    if not isinstance(x, torch.Tensor) or x.device.type != "cuda":
        raise RuntimeError("lowrank_denoise runs on a CUDA tensor")
    if x.is_complex():
        raise NotImplementedError("the differentiable path handles real volumes")
    if shrink == "soft" and noise_std is None:
        raise ValueError("the soft threshold needs noise_std")
    xs = x.to(torch.float32).contiguous()
    p_s, p_o = patch_geometry(tuple(x.shape), patch_shape, patch_overlap)
    nmap = None
    if noise_std is not None:
        nmap = BaseSpaceTimeDenoiser._spatial_map(noise_std, tuple(x.shape), x.device)
    cfg = {"p_s": p_s, "p_o": p_o, "shrink": shrink, "recombination": recombination, "noise_map": nmap}
    if not isinstance(threshold_scale, torch.Tensor):
        threshold_scale = torch.tensor(float(threshold_scale), device=x.device)
    return LowRankDenoiseFunction.apply(xs, threshold_scale, cfg)


class LowRankDenoiseLayer(torch.nn.Module):
    """``lowrank_denoise`` with a learnable ``threshold_scale`` (initial value ``init_scale``)."""

    def __init__(self, patch_shape, patch_overlap, init_scale=1.0, *, shrink="soft", recombination="average"):
        super().__init__()
        self.patch_shape, self.patch_overlap = patch_shape, patch_overlap
        self.shrink, self.recombination = shrink, recombination
        self.threshold_scale = torch.nn.Parameter(torch.tensor(float(init_scale)))

    def forward(self, x, noise_std=None):
        return lowrank_denoise(x, self.patch_shape, self.patch_overlap, self.threshold_scale, noise_std,
                               shrink=self.shrink, recombination=self.recombination)


def mc_sure(layer, y, noise_std, eps=None, probe=None):
    """Monte-Carlo SURE of ``layer`` at ``y`` (Ramani, Blu & Unser 2008):
    ||f(y) - y||^2 + 2 sigma^2 b^T (f(y + eps b) - f(y)) / eps - N sigma^2 over
    the voxels every patch covers, b a fixed +-1 probe. Differentiable in the
    layer's threshold_scale through the backward pass."""
    sigma = float(noise_std)
    if eps is None:
        eps = 1e-3 * float(y.abs().max())
    if probe is None:
        gen = torch.Generator(device=y.device).manual_seed(0)
        probe = torch.randint(0, 2, y.shape, generator=gen, device=y.device, dtype=torch.int8).to(y.dtype) * 2 - 1
    f0 = layer(y, sigma)
    f1 = layer(y + eps * probe, sigma)
    ok = torch.isfinite(f0) & torch.isfinite(f1)
    n = ok.sum()
    fid = torch.where(ok, f0 - y, torch.zeros_like(y)).pow(2).sum()
    div = torch.where(ok, probe * (f1 - f0), torch.zeros_like(y)).sum() / eps
    return fid + 2 * sigma**2 * div - n * sigma**2


def sure_tune_threshold(y, noise_std, patch_shape, patch_overlap, *, init_scale=1.0, steps=20, lr=0.05,
                        shrink="soft", recombination="average"):
    """Tune threshold_scale by ``steps`` gradient steps on log(threshold_scale)
    minimising the Monte-Carlo SURE of the soft-threshold denoiser. Returns
    (final scale, list of (scale, SURE) per step)."""
    log_s = torch.nn.Parameter(torch.tensor(math.log(float(init_scale)), device=y.device))
    opt = torch.optim.Adam([log_s], lr=lr)
    history = []
    for _ in range(steps):
        opt.zero_grad()
        scale = log_s.exp()
        risk = mc_sure(lambda v, s: lowrank_denoise(v, patch_shape, patch_overlap, scale, s, shrink=shrink,
                                                    recombination=recombination), y, noise_std)
        risk.backward()
        history.append((float(scale), float(risk)))
        opt.step()
    return float(log_s.exp()), history
