"""Batched denoising of many volumes of uneven shape in one set of launches.

``denoise_batch(volumes, method, ...)`` runs the same method on every volume
(each with its own shape, frame count, mask and noise level) through
``pd_denoise_batch``: the selected patches of all volumes form one work list
and every patch kernel (mean, Gram, eigensolver, synthesis) covers all volumes
in one launch, reading each patch's volume from a device table. Results equal
per-volume ``denoise`` calls. The reference denoises one volume per call
(space_time/base.py:177-270).

The launch shape is tuned per workload (``tuning="auto"``): ``autotune`` times
the candidate settings of ``pd_batch_tuning`` on the workload itself and keeps
the fastest, cached by the volumes' shapes, method and patch parameters.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _engine, _lib
from .space_time.base import BaseSpaceTimeDenoiser
from .space_time.diff import patch_geometry

METHODS = ("mp-pca", "hybrid-pca", "raw", "optimal")
_TUNED = {}  # workload signature -> pd_batch_tuning fields


def _vp(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


class _Prepared:
    """Device buffers and the pd_volume records of one batched call."""

    def __init__(self, volumes, method, patch_shape, patch_overlap, recombination, masks, mask_threshold,
                 threshold_value, threshold_scale, noise_std, loss, eps_mp, device):
        lib = _lib.load()
        s = ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)
        self.items = []
        self.recs = (_lib.Volume * len(volumes))()
        cplx = None
        for i, vol in enumerate(volumes):
            x = _engine.to_device(vol, device, _engine.compute_dtype(vol.dtype))
            if cplx is None:
                cplx = x.is_complex()
            elif cplx != x.is_complex():
                raise ValueError("a batch is either all real or all complex")
            shape = tuple(x.shape)
            p_s, p_o = patch_geometry(shape, patch_shape, patch_overlap)
            g = _engine.geometry(shape, p_s, p_o)
            gp = ctypes.byref(g)
            mask = None if masks is None else masks[i]
            m = BaseSpaceTimeDenoiser._device_mask(mask, shape, device)
            need = ctypes.c_size_t()
            _lib.check(lib.pd_select_workspace_size(gp, ctypes.byref(need)))
            sws = torch.empty(max(need.value, 1), dtype=torch.uint8, device=device)
            plist = torch.empty(max(int(g.n_patches), 1), dtype=torch.int32, device=device)
            count = torch.zeros(1, dtype=torch.int32, device=device)
            mask_4d = 1 if (m is not None and m.dim() == len(shape)) else 0
            _lib.check(lib.pd_select_patches(gp, _vp(m), mask_4d, float(mask_threshold), _vp(plist), _vp(count),
                                             _vp(sws), need.value, s))
            self.items.append(dict(x=x, g=g, mask=m, mask_4d=mask_4d, plist=plist, count=count, shape=shape,
                                   p_s=p_s))
        torch.cuda.current_stream(device).synchronize()  # the selected counts, all volumes at once
        self.cplx = bool(cplx)
        for i, it in enumerate(self.items):
            g, shape = it["g"], it["shape"]
            n_sel = int(it["count"].item())
            nvox = int(np.prod(shape[:-1]))
            it.update(
                n_sel=n_sel,
                out=torch.zeros(shape, dtype=it["x"].dtype, device=device),
                wacc=torch.zeros(nvox * int(g.grid[3]), dtype=torch.float32, device=device),
                nctr=torch.zeros(shape, dtype=torch.float32, device=device),
                rank_map=torch.zeros(shape, dtype=torch.int32, device=device),
                prank=torch.zeros(max(n_sel, 1), dtype=torch.int32, device=device),
                pnoise=torch.zeros(max(n_sel, 1), dtype=torch.float32, device=device),
            )
            it["nacc"] = torch.zeros_like(it["wacc"])
            ns = None
            if noise_std is not None:
                nsv = noise_std[i] if isinstance(noise_std, (list, tuple)) else noise_std
                ns = BaseSpaceTimeDenoiser._spatial_map(nsv, shape, device)
            it["ns"] = ns
            r = self.recs[i]
            r.geometry = g
            r.d_in, r.d_noise_std, r.d_patch_list = _vp(it["x"]), _vp(ns), _vp(it["plist"])
            r.n_selected = n_sel
            r.d_out_acc, r.d_weight_acc, r.d_noise_acc = _vp(it["out"]), _vp(it["wacc"]), _vp(it["nacc"])
            r.d_noise_ctr, r.d_rank_map = _vp(it["nctr"]), _vp(it["rank_map"])
            r.d_patch_rank, r.d_patch_noise = _vp(it["prank"]), _vp(it["pnoise"])
            r.threshold = float(threshold_value)
            if method == "optimal":
                p_s = it["p_s"]
                r.mp_median = _engine.mp_median(p_s[-1] / np.prod(p_s[:-1]), eps_mp)
        self.prm = _lib.Params()
        self.prm.method = _lib.METHOD[method]
        self.prm.recombination = _lib.RECOMBINATION[recombination]
        self.prm.loss = _lib.LOSS[loss]
        self.prm.precision = _lib.PRECISION["fp32"]
        self.prm.is_complex = 1 if self.cplx else 0
        self.prm.has_prior = 1 if noise_std is not None else 0
        self.prm.threshold_scale = float(threshold_scale)
        self.recombination = recombination
        self.device = device

    def zero(self):
        for it in self.items:
            for k in ("out", "wacc", "nacc", "nctr", "rank_map"):
                it[k].zero_()

    def run(self, tuning):
        lib = _lib.load()
        tn = _lib.BatchTuning(**tuning)
        need = ctypes.c_size_t()
        _lib.check(lib.pd_denoise_batch_workspace_size(self.recs, len(self.items), ctypes.byref(self.prm),
                                                       tn.chunk_patches, ctypes.byref(need)))
        ws = torch.empty(max(need.value, 1), dtype=torch.uint8, device=self.device)
        s = ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        _lib.check(lib.pd_denoise_batch(self.recs, len(self.items), ctypes.byref(self.prm), ctypes.byref(tn),
                                        _vp(ws), need.value, s))
        _engine._queue_error_check([ws], self.device)

    def finalize(self):
        lib = _lib.load()
        s = ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        results = []
        for it in self.items:
            w = torch.empty(it["shape"], dtype=torch.float32, device=self.device)
            nm = torch.empty_like(w)
            _lib.check(lib.pd_finalize(ctypes.byref(it["g"]), ctypes.byref(self.prm), _vp(it["out"]),
                                       _vp(it["wacc"]), _vp(it["nacc"]), _vp(it["nctr"]), _vp(w), _vp(nm),
                                       _vp(it["mask"]), it["mask_4d"], s))
            results.append((it["out"], w, nm, it["rank_map"], it["prank"][: it["n_sel"]]))
        return results

    def signature(self, method):
        return (method, self.recombination, self.cplx,
                tuple((it["shape"], it["p_s"], it["n_sel"]) for it in self.items))


CANDIDATES = [dict(synth_row_blocks=b, order_by_cost=1, chunk_patches=0) for b in (0, 1, 2, 4, 8)] + \
             [dict(synth_row_blocks=0, order_by_cost=0, chunk_patches=0)]


def autotune(prep, method, repeats=2):
    """Time every candidate pd_batch_tuning on the prepared workload (CUDA
    events, best of ``repeats``); return the fastest and the timings."""
    timings = []
    for cand in CANDIDATES:
        best = float("inf")
        for _ in range(repeats):
            prep.zero()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            prep.run(cand)
            b.record()
            b.synchronize()
            best = min(best, a.elapsed_time(b))
        timings.append((cand, best))
    choice = min(timings, key=lambda cb: cb[1])[0]
    _TUNED[prep.signature(method)] = choice
    return choice, timings


def denoise_batch(volumes, method, patch_shape, patch_overlap, recombination="weighted", masks=None,
                  mask_threshold=50, *, threshold_scale=1.0, threshold_value=1.0, noise_std=None, loss="fro",
                  eps_marshenko_pastur=1e-7,
                  tuning="auto", device=None, return_tuning=False):
    """Denoise a list of volumes (NumPy arrays or CUDA tensors) with one method.

    Returns a list of ``(denoised, weights, noise_map, rank_map)`` CUDA tensors
    (per volume) and, with ``return_tuning``, the pd_batch_tuning used.
    ``threshold_scale`` (MP-PCA), ``threshold_value`` (raw), ``loss`` (optimal)
    as in the single-volume denoisers. ``noise_std``: one float / map for all
    volumes, or a list (hybrid, optimal).
    ``tuning``: "auto" (autotuned, cached per workload), None (defaults) or a
    dict of pd_batch_tuning fields.
    """
    if method not in METHODS:
        raise ValueError(f"batched method must be one of {METHODS}")
    if len(volumes) > _lib.BATCH_MAX_VOLUMES:
        raise ValueError(f"at most {_lib.BATCH_MAX_VOLUMES} volumes per batch")
    if recombination not in ("weighted", "average", "center"):
        raise ValueError("recombination must be one of 'weighted', 'average', 'center'")
    if method == "hybrid-pca" and noise_std is None:
        noise_std = 1.0
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device())
    with torch.cuda.device(device):
        _engine.check_device_errors()
        prep = _Prepared(volumes, method, patch_shape, patch_overlap, recombination, masks, mask_threshold,
                         threshold_value, threshold_scale, noise_std, loss, eps_marshenko_pastur, device)
        if tuning == "auto":
            tn = _TUNED.get(prep.signature(method))
            if tn is None:
                tn, _ = autotune(prep, method)
                prep.zero()
        elif tuning is None:
            tn = dict(synth_row_blocks=0, order_by_cost=1, chunk_patches=0)
        else:
            tn = {**dict(synth_row_blocks=0, order_by_cost=1, chunk_patches=0), **tuning}
        prep.run(tn)
        res = [r[:4] for r in prep.finalize()]
    return (res, tn) if return_tuning else res
