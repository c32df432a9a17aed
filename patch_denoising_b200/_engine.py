"""Device orchestration of one ``denoise()`` call through the C ABI.

PyTorch provides device memory and the stream; every computation on the volume
runs in ``libpd_b200.so``. The call sequence mirrors
``BaseSpaceTimeDenoiser.denoise`` (space_time/base.py:177-270):

  pd_select_patches   mask scoring + ascending list of kept patches (base.py:202-227)
  pd_denoise_patches  per-patch decomposition, threshold, synthesis, scatter (base.py:235-258)
  pd_finalize         normalisation by the weights, masking (base.py:262-270)
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib


def _vp(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def geometry(shape, p_s, p_o) -> _lib.Geometry:
    """``pd_geometry_init`` over the full (time-appended) patch shape and overlap."""
    lib = _lib.load()
    nd = len(shape)
    arr = lambda v: (ctypes.c_int64 * nd)(*[int(x) for x in v])  # noqa: E731
    g = _lib.Geometry()
    _lib.check(lib.pd_geometry_init(nd, arr(shape), arr(p_s), arr(p_o), ctypes.byref(g)))
    return g


def mp_median(beta: float, eps: float = 1e-7) -> float:
    """Marchenko-Pastur median (``pd_mp_median``)."""
    out = ctypes.c_double()
    _lib.check(_lib.load().pd_mp_median(float(beta), float(eps), ctypes.byref(out)))
    return out.value


def nordic_max_sval(rows: int, cols: int, n_iter: int, seed: int, device, precision: str = "fp32") -> float:
    """Mean largest singular value of ``n_iter`` Gaussian rows x cols draws."""
    lib = _lib.load()
    need = ctypes.c_size_t()
    _lib.check(lib.pd_nordic_workspace_size(int(rows), int(cols), int(n_iter), ctypes.byref(need)))
    ws = torch.empty(max(need.value, 1), dtype=torch.uint8, device=device)
    out = ctypes.c_double()
    _lib.check(
        lib.pd_nordic_mc_threshold(
            int(rows), int(cols), int(n_iter), ctypes.c_uint64(int(seed) & (2**64 - 1)),
            _lib.PRECISION[precision], ctypes.byref(out), _vp(ws), need.value, _stream(device),
        )
    )
    return out.value


def adaptive_qut_level(rows: int, cols: int, n_sim: int, seed: int, device, precision: str = "fp32") -> float:
    """QUT quantile of the largest singular value of ``n_sim`` Gaussian rows x cols draws."""
    lib = _lib.load()
    need = ctypes.c_size_t()
    _lib.check(lib.pd_nordic_workspace_size(int(rows), int(cols), int(n_sim), ctypes.byref(need)))
    ws = torch.empty(max(need.value, 1), dtype=torch.uint8, device=device)
    out = ctypes.c_double()
    _lib.check(
        lib.pd_adaptive_qut_level(
            int(rows), int(cols), int(n_sim), ctypes.c_uint64(int(seed) & (2**64 - 1)),
            _lib.PRECISION[precision], ctypes.byref(out), _vp(ws), need.value, _stream(device),
        )
    )
    return out.value


def _adaptive_struct(adaptive: dict):
    ad = _lib.Adaptive()
    ad.mode = _lib.ADAPTIVE_MODE[adaptive["mode"]]
    gam = list(adaptive.get("gamma") or [])
    ad.n_gamma = len(gam)
    for i, v in enumerate(gam):
        ad.gamma[i] = float(v)
    tau0 = adaptive.get("tau0")
    ad.has_tau0 = 0 if tau0 is None else 1
    ad.tau0 = 0.0 if tau0 is None else float(tau0)
    ad.qut_level = float(adaptive.get("qut_level") or 0.0)
    return ad


@dataclass
class DeviceResult:
    """Outputs of one call, on the device."""

    out: torch.Tensor
    weights: torch.Tensor
    noise_map: torch.Tensor
    rank_map: torch.Tensor
    patch_index: torch.Tensor
    patch_rank: torch.Tensor
    patch_noise: torch.Tensor
    level: torch.Tensor | None = None  # NORDIC: float64 [level, noise_std * level]


def compute_dtype(dtype) -> torch.dtype:
    """Arithmetic type of the CUDA path for an input dtype."""
    if dtype in (torch.complex64, torch.complex128, np.complex64, np.complex128):
        return torch.complex64
    return torch.float32


def to_device(x, device, dtype=None) -> torch.Tensor:
    """Host array or tensor -> contiguous device tensor of ``dtype``."""
    if isinstance(x, torch.Tensor):
        t = x
        if dtype is not None and t.dtype != dtype:
            t = t.to(dtype)
        return t.to(device).contiguous()
    a = np.ascontiguousarray(x)
    if dtype is not None and a.dtype != _NP[dtype]:
        a = a.astype(_NP[dtype])
    if a.nbytes < _STAGE_MIN:
        t = torch.from_numpy(a) if a.flags.writeable else torch.from_numpy(a.copy())
        return t.to(device)
    return _staged_h2d(a, device)


# Host-to-device copies of pageable NumPy memory run through two pinned staging
# buffers: the host copy of chunk k + 1 (torch's multi-threaded memcpy) overlaps
# the DMA of chunk k, instead of the driver's single-threaded staging.
_STAGE_MIN = 16 << 20
_STAGE_CHUNK = 16 << 20


def _staged_h2d(a: np.ndarray, device) -> torch.Tensor:
    src = torch.from_numpy(a.reshape(-1).view(np.uint8))
    nbytes = src.numel()
    dst = torch.empty(nbytes, dtype=torch.uint8, device=device)
    stream = torch.cuda.current_stream(device)
    chunk = min(_STAGE_CHUNK, nbytes)
    stage = [torch.empty(chunk, dtype=torch.uint8, pin_memory=True) for _ in range(2)]
    done = [None, None]
    for k, lo in enumerate(range(0, nbytes, chunk)):
        hi = min(lo + chunk, nbytes)
        b = k & 1
        if done[b] is not None:
            done[b].synchronize()  # the DMA out of this buffer has finished
        stage[b][: hi - lo].copy_(src[lo:hi])
        dst[lo:hi].copy_(stage[b][: hi - lo], non_blocking=True)
        done[b] = torch.cuda.Event()
        done[b].record(stream)
    return dst.view(torch.from_numpy(a[:0]).dtype).view(a.shape)


_NP = {torch.float32: np.float32, torch.complex64: np.complex64}


def spread_over_frames(spatial, shape):
    """A read-only 4D view of a map that is constant along frames (no copy)."""
    return np.broadcast_to(spatial[..., None], shape)


def to_host(tensors):
    """Device tensors -> NumPy arrays through pinned buffers (torch's host cache)."""
    hosts = []
    for t in tensors:
        h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
        h.copy_(t, non_blocking=True)
        hosts.append(h)
    if tensors:
        torch.cuda.current_stream(tensors[0].device).synchronize()
    check_device_errors(block=True)
    return [h.numpy() for h in hosts]


# Device-side error words (bounded waits that timed out) are read without
# stalling the host: each call queues a copy of its words into pinned memory and
# the check happens when that copy has landed -- at the next call, at the host
# copy of the results, or at an explicit check_device_errors(block=True).
_pending_errors = []


def _queue_error_check(words, device):
    h = torch.empty(len(words), dtype=torch.int32, pin_memory=True)
    for i, w in enumerate(words):
        h[i : i + 1].copy_(w[:4].view(torch.int32), non_blocking=True)
    ev = torch.cuda.Event()
    ev.record(torch.cuda.current_stream(device))
    _pending_errors.append((ev, h))


NONFINITE = 7  # error word of a processed patch with a NaN / inf sample (PD_DEVERR_NONFINITE)


def check_device_errors(block: bool = False) -> None:
    """Raise for an earlier call's device error word: ValueError for a NaN / inf
    sample in a processed patch (the reference's LAPACK calls reject those),
    RuntimeError for a timed-out device-side wait.

    ``block``: wait for the pending checks instead of taking only the finished ones.
    """
    keep, code = [], 0
    for ev, h in _pending_errors:
        if block:
            ev.synchronize()
        elif not ev.query():
            keep.append((ev, h))
            continue
        code = code or int(h.max())
    _pending_errors[:] = keep
    if code == NONFINITE:
        raise ValueError("array must not contain infs or NaNs")
    if code:
        raise RuntimeError(f"a device-side wait timed out (code {code})")


def run(
    method: str,
    data: torch.Tensor,
    p_s,
    p_o,
    recombination: str,
    mask: torch.Tensor | None,
    mask_threshold: float,
    *,
    threshold_scale: float = 1.0,
    threshold: float = 0.0,
    noise_std: torch.Tensor | None = None,
    loss: str = "fro",
    mp_med: float = 0.0,
    precision: str = "fp32",
    nordic: dict | None = None,
    adaptive: dict | None = None,
) -> DeviceResult:
    """Denoise ``data`` (device tensor, float32 or complex64, C-contiguous).

    ``mask``: uint8 device tensor of the data shape or of its spatial shape, or None.
    ``noise_std``: float64 device tensor of the spatial shape, or None.
    ``nordic``: {"noise_std", "rows", "n_iter", "seed"}: compute the NORDIC
    Monte-Carlo level on the device ahead of the patch loop, with no host
    round trip (``pd_nordic_denoise_patches``); ``threshold`` is then unused.
    ``adaptive``: {"mode", "gamma", "tau0", "qut_level"} for the adaptive
    shrinkage (``pd_adaptive_denoise_patches``).
    """
    lib = _lib.load()
    device = data.device
    if device.type != "cuda":
        raise RuntimeError("the denoising path runs on a CUDA device only")
    check_device_errors()
    cplx = data.is_complex()
    shape = tuple(data.shape)
    g = geometry(shape, p_s, p_o)
    s = _stream(device)
    gp = ctypes.byref(g)

    # ---- selection
    need = ctypes.c_size_t()
    _lib.check(lib.pd_select_workspace_size(gp, ctypes.byref(need)))
    ws = torch.empty(max(need.value, 1), dtype=torch.uint8, device=device)
    plist = torch.empty(max(g.n_patches, 1), dtype=torch.int32, device=device)
    count = torch.zeros(1, dtype=torch.int32, device=device)
    mask_4d = 0
    if mask is not None:
        mask_4d = 1 if mask.dim() == len(shape) else 0
    _lib.check(
        lib.pd_select_patches(gp, _vp(mask), mask_4d, float(mask_threshold), _vp(plist), _vp(count), _vp(ws),
                              need.value, s)
    )
    if mask is None:
        # every patch scores 100 % (k_patch_flags without a mask): no device round trip
        n_sel = int(g.n_patches) if 100.0 > float(mask_threshold) else 0
    else:
        n_sel = int(count.item())

    # ---- parameters
    prm = _lib.Params()
    prm.method = _lib.METHOD[method]
    prm.recombination = _lib.RECOMBINATION[recombination]
    prm.loss = _lib.LOSS[loss]
    prm.precision = _lib.PRECISION[precision]
    prm.is_complex = 1 if cplx else 0
    prm.has_prior = 1 if noise_std is not None else 0
    prm.threshold_scale = float(threshold_scale)
    prm.threshold = float(threshold)
    prm.mp_median = float(mp_med)
    pp = ctypes.byref(prm)

    # ---- accumulators and outputs
    full = (int(g.shape[0]), int(g.shape[1]), int(g.shape[2]), int(g.shape[3]))
    nvox = full[0] * full[1] * full[2]
    out = torch.zeros(shape, dtype=data.dtype, device=device)
    wacc = torch.zeros(nvox * int(g.grid[3]), dtype=torch.float32, device=device)
    nacc = torch.zeros_like(wacc)
    # the centre-element noise map is read and written by "center" recombination only
    nctr = torch.zeros(shape if recombination == "center" else (1,), dtype=torch.float32, device=device)
    rank_map = torch.zeros(shape, dtype=torch.int32, device=device)
    prank = torch.zeros(max(n_sel, 1), dtype=torch.int32, device=device)
    pnoise = torch.zeros(max(n_sel, 1), dtype=torch.float32, device=device)
    _lib.check(lib.pd_denoise_workspace_size(gp, pp, n_sel, ctypes.byref(need)))
    ws = torch.empty(max(need.value, 1), dtype=torch.uint8, device=device)
    level = mc_ws = None
    if adaptive is not None:
        ad = _adaptive_struct(adaptive)
        _lib.check(
            lib.pd_adaptive_denoise_patches(
                gp, pp, ctypes.byref(ad), _vp(data), _vp(noise_std), _vp(plist), n_sel, _vp(out), _vp(wacc),
                _vp(nacc), _vp(nctr), _vp(rank_map), _vp(prank), _vp(pnoise), _vp(ws), need.value, s,
            )
        )
    elif nordic is None:
        _lib.check(
            lib.pd_denoise_patches(
                gp, pp, _vp(data), _vp(noise_std), _vp(plist), n_sel, _vp(out), _vp(wacc), _vp(nacc), _vp(nctr),
                _vp(rank_map), _vp(prank), _vp(pnoise), _vp(ws), need.value, s,
            )
        )
    else:
        mc_need = ctypes.c_size_t()
        rows, n_iter = int(nordic["rows"]), int(nordic["n_iter"])
        _lib.check(lib.pd_nordic_workspace_size(rows, int(g.cols), n_iter, ctypes.byref(mc_need)))
        mc_ws = torch.empty(max(mc_need.value, 1), dtype=torch.uint8, device=device)
        level = torch.empty(2, dtype=torch.float64, device=device)
        _lib.check(
            lib.pd_nordic_denoise_patches(
                gp, pp, float(nordic["noise_std"]), rows, n_iter, ctypes.c_uint64(int(nordic["seed"]) & (2**64 - 1)),
                _vp(level), _vp(mc_ws), mc_need.value, _vp(data), _vp(plist), n_sel, _vp(out), _vp(wacc),
                _vp(nacc), _vp(nctr), _vp(rank_map), _vp(prank), _vp(pnoise), _vp(ws), need.value, s,
            )
        )
    weights = torch.empty(shape, dtype=torch.float32, device=device)
    noise_map = torch.empty(shape, dtype=torch.float32, device=device)
    _lib.check(
        lib.pd_finalize(gp, pp, _vp(out), _vp(wacc), _vp(nacc), _vp(nctr), _vp(weights), _vp(noise_map), _vp(mask),
                        mask_4d, s)
    )
    words = ([ws] if n_sel else []) + ([mc_ws] if mc_ws is not None else [])
    if words:
        _queue_error_check(words, device)
    return DeviceResult(out, weights, noise_map, rank_map, plist[:n_sel], prank[:n_sel], pnoise[:n_sel], level)


def estimate_noise(data: torch.Tensor, block_size: int) -> torch.Tensor:
    """``pd_estimate_noise`` on a device tensor (float32 or complex64, time last)."""
    lib = _lib.load()
    device = data.device
    shape = tuple(int(v) for v in data.shape)
    arr = (ctypes.c_int64 * len(shape))(*shape)
    cplx = 1 if data.is_complex() else 0
    need = ctypes.c_size_t()
    _lib.check(lib.pd_estimate_noise_workspace_size(len(shape), arr, cplx, ctypes.byref(need)))
    ws = torch.empty(max(need.value, 1), dtype=torch.uint8, device=device)
    out = torch.empty(shape[:-1], dtype=torch.float64, device=device)
    with torch.cuda.device(device):
        _lib.check(lib.pd_estimate_noise(len(shape), arr, cplx, _vp(data), int(block_size), _vp(out), _vp(ws),
                                         need.value, _stream(device)))
    return out


# --------------------------------------------------------------------------- #
# Host (NumPy) volumes: upload, patch work and download overlap               #
# --------------------------------------------------------------------------- #
# A host volume at least this large, without a mask, is streamed: patches are
# processed in ranges of patch-grid x positions (each range one eigensolver
# wave), each range starts as soon as the x slabs it reads are on the device,
# and the x slabs no later patch touches are normalised and copied back while
# the next range runs. Uploads and downloads each have a stream of their own.
STREAM_MIN_BYTES = 64 << 20
_copy_streams = {}
# bytes the last streamed call moved over PCIe (host to device, device to host)
LAST_TRANSFER = {"h2d": 0, "d2h": 0}


def _copy_stream(device, which):
    """Per-device upload ("h2d") or download ("d2h") stream: separate, so the two
    directions run on both copy engines at once."""
    idx = device.index if device.index is not None else torch.cuda.current_device()
    key = (idx, which)
    if key not in _copy_streams:
        _copy_streams[key] = torch.cuda.Stream(device)
    return _copy_streams[key]


def _params(method, recombination, loss, precision, cplx, has_prior, threshold_scale, threshold, mp_med):
    prm = _lib.Params()
    prm.method = _lib.METHOD[method]
    prm.recombination = _lib.RECOMBINATION[recombination]
    prm.loss = _lib.LOSS[loss]
    prm.precision = _lib.PRECISION[precision]
    prm.is_complex = 1 if cplx else 0
    prm.has_prior = 1 if has_prior else 0
    prm.threshold_scale = float(threshold_scale)
    prm.threshold = float(threshold)
    prm.mp_median = float(mp_med)
    return prm


def run_host(
    method: str,
    x: np.ndarray,
    p_s,
    p_o,
    recombination: str,
    mask_threshold: float,
    *,
    threshold_scale: float = 1.0,
    threshold: float = 0.0,
    noise_std: torch.Tensor | None = None,
    loss: str = "fro",
    mp_med: float = 0.0,
    precision: str = "fp32",
    nordic: dict | None = None,
    adaptive: dict | None = None,
    device=None,
):
    """Denoise a host volume (float32 / complex64, C order, no mask) with streaming.

    Returns ``(out, weights, noise_map, rank_map)`` as NumPy arrays (pinned
    memory) and the DeviceResult of the per-patch records, or ``None`` when the
    volume does not stream (then use ``to_device`` + ``run``).
    """
    lib = _lib.load()
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device())
    shape = tuple(x.shape)
    cplx = np.iscomplexobj(x)
    if x.nbytes < STREAM_MIN_BYTES or len(shape) != 4 or adaptive is not None:
        return None
    g = geometry(shape, p_s, p_o)
    gx = int(g.grid[0])
    per_x = int(g.n_patches) // gx
    n_sel = int(g.n_patches) if 100.0 > float(mask_threshold) else 0
    if gx < 2 or n_sel == 0:
        return None
    check_device_errors()
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    xs_per = max(1, sms // per_x)  # x positions per range: at most one eigensolver wave
    step_x, patch_x = int(g.step[0]), int(g.patch[0])
    comp = torch.cuda.current_stream(device)
    upl = _copy_stream(device, "h2d")
    dnl = _copy_stream(device, "d2h")
    s = ctypes.c_void_p(comp.cuda_stream)
    gp = ctypes.byref(g)
    tdtype = torch.complex64 if cplx else torch.float32

    # identity patch list (no mask), accumulators, parameters: on the compute stream
    need = ctypes.c_size_t()
    _lib.check(lib.pd_select_workspace_size(gp, ctypes.byref(need)))
    sel_ws = torch.empty(max(need.value, 1), dtype=torch.uint8, device=device)
    plist = torch.empty(g.n_patches, dtype=torch.int32, device=device)
    count = torch.zeros(1, dtype=torch.int32, device=device)
    _lib.check(lib.pd_select_patches(gp, None, 0, float(mask_threshold), _vp(plist), _vp(count), _vp(sel_ws),
                                     need.value, s))
    prm = _params(method, recombination, loss, precision, cplx, noise_std is not None, threshold_scale, threshold,
                  mp_med)
    pp = ctypes.byref(prm)
    nvox = shape[0] * shape[1] * shape[2]
    ngt = int(g.grid[3])
    out = torch.zeros(shape, dtype=tdtype, device=device)
    wacc = torch.zeros(nvox * ngt, dtype=torch.float32, device=device)
    nacc = torch.zeros_like(wacc)
    nctr = torch.zeros(shape if recombination == "center" else (1,), dtype=torch.float32, device=device)
    rank_map = torch.zeros(shape, dtype=torch.int32, device=device)
    weights = torch.empty(shape, dtype=torch.float32, device=device)
    noise_map = torch.empty(shape, dtype=torch.float32, device=device)
    prank = torch.zeros(n_sel, dtype=torch.int32, device=device)
    pnoise = torch.zeros(n_sel, dtype=torch.float32, device=device)
    level = mc_ws = None
    mc_need = ctypes.c_size_t()
    if nordic is not None:
        _lib.check(lib.pd_nordic_workspace_size(int(nordic["rows"]), int(g.cols), int(nordic["n_iter"]),
                                                ctypes.byref(mc_need)))
        mc_ws = torch.empty(max(mc_need.value, 1), dtype=torch.uint8, device=device)
        level = torch.empty(2, dtype=torch.float64, device=device)

    # host buffers of the results (pinned, returned as NumPy views); with one
    # time window the maps are constant along frames: only their spatial part
    # crosses PCIe (returned as broadcast views)
    h_out = torch.empty(shape, dtype=tdtype, pin_memory=True)
    h_w = torch.empty(shape, dtype=torch.float32, pin_memory=True)
    maps_spatial = ngt == 1
    # with one time window the weights are constant along frames too: their
    # spatial part comes down and is spread over the frames of the returned
    # (full, writable) array on the host, while the output is still in flight
    h_w_sp = torch.empty(shape[:-1], dtype=torch.float32, pin_memory=True) if maps_spatial else None
    w_slabs = []
    d2h = 0
    nm_spatial = maps_spatial and recombination != "center"  # "center": the centre frame only
    h_nm = torch.empty(shape[:-1] if nm_spatial else shape, dtype=torch.float32, pin_memory=True)
    h_rm = torch.empty(shape[:-1] if maps_spatial else shape, dtype=torch.int32, pin_memory=True)

    # upload state: the input goes up slab by slab on the copy stream
    src = torch.from_numpy(x.reshape(-1).view(np.uint8))
    dst = torch.empty(x.nbytes, dtype=torch.uint8, device=device)
    data = dst.view(tdtype).view(shape)
    slab = x.nbytes // shape[0]
    stage_n = max(slab, (_STAGE_CHUNK // slab) * slab)
    stage = [torch.empty(stage_n, dtype=torch.uint8, pin_memory=True) for _ in range(2)]
    done = [None, None]
    up = {"bytes": 0, "k": 0}
    upl.wait_stream(comp)  # buffers allocated on the compute stream
    dnl.wait_stream(comp)

    def upload_to(nbytes):
        ev = None
        while up["bytes"] < nbytes:
            lo = up["bytes"]
            hi = min(lo + stage_n, x.nbytes)
            b = up["k"] & 1
            if done[b] is not None:
                done[b].synchronize()
            stage[b][: hi - lo].copy_(src[lo:hi])
            with torch.cuda.stream(upl):
                dst[lo:hi].copy_(stage[b][: hi - lo], non_blocking=True)
                done[b] = torch.cuda.Event()
                done[b].record(upl)
            up["bytes"], up["k"] = hi, up["k"] + 1
            ev = done[b]
        return ev

    # ranges of x positions, each at most one eigensolver wave. The first is a
    # single position, so the first download starts once a sixth of the input
    # is up; so is the last, so the final slab (everything the last range
    # completes) is small and its download short once the last input has landed
    bounds = [(0, 1)] if gx > 2 else []
    a = bounds[-1][1] if bounds else 0
    while a < gx:
        bounds.append((a, min(gx, a + xs_per)))
        a = bounds[-1][1]
    if bounds[-1][1] - bounds[-1][0] > 1:
        a, b_ = bounds.pop()
        bounds += [(a, b_ - 1), (b_ - 1, b_)]
    words = []
    x_done = 0
    for a, b_ in bounds:
        first, cnt = a * per_x, (b_ - a) * per_x
        ev = upload_to(((b_ - 1) * step_x + patch_x) * slab)
        if ev is not None:
            comp.wait_event(ev)
        _lib.check(lib.pd_denoise_workspace_size(gp, pp, cnt, ctypes.byref(need)))
        ws = torch.empty(max(need.value, 1), dtype=torch.uint8, device=device)
        words.append(ws)
        lst = ctypes.c_void_p(plist.data_ptr() + 4 * first)
        if nordic is None:
            _lib.check(lib.pd_denoise_patches(
                gp, pp, _vp(data), _vp(noise_std), lst, cnt, _vp(out), _vp(wacc), _vp(nacc), _vp(nctr),
                _vp(rank_map), ctypes.c_void_p(prank.data_ptr() + 4 * first),
                ctypes.c_void_p(pnoise.data_ptr() + 4 * first), _vp(ws), need.value, s))
        else:
            rows = int(nordic["rows"]) if a == 0 else 0  # later ranges reuse the level on the device
            _lib.check(lib.pd_nordic_denoise_patches(
                gp, pp, float(nordic["noise_std"]), rows, int(nordic["n_iter"]),
                ctypes.c_uint64(int(nordic["seed"]) & (2**64 - 1)), _vp(level), _vp(mc_ws), mc_need.value,
                _vp(data), lst, cnt, _vp(out), _vp(wacc), _vp(nacc), _vp(nctr), _vp(rank_map),
                ctypes.c_void_p(prank.data_ptr() + 4 * first), ctypes.c_void_p(pnoise.data_ptr() + 4 * first),
                _vp(ws), need.value, s))
        # voxels below the next range's first patch are final: normalise and download them
        x_end = b_ * step_x if b_ < gx else shape[0]
        if x_end > x_done:
            sub = _lib.Geometry.from_buffer_copy(g)
            sub.shape[0] = x_end - x_done
            v0 = x_done * shape[1] * shape[2]
            e0 = v0 * shape[3]
            _lib.check(lib.pd_finalize(
                ctypes.byref(sub), pp, ctypes.c_void_p(out.data_ptr() + e0 * out.element_size()),
                ctypes.c_void_p(wacc.data_ptr() + 4 * v0 * ngt), ctypes.c_void_p(nacc.data_ptr() + 4 * v0 * ngt),
                ctypes.c_void_p(nctr.data_ptr() + (4 * e0 if recombination == "center" else 0)),
                ctypes.c_void_p(weights.data_ptr() + 4 * e0),
                ctypes.c_void_p(noise_map.data_ptr() + 4 * e0), None, 0, s))
            fin = torch.cuda.Event()
            fin.record(comp)
            dnl.wait_event(fin)
            with torch.cuda.stream(dnl):
                if maps_spatial:  # first, so that its spreading overlaps the output's download
                    h_w_sp[x_done:x_end].copy_(weights[x_done:x_end, ..., 0], non_blocking=True)
                    ev_w = torch.cuda.Event()
                    ev_w.record(dnl)
                    w_slabs.append((x_done, x_end, ev_w))
                else:
                    h_w[x_done:x_end].copy_(weights[x_done:x_end], non_blocking=True)
                h_out[x_done:x_end].copy_(out[x_done:x_end], non_blocking=True)
                for h, d, flat in ((h_nm, noise_map, nm_spatial), (h_rm, rank_map, maps_spatial)):
                    piece = d[x_done:x_end, ..., 0] if flat else d[x_done:x_end]
                    h[x_done:x_end].copy_(piece, non_blocking=True)
            d2h += out[x_done:x_end].nbytes + (h_w_sp[x_done:x_end] if maps_spatial else h_w[x_done:x_end]).nbytes
            d2h += h_nm[x_done:x_end].nbytes + h_rm[x_done:x_end].nbytes
            x_done = x_end
    # spread each slab's spatial weights over the frames as soon as it has landed
    # (torch's multithreaded host copy; the output slabs are still coming down)
    for x0, x1, ev_w in w_slabs:
        ev_w.synchronize()
        h_w[x0:x1].copy_(h_w_sp[x0:x1, ..., None].expand(x1 - x0, *shape[1:]))
    # the compute stream's later work (and buffer reuse) comes after both copy streams
    comp.wait_stream(upl)
    comp.wait_stream(dnl)
    words = words + ([mc_ws] if mc_ws is not None else [])
    _queue_error_check(words, device)
    res = DeviceResult(out, weights, noise_map, rank_map, plist[:n_sel], prank, pnoise, level)
    dnl.synchronize()
    comp.synchronize()
    check_device_errors(block=True)
    LAST_TRANSFER.update(h2d=int(x.nbytes), d2h=int(d2h))
    nm, rm = h_nm.numpy(), h_rm.numpy()
    if nm_spatial:
        nm = spread_over_frames(nm, shape)
    if maps_spatial:
        rm = spread_over_frames(rm, shape)
    return (h_out.numpy(), h_w.numpy(), nm, rm), res
