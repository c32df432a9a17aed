"""pd_denoise_patches_noalloc against pd_denoise_patches, through the C ABI.

pd_denoise_patches_noalloc is for callers that cannot allocate device memory
while they denoise (a host application that manages a fixed device-memory budget
itself, or a loop where cudaMalloc's implicit synchronisation is not acceptable):
its scratch lives in a static device array inside the library instead of a
caller-provided workspace. Two calls in a row must each match the
workspace-based entry point, so the shared array's leftover contents from the
previous call must not leak into the next one. The cases cover both
precisions (the mixed one builds its tensor-core operand maps over the static
array), a patch list that needs several chunks of the array, and the device
error word, read back with pd_noalloc_check.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from parity import OUT_TOL
from patch_denoising_b200 import _engine, _lib
from patch_denoising_b200.synthetic import lowrank_volume

pytestmark = pytest.mark.gpu

NOALLOC_BYTES = 32 << 20  # the static array's size


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def _accumulators(shape, grid_t, n_sel, dtype, dev):
    nvox = int(np.prod(shape[:-1]))
    return dict(
        out=torch.zeros(shape, dtype=dtype, device=dev),
        wacc=torch.zeros(nvox * grid_t, dtype=torch.float32, device=dev),
        nacc=torch.zeros(nvox * grid_t, dtype=torch.float32, device=dev),
        nctr=torch.zeros(shape, dtype=torch.float32, device=dev),
        rank_map=torch.zeros(shape, dtype=torch.int32, device=dev),
        prank=torch.zeros(n_sel, dtype=torch.int32, device=dev),
        pnoise=torch.zeros(n_sel, dtype=torch.float32, device=dev),
    )


def _rel(a, b):
    a = a.cpu().numpy().astype(np.complex128).ravel()
    b = b.cpu().numpy().astype(np.complex128).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _setup(x, p_s, p_o, precision, dev):
    lib = _lib.load()
    g = _engine.geometry(tuple(x.shape), p_s, p_o)
    gp = ctypes.byref(g)
    s = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    need = ctypes.c_size_t()
    _lib.check(lib.pd_select_workspace_size(gp, ctypes.byref(need)))
    sws = torch.empty(need.value, dtype=torch.uint8, device=dev)
    plist = torch.empty(g.n_patches, dtype=torch.int32, device=dev)
    count = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.check(lib.pd_select_patches(gp, None, 0, 50.0, _vp(plist), _vp(count), _vp(sws), need.value, s))
    n_sel = int(count.item())
    prm = _lib.Params()
    prm.method = _lib.METHOD["mp-pca"]
    prm.recombination = _lib.RECOMBINATION["weighted"]
    prm.precision = _lib.PRECISION[precision]
    prm.is_complex = 1 if x.is_complex() else 0
    prm.threshold_scale = 1.0
    return lib, g, gp, s, plist, n_sel, prm


def _call_noalloc(lib, gp, pp, x, plist, n_sel, acc, s):
    return lib.pd_denoise_patches_noalloc(gp, pp, _vp(x), None, _vp(plist), n_sel, _vp(acc["out"]), _vp(acc["wacc"]),
                                          _vp(acc["nacc"]), _vp(acc["nctr"]), _vp(acc["rank_map"]),
                                          _vp(acc["prank"]), _vp(acc["pnoise"]), s)


# (shape, patch, overlap, complex, precision): one chunk in each precision, and a
# 700-patch list of 100 frames whose scratch needs several chunks of the array
CASES = [
    ((24, 22, 16, 40), (5, 5, 5, 40), (2, 2, 2, 40), False, "fp32"),
    ((24, 22, 16, 40), (5, 5, 5, 40), (2, 2, 2, 40), True, "fp32"),
    ((24, 22, 16, 40), (5, 5, 5, 40), (2, 2, 2, 40), False, "mixed"),
    ((32, 32, 24, 100), (5, 5, 5, 100), (2, 2, 2, 100), False, "fp32"),
    ((32, 32, 24, 100), (5, 5, 5, 100), (2, 2, 2, 100), True, "mixed"),
]


@pytest.mark.parametrize("shape,p_s,p_o,cplx,precision", CASES)
def test_noalloc_matches_workspace_entry_point_twice(shape, p_s, p_o, cplx, precision):
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    x_np, _ = lowrank_volume(shape, 3, amplitude=50.0, noise=3.0, complex_valued=cplx, seed=31)
    x = torch.from_numpy(x_np).to(dev)
    lib, g, gp, s, plist, n_sel, prm = _setup(x, p_s, p_o, precision, dev)
    assert n_sel > 0
    pp = ctypes.byref(prm)
    need = ctypes.c_size_t()
    _lib.check(lib.pd_denoise_workspace_size(gp, pp, 1, ctypes.byref(need)))
    if shape[-1] == 100:
        assert need.value * n_sel > 2 * NOALLOC_BYTES  # the case runs the chunk loop

    ref = _accumulators(shape, int(g.grid[3]), n_sel, x.dtype, dev)
    _lib.check(lib.pd_denoise_workspace_size(gp, pp, n_sel, ctypes.byref(need)))
    ws = torch.empty(need.value, dtype=torch.uint8, device=dev)
    _lib.check(lib.pd_denoise_patches(gp, pp, _vp(x), None, _vp(plist), n_sel, _vp(ref["out"]), _vp(ref["wacc"]),
                                      _vp(ref["nacc"]), _vp(ref["nctr"]), _vp(ref["rank_map"]), _vp(ref["prank"]),
                                      _vp(ref["pnoise"]), _vp(ws), need.value, s))
    _lib.check(lib.pd_workspace_check(_vp(ws), s))
    for _ in range(2):
        got = _accumulators(shape, int(g.grid[3]), n_sel, x.dtype, dev)
        _lib.check(_call_noalloc(lib, gp, pp, x, plist, n_sel, got, s))
        _lib.check(lib.pd_noalloc_check(s))
        torch.cuda.synchronize()
        assert torch.equal(got["prank"], ref["prank"])
        assert torch.equal(got["rank_map"], ref["rank_map"])
        assert _rel(got["out"], ref["out"]) <= OUT_TOL[precision]
        assert _rel(got["wacc"], ref["wacc"]) <= 1e-6
        assert _rel(got["nacc"], ref["nacc"]) <= OUT_TOL[precision]


def test_noalloc_reports_a_non_finite_sample_then_recovers():
    """A NaN inside a processed patch sets the device error word in the static
    array; pd_noalloc_check turns it into PD_ERR_INVALID (ValueError, as the
    reference's LAPACK calls raise), and the next clean call clears it."""
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    shape = (24, 22, 16, 40)
    x_np, _ = lowrank_volume(shape, 3, amplitude=50.0, noise=3.0, seed=32)
    bad = x_np.copy()
    bad[3, 4, 5, 6] = np.nan
    for arr, expect in ((bad, _lib.PD_ERR_INVALID), (x_np, _lib.PD_OK)):
        x = torch.from_numpy(arr).to(dev)
        lib, g, gp, s, plist, n_sel, prm = _setup(x, (5, 5, 5, 40), (2, 2, 2, 40), "fp32", dev)
        acc = _accumulators(shape, int(g.grid[3]), n_sel, x.dtype, dev)
        _lib.check(_call_noalloc(lib, gp, ctypes.byref(prm), x, plist, n_sel, acc, s))
        assert lib.pd_noalloc_check(s) == expect
