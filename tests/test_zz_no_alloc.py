"""pd_denoise_patches_noalloc against pd_denoise_patches, through the C ABI.

pd_denoise_patches_noalloc is for callers that cannot allocate device memory
while they denoise (a host application that manages a fixed device-memory budget
itself, or a loop where cudaMalloc's implicit synchronisation is not acceptable):
its scratch lives in a static device array inside the library instead of a
caller-provided workspace. Two calls in a row must each match the
workspace-based entry point, so the shared array's leftover contents from the
previous call must not leak into the next one.
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


@pytest.mark.parametrize("cplx", [False, True])
def test_noalloc_matches_workspace_entry_point_twice(cplx):
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    shape = (24, 22, 16, 40)
    x_np, _ = lowrank_volume(shape, 3, amplitude=50.0, noise=3.0, complex_valued=cplx, seed=31)
    x = torch.from_numpy(x_np).to(dev)
    p_s, p_o = (5, 5, 5, 40), (2, 2, 2, 40)
    g = _engine.geometry(shape, p_s, p_o)
    gp = ctypes.byref(g)
    s = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)

    need = ctypes.c_size_t()
    _lib.check(lib.pd_select_workspace_size(gp, ctypes.byref(need)))
    sws = torch.empty(need.value, dtype=torch.uint8, device=dev)
    plist = torch.empty(g.n_patches, dtype=torch.int32, device=dev)
    count = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.check(lib.pd_select_patches(gp, None, 0, 50.0, _vp(plist), _vp(count), _vp(sws), need.value, s))
    n_sel = int(count.item())
    assert n_sel > 0

    prm = _lib.Params()
    prm.method = _lib.METHOD["mp-pca"]
    prm.recombination = _lib.RECOMBINATION["weighted"]
    prm.precision = _lib.PRECISION["fp32"]
    prm.is_complex = 1 if cplx else 0
    prm.threshold_scale = 1.0
    pp = ctypes.byref(prm)

    def outputs(acc):
        return [acc["out"], acc["wacc"], acc["nacc"], acc["rank_map"], acc["prank"], acc["pnoise"]]

    ref = _accumulators(shape, int(g.grid[3]), n_sel, x.dtype, dev)
    _lib.check(lib.pd_denoise_workspace_size(gp, pp, n_sel, ctypes.byref(need)))
    ws = torch.empty(need.value, dtype=torch.uint8, device=dev)
    _lib.check(lib.pd_denoise_patches(gp, pp, _vp(x), None, _vp(plist), n_sel, _vp(ref["out"]), _vp(ref["wacc"]),
                                      _vp(ref["nacc"]), _vp(ref["nctr"]), _vp(ref["rank_map"]), _vp(ref["prank"]),
                                      _vp(ref["pnoise"]), _vp(ws), need.value, s))
    torch.cuda.synchronize()
    for _ in range(2):
        got = _accumulators(shape, int(g.grid[3]), n_sel, x.dtype, dev)
        _lib.check(lib.pd_denoise_patches_noalloc(gp, pp, _vp(x), None, _vp(plist), n_sel, _vp(got["out"]),
                                                  _vp(got["wacc"]), _vp(got["nacc"]), _vp(got["nctr"]),
                                                  _vp(got["rank_map"]), _vp(got["prank"]), _vp(got["pnoise"]), s))
        torch.cuda.synchronize()
        assert torch.equal(got["prank"], ref["prank"])
        assert torch.equal(got["rank_map"], ref["rank_map"])
        assert _rel(got["out"], ref["out"]) <= OUT_TOL["fp32"]
        assert _rel(got["wacc"], ref["wacc"]) <= 1e-6
        assert _rel(got["nacc"], ref["nacc"]) <= OUT_TOL["fp32"]
