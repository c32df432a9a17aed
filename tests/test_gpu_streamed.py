"""Large host volumes stream (upload, patch ranges, download overlap): same results
as the device-resident path."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from parity import rel_l2
from patch_denoising_b200 import _engine
from patch_denoising_b200.space_time import (
    HybridPCADenoiser,
    MPPCADenoiser,
    NordicDenoiser,
    OptimalSVDDenoiser,
)
from patch_denoising_b200.synthetic import lowrank_volume

pytestmark = pytest.mark.gpu


def _make(kind):
    if kind == "mppca":
        x, _ = lowrank_volume((40, 24, 14, 60), 4, seed=41)
        return x, lambda: MPPCADenoiser(5, 2, threshold_scale=1.0), {}
    if kind == "hybrid":
        x, _ = lowrank_volume((40, 24, 14, 60), 4, seed=42)
        return x, lambda: HybridPCADenoiser(5, 2, recombination="average"), {"noise_std": 5.0}
    if kind == "mppca_time_tiled":
        x, _ = lowrank_volume((40, 24, 14, 60), 4, seed=45)
        return x, lambda: MPPCADenoiser((5, 5, 5, 20), (2, 2, 2, 10), threshold_scale=1.0), {}
    if kind == "optimal_center":
        x, _ = lowrank_volume((40, 24, 14, 60), 4, seed=43)
        return x, lambda: OptimalSVDDenoiser(7, 3, loss="nuc", recombination="center"), {}
    x, _ = lowrank_volume((36, 22, 14, 48), 3, seed=44, complex_valued=True)
    return x, lambda: NordicDenoiser(7, 3, precision="mixed"), {"noise_std": 5.0, "n_iter_threshold": 3}


@pytest.mark.parametrize("kind", ["mppca", "mppca_time_tiled", "hybrid", "optimal_center", "nordic_mixed"])
def test_streamed_host_volume_matches_device_path(kind, monkeypatch):
    x, make, kw = _make(kind)
    monkeypatch.setattr(_engine, "STREAM_MIN_BYTES", 1 << 20)
    called = {}
    real = _engine.run_host

    def spy(*a, **k):
        r = real(*a, **k)
        called["streamed"] = r is not None
        return r

    monkeypatch.setattr(_engine, "run_host", spy)
    np.random.seed(3)
    den_h = make()
    out_h, w_h, nm_h, rm_h = den_h.denoise(x, **kw)
    assert called.get("streamed")
    np.random.seed(3)
    den_d = make()
    out_d, w_d, nm_d, rm_d = (t.cpu().numpy() for t in den_d.denoise(torch.from_numpy(x).cuda(), **kw))
    np.testing.assert_array_equal(np.asarray(den_h.patch_rank_), den_d.patch_rank_.cpu().numpy())
    np.testing.assert_array_equal(rm_h, rm_d)
    np.testing.assert_array_equal(np.isnan(out_h), np.isnan(out_d))
    ok = ~np.isnan(out_d)
    cdt = np.complex128 if np.iscomplexobj(out_d) else np.float64
    assert rel_l2(out_h[ok].astype(cdt), out_d[ok].astype(cdt)) <= 1e-6
    assert rel_l2(w_h.astype(np.float64), w_d.astype(np.float64)) <= 1e-6
    # the weights come back as a full, writable array even where only their
    # spatial part crossed PCIe (patches spanning every frame)
    assert w_h.flags.writeable and w_h.strides[-1] != 0
    spans_all = kind != "mppca_time_tiled"
    frames = x.shape[-1] if spans_all else 1
    nm_frames = 1 if kind == "optimal_center" else frames  # "center": the full noise map
    sent = out_h.nbytes + w_h.nbytes // frames + nm_h.nbytes // nm_frames + rm_h.nbytes // frames
    assert _engine.LAST_TRANSFER["h2d"] == x.nbytes
    assert _engine.LAST_TRANSFER["d2h"] == sent
    fin = np.isfinite(nm_d)
    np.testing.assert_array_equal(fin, np.isfinite(nm_h))
    if fin.any():
        assert rel_l2(nm_h[fin].astype(np.float64), nm_d[fin].astype(np.float64)) <= 1e-5
    if kind == "nordic_mixed":
        assert den_h.mc_max_sval_ == den_d.mc_max_sval_
