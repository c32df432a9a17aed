"""Host-side logic (no GPU): C ABI exports, geometry, MP median, API surface, errors."""

from __future__ import annotations

import ctypes
import itertools
import re

import numpy as np
import pytest

import oracle
from conftest import ROOT
from patch_denoising_b200 import _engine, _lib
from patch_denoising_b200.bindings.utils import DENOISER_MAP, DenoiseParameters
from patch_denoising_b200.space_time import (
    HybridPCADenoiser,
    MPPCADenoiser,
    NordicDenoiser,
    OptimalSVDDenoiser,
    PatchedArray,
)


def _header_symbols():
    text = (ROOT / "include" / "patch_denoise_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pd_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    syms = _header_symbols()
    assert len(syms) >= 10
    for name in syms:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"
    assert lib.pd_version() >= 100


@pytest.mark.parametrize(
    "shape,patch,overlap",
    [
        ((32, 32, 24, 60), 5, 2),
        ((64, 64, 40, 200), 11, 5),
        ((10, 9, 8, 20), 4, 2),
        ((10, 9, 8, 20), (4, 4, 4, 12), (2, 2, 2, 6)),
        ((64, 64, 20), 6, 5),
        ((64, 64, 20), 10, 9),
        ((30, 20), 5, 0),
        ((12, 12, 12, 30), 12, 3),
        ((13, 17, 19, 25), (3, 5, 7), (1, 2, 7)),
    ],
)
def test_geometry_matches_oracle(shape, patch, overlap):
    p_s, p_o = oracle.patch_params(shape, patch, overlap)
    ps, step, grid = oracle.grid_geometry(shape, p_s, p_o)
    g = _engine.geometry(shape, p_s, p_o)
    pad = 4 - len(shape)
    assert tuple(g.grid)[pad:] == grid
    assert tuple(g.patch)[pad:] == ps
    assert tuple(g.shape)[pad:] == shape
    assert g.n_patches == int(np.prod(grid))
    assert g.rows == int(np.prod(ps[:-1]))
    assert g.cols == ps[-1]
    # the reference's strided view has the same grid
    view = PatchedArray(np.zeros(shape, np.float32), p_s, p_o)
    assert view.n_patches == g.n_patches


def test_geometry_errors():
    with pytest.raises(ValueError, match="overlap should be smaller"):
        _engine.geometry((10, 10, 10, 20), (4, 4, 4, 20), (5, 2, 2, 0))
    with pytest.raises(ValueError):
        _engine.geometry((10, 10, 10, 20), (11, 4, 4, 20), (2, 2, 2, 0))
    with pytest.raises(NotImplementedError):
        _engine.geometry((4, 4, 4, 4, 20), (2, 2, 2, 2, 20), (0, 0, 0, 0, 0))


@pytest.mark.parametrize("beta", list(np.arange(1, 10) * 0.1) + [0.0, 1.0, 20 / 216, 60 / 125, 200 / 1331,
                                                                     300 / 1331, 120 / 343])
def test_mp_median_matches_reference_dichotomy(beta):
    got = _engine.mp_median(beta, 1e-7)
    ref = oracle.marchenko_pastur_median(beta, eps=1e-7)
    # identical bracket decisions except where quad's own error flips one
    assert abs(got - ref) <= 1e-7


def test_mp_median_rejects_bad_beta():
    with pytest.raises(ValueError, match="Aspect Ratio"):
        _engine.mp_median(1.5)


def test_denoise_parameters_roundtrip():
    d = DenoiseParameters("optimal-fro", 11, 10, "weighted", 10)
    d2 = DenoiseParameters.from_str(str(d))
    assert d == d2
    assert DenoiseParameters.from_str("noisy").method is None
    d3 = DenoiseParameters.from_str("mp-pca_6_5_weighted")
    assert (d3.method, d3.patch_shape, d3.patch_overlap, d3.recombination) == ("mp-pca", 6, 5, "weighted")


def test_registry_names():
    assert set(DENOISER_MAP) == {None, "mp-pca", "hybrid-pca", "raw", "optimal-fro", "optimal-fro-noise",
                                 "optimal-nuc", "optimal-ope", "nordic", "adaptive-qut"}


def test_constructor_errors():
    with pytest.raises(ValueError, match="recombination"):
        MPPCADenoiser(5, 2, 1.0, recombination="median")
    with pytest.raises(KeyError):
        OptimalSVDDenoiser(5, 2, loss="l1")


def test_custom_patch_processing_is_rejected_at_construction():
    """The reference's extension point is a per-patch ``_patch_processing``
    (base.py:352-357); the CUDA loop cannot call Python per patch, so a subclass
    that overrides it (or names no built-in method) fails at once with a message
    that lists the supported methods."""
    from patch_denoising_b200.space_time.base import BaseSpaceTimeDenoiser

    class Custom(MPPCADenoiser):
        def _patch_processing(self, patch, patch_idx=None, **kwargs):
            return patch, 0, 0.0

    class Bare(BaseSpaceTimeDenoiser):
        def _patch_processing(self, patch, patch_idx=None, **kwargs):
            return patch, 0, 0.0

    for make in (lambda: Custom(5, 2, 1.0), lambda: Bare(5, 2)):
        with pytest.raises(NotImplementedError, match="mp-pca, hybrid-pca, raw, nordic, optimal, adaptive"):
            make()
    MPPCADenoiser(5, 2, 1.0)  # the built-in classes still construct


def test_nordic_noise_std_type_error_before_device_use():
    # space_time/lowrank.py:234-240: a non-float, non-array noise level is a ValueError
    x = np.zeros((10, 10, 10, 20), np.float32)
    with pytest.raises(ValueError, match="NORDIC"):
        NordicDenoiser(4, 2).denoise(x, noise_std="not_a_float_or_array")


def test_patch_param_int_and_tuple():
    den = HybridPCADenoiser(6, 5)
    assert den._get_patch_param((64, 64, 20)) == ((6, 6, 20), (5, 5, 20))
    den = HybridPCADenoiser([3, 4, 5], (1, 1, 1))
    assert den._get_patch_param((10, 10, 10, 30)) == ((3, 4, 5, 30), (1, 1, 1, 30))


def test_device_error_words_checked_without_a_stall():
    """A queued error word raises once its copy has landed, and only then."""
    import torch

    from patch_denoising_b200 import _engine

    class FakeEvent:
        def __init__(self, done):
            self.done = done

        def query(self):
            return self.done

        def synchronize(self):
            self.done = True

    _engine._pending_errors[:] = [(FakeEvent(False), torch.tensor([0, 5], dtype=torch.int32))]
    _engine.check_device_errors()  # copy not landed yet: nothing to report
    assert len(_engine._pending_errors) == 1
    with pytest.raises(RuntimeError, match="timed out"):
        _engine.check_device_errors(block=True)
    assert not _engine._pending_errors
    _engine._pending_errors[:] = [(FakeEvent(True), torch.tensor([0, 0], dtype=torch.int32))]
    _engine.check_device_errors()
    assert not _engine._pending_errors


def test_nonfinite_patch_word_raises_value_error():
    """Error word 7 (a NaN / inf sample in a processed patch) is the reference's ValueError."""
    import torch

    from patch_denoising_b200 import _engine

    class Done:
        def query(self):
            return True

        def synchronize(self):
            pass

    _engine._pending_errors[:] = [(Done(), torch.tensor([7], dtype=torch.int32))]
    with pytest.raises(ValueError, match="infs or NaNs"):
        _engine.check_device_errors()
    assert not _engine._pending_errors


def test_adaptive_argument_errors_match_the_reference():
    """Raised before any device work, as the reference raises them."""
    from patch_denoising_b200.space_time import AdaptiveDenoiser

    with pytest.raises(ValueError):
        AdaptiveDenoiser(4, 2, method="lasso")
    x = np.zeros((8, 8, 8, 10), dtype=np.float32)
    with pytest.raises(TypeError):  # noise_std ** 2 with None
        AdaptiveDenoiser(4, 2, method="sure").denoise(x, gamma0=[1.0])
    with pytest.raises(TypeError):  # for g in gamma0 with None / a scalar
        AdaptiveDenoiser(4, 2, method="sure").denoise(x, noise_std=1.0, gamma0=None)
    with pytest.raises(TypeError):
        AdaptiveDenoiser(4, 2, method="gsure").denoise(x, noise_std=1.0, gamma0=2.0)


def test_ctypes_structs_match_the_c_header(tmp_path):
    """pd_geometry, pd_params, pd_adaptive, pd_volume and pd_batch_tuning: the ctypes mirrors have the C layout
    (size and every field offset), checked by compiling the header with the C compiler."""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    structs = {"pd_geometry": _lib.Geometry, "pd_params": _lib.Params, "pd_adaptive": _lib.Adaptive,
               "pd_volume": _lib.Volume, "pd_batch_tuning": _lib.BatchTuning}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "patch_denoise_b200.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(line.split()[:2]): int(line.split()[2]) for line in out if line}
    for cname, py in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for field, _ in py._fields_:
            assert got[(cname, field)] == getattr(py, field).offset, (cname, field)


def test_adaptive_record_from_the_denoiser_settings():
    """The pd_adaptive record that pd_adaptive_denoise_patches receives."""
    ad = _engine._adaptive_struct({"mode": "gsure", "gamma": [1.0, 2.5, 4.0], "tau0": None})
    assert (ad.mode, ad.n_gamma, ad.has_tau0) == (_lib.ADAPTIVE_MODE["gsure"], 3, 0)
    assert list(ad.gamma[:3]) == [1.0, 2.5, 4.0]
    ad = _engine._adaptive_struct({"mode": "sure", "gamma": [2.0], "tau0": 1.75})
    assert (ad.has_tau0, ad.tau0) == (1, 1.75)
    ad = _engine._adaptive_struct({"mode": "qut", "gamma": [], "qut_level": 12.5})
    assert (ad.mode, ad.n_gamma, ad.qut_level) == (_lib.ADAPTIVE_MODE["qut"], 0, 12.5)


def test_qut_level_rejects_a_quantile_outside_0_1():
    """max(M, T) < 3 puts the QUT probability 1 - 1/sqrt(log max(M, T)) below 0,
    which numpy.quantile (and so the reference) rejects; checked before any device work."""
    lib = _lib.load()
    out = ctypes.c_double()
    st = lib.pd_adaptive_qut_level(2, 2, 10, ctypes.c_uint64(1), 0, ctypes.byref(out), None, 0, None)
    assert st == _lib.PD_ERR_INVALID
    assert b"Quantiles must be in the range" in lib.pd_last_error()
