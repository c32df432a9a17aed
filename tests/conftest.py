"""Shared test configuration: the ``gpu`` marker and golden-fixture helpers."""

from __future__ import annotations

import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def golden_names():
    return sorted(p.stem for p in GOLDEN.glob("*.npz"))


def noise_golden_names():
    return sorted(p.stem for p in (GOLDEN / "noise").glob("*.npz"))


def load_noise_golden(name):
    """(input, block_size, reference noise map, map of the voxels the reference writes)."""
    z = np.load(GOLDEN / "noise" / f"{name}.npz", allow_pickle=False)
    return z["input"], int(z["block_size"]), z["noise_map"], z["covered"]


def load_golden(name):
    """Return (arrays, call) for a fixture; ``call`` holds oracle/denoiser kwargs."""
    z = np.load(GOLDEN / f"{name}.npz", allow_pickle=False)
    arrays = {k: z[k] for k in z.files if not k.startswith("meta_")}
    meta = {k[5:]: z[k] for k in z.files if k.startswith("meta_")}
    method = str(meta["method"])
    patch = meta["patch"]
    overlap = meta["overlap"]
    call = dict(
        method=method,
        patch_shape=int(patch) if patch.ndim == 0 else tuple(int(v) for v in patch),
        patch_overlap=int(overlap) if overlap.ndim == 0 else tuple(int(v) for v in overlap),
        recombination=str(meta["recombination"]),
    )
    if "mask" in arrays:
        call["mask"] = arrays["mask"]
    if "mask_threshold" in meta:
        call["mask_threshold"] = int(meta["mask_threshold"])
    if "threshold_scale" in meta:
        call["threshold_scale"] = float(meta["threshold_scale"])
    if "threshold_value" in meta:
        call["threshold_value"] = float(meta["threshold_value"])
    if "loss" in meta:
        call["loss"] = str(meta["loss"])
    if "noise_std" in arrays:
        ns = arrays["noise_std"]
        call["noise_std"] = float(ns) if ns.ndim == 0 else ns
    if "seed" in meta:
        call["seed"] = int(meta["seed"])
    return arrays, call


def adaptive_golden_names():
    return sorted(p.stem for p in (GOLDEN / "adaptive").glob("*.npz"))


def load_adaptive_golden(name):
    """(arrays, call) of an adaptive fixture; ``call`` holds the oracle's keyword
    arguments (``adaptive_method``, ``gamma0``, ``tau0``, ``nbsim``, ``seed``)."""
    z = np.load(GOLDEN / "adaptive" / f"{name}.npz", allow_pickle=False)
    arrays = {k: z[k] for k in z.files if not k.startswith("meta_")}
    meta = {k[5:]: z[k] for k in z.files if k.startswith("meta_")}
    ns = arrays["noise_std"]
    call = dict(
        method="adaptive",
        patch_shape=int(meta["patch"]),
        patch_overlap=int(meta["overlap"]),
        recombination=str(meta["recombination"]),
        adaptive_method=str(meta["method"]),
        noise_std=float(ns) if ns.ndim == 0 else ns,
        nbsim=int(meta["nbsim"]),
        gamma0=None,
        tau0=float(meta["tau0"]) if "tau0" in meta else None,
    )
    if "gamma0" in arrays:
        g = arrays["gamma0"]
        call["gamma0"] = float(g) if g.ndim == 0 else g
    if "seed" in meta:
        call["seed"] = int(meta["seed"])
    return arrays, call


@pytest.fixture(scope="session")
def golden():
    return {n: load_golden(n) for n in golden_names()}


def pytest_terminal_summary(terminalreporter):
    """Print the near-threshold rank ties of the GPU parity comparisons."""
    parity = sys.modules.get("parity")
    log = getattr(parity, "TIE_LOG", None)
    if not log:
        return
    tied = [r for r in log if r[2]]
    terminalreporter.write_line(
        f"parity: {len(log)} comparisons, {sum(r[2] for r in log)} rank ties in {len(tied)} of them "
        f"(bands: {parity.TIE_TOL})")
    for test, precision, n, margin in tied:
        terminalreporter.write_line(f"  {test} [{precision}]: {n} ties, largest margin {margin:.3g}")
