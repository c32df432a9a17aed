"""Store the reference test suite's phantom fixture (tests/conftest.py of the
reference): a 2D Shepp-Logan T2* slice x 20 frames with Gaussian noise scaled by
the Hamming g-factor map (RandomState(42)), built with the reference's own
simulation functions. Runs only where the reference sources are present.

    python tests/golden/make_phantom.py --ref /path/to/patch-denoising
"""

from __future__ import annotations

import argparse
import pathlib
import sys
import types

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent / "phantom"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="reference project root")
    args = ap.parse_args()
    stub = types.ModuleType("patch_denoise._version")
    stub.version = stub.__version__ = "0.0.0"
    sys.modules["patch_denoise._version"] = stub
    sys.path.insert(0, str(pathlib.Path(args.ref) / "src"))
    from patch_denoise.simulation.activations import add_frames
    from patch_denoise.simulation.noise import add_temporal_gaussian_noise
    from patch_denoise.simulation.phantom import g_factor_map, mr_shepp_logan_t2_star

    phantom = add_frames(mr_shepp_logan_t2_star(64)[32], 20)
    g_map = g_factor_map(phantom.shape[:-1])
    noisy = add_temporal_gaussian_noise(phantom, sigma=1, rng=np.random.RandomState(42), g_factor_map=g_map)
    HERE.mkdir(exist_ok=True)
    np.savez_compressed(HERE / "phantom.npz", phantom=phantom, noisy=noisy, g_map=g_map)
    print(phantom.shape, phantom.dtype, noisy.dtype)


if __name__ == "__main__":
    main()
