"""Generate the noise-map fixtures by running the reference's ``estimate_noise``.

Like ``make_golden.py``, this runs only where the reference sources are present
(``--ref`` = reference project root). Inputs are rounded to float32 / complex64
and the reference runs on their float64 / complex128 copies. The reference
leaves voxels that no block centres on as ``np.empty`` content, so each fixture
also stores the map of the voxels it writes (``covered``).

    python tests/golden/make_golden_noise.py --ref /path/to/patch-denoising
"""

from __future__ import annotations

import argparse
import pathlib
import sys
import types

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent / "noise"


def _cases():
    rng = np.random.default_rng(2024)
    c = []
    c.append(("f32_12x10x8x20_b3", rng.normal(size=(12, 10, 8, 20)), 3))
    c.append(("f32_9x9x6x16_b1", rng.normal(scale=2.0, size=(9, 9, 6, 16)), 1))
    c.append(("f32_10x8x7x12_b2", rng.normal(size=(10, 8, 7, 12)), 2))
    c.append(("f32_offset_11x9x8x15_b3", 50.0 + rng.normal(scale=0.5, size=(11, 9, 8, 15)), 3))
    c.append(("c64_8x8x6x10_b3", rng.normal(size=(8, 8, 6, 10)) + 1j * rng.normal(size=(8, 8, 6, 10)), 3))
    c.append(("f32_2d_16x12x24_b3", rng.normal(size=(16, 12, 24)), 3))
    return c


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="reference project root")
    args = ap.parse_args()
    stub = types.ModuleType("patch_denoise._version")
    stub.version = stub.__version__ = "0.0.0"
    sys.modules["patch_denoise._version"] = stub
    sys.path.insert(0, str(pathlib.Path(args.ref) / "src"))
    from patch_denoise.space_time.utils import estimate_noise

    HERE.mkdir(exist_ok=True)
    for name, data, b in _cases():
        x32 = data.astype(np.complex64 if np.iscomplexobj(data) else np.float32)
        x64 = x32.astype(np.complex128 if np.iscomplexobj(data) else np.float64)
        out = estimate_noise(x64, b)
        v = x32.shape[:-1]
        cov = np.zeros(v, dtype=bool)
        cov[tuple(slice(b // 2, s - b + b // 2 + 1) for s in v)] = True
        out = np.where(cov, out, 0.0)
        np.savez_compressed(HERE / f"{name}.npz", input=x32, noise_map=out, covered=cov,
                            block_size=np.int64(b))
        print(name, out.shape, int(cov.sum()))


if __name__ == "__main__":
    main()
