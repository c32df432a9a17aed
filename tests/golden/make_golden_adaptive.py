"""Golden fixtures of the adaptive shrinkage, made by running the reference's
``AdaptiveDenoiser`` itself (space_time/lowrank.py:536-636).

Run in a checkout that has the reference sources (``--ref`` points at the
reference project root, as for ``make_golden.py``); the GPU test machines only
read the ``.npz`` files this writes under ``adaptive/``. Inputs are rounded to
float32 first and the reference runs on their float64 (complex128) copies. The
per-patch maxidx is recorded by wrapping ``_patch_processing``. QUT cases seed
NumPy's global generator, whose per-patch Gaussian draws the oracle replays.

    python tests/golden/make_golden_adaptive.py --ref /path/to/patch-denoising
"""

from __future__ import annotations

import argparse
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parents[1]))

from make_golden import _import_reference  # noqa: E402

from patch_denoising_b200.synthetic import lowrank_volume  # noqa: E402

OUT = HERE / "adaptive"


def _cases():
    shape = (10, 9, 8, 20)
    x, _ = lowrank_volume(shape, 3, amplitude=20.0, sigma_space=3.0, noise=1.0, seed=21)
    xc, _ = lowrank_volume(shape, 3, amplitude=20.0, sigma_space=3.0, noise=1.0, seed=22, complex_valued=True)
    rng = np.random.default_rng(6)
    nmap = 0.8 + 0.4 * rng.random(shape[:-1])
    return [
        ("sure_weighted", x, dict(method="sure", patch=4, overlap=2, recombination="weighted", noise_std=1.0,
                                  gamma0=np.array([1.0, 2.0, 3.0]))),
        ("gsure_average_map", x, dict(method="gsure", patch=4, overlap=2, recombination="average",
                                      noise_std=nmap, gamma0=np.linspace(1, 4, 4))),
        ("sure_tau0", x, dict(method="sure", patch=4, overlap=2, recombination="weighted", noise_std=1.0,
                              gamma0=np.array([2.0]), tau0=np.log(6.0))),
        ("qut_fixed_gamma", x, dict(method="qut", patch=4, overlap=2, recombination="weighted", noise_std=1.0,
                                    gamma0=2.0, nbsim=30, seed=7)),
        ("qut_estimated_gamma", x, dict(method="qut", patch=4, overlap=2, recombination="weighted",
                                        noise_std=nmap, gamma0=None, nbsim=30, seed=8)),
        ("cplx_sure", xc, dict(method="sure", patch=4, overlap=2, recombination="weighted", noise_std=1.0,
                               gamma0=np.array([1.0, 2.0]))),
    ]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="reference project root")
    args = ap.parse_args()
    ref = _import_reference(args.ref)
    OUT.mkdir(exist_ok=True)
    for name, data, kw in _cases():
        kw = dict(kw)
        data32 = np.asarray(data).astype(np.complex64 if np.iscomplexobj(data) else np.float32)
        data64 = data32.astype(np.complex128 if np.iscomplexobj(data) else np.float64)
        den = ref.lowrank.AdaptiveDenoiser(kw["patch"], kw["overlap"], method=kw["method"],
                                           recombination=kw["recombination"], nbsim=kw.get("nbsim", 500))
        rec = {}
        inner = den._patch_processing

        def recording(patch_arr, patch_idx=None, _inner=inner, _rec=rec, **pkw):
            res = _inner(patch_arr, patch_idx=patch_idx, **pkw)
            _rec[int(patch_idx)] = int(res[1])
            return res

        den._patch_processing = recording
        if "seed" in kw:
            np.random.seed(kw["seed"])
        out, weights, _, _ = den.denoise(data64, tau0=kw.get("tau0"), noise_std=kw["noise_std"],
                                         gamma0=kw["gamma0"], progbar=False)
        idx = np.array(sorted(rec), dtype=np.int64)
        arrays = dict(
            input=data32,
            out=np.asarray(out).astype(np.complex64 if np.iscomplexobj(out) else np.float32),
            weights=np.asarray(weights, dtype=np.float32),
            patches=idx,
            patch_rank=np.array([rec[i] for i in idx], dtype=np.int64),
            noise_std=np.asarray(kw["noise_std"], dtype=np.float64),
        )
        if kw["gamma0"] is not None:
            arrays["gamma0"] = np.asarray(kw["gamma0"], dtype=np.float64)
        meta = dict(method=kw["method"], patch=np.array(kw["patch"]), overlap=np.array(kw["overlap"]),
                    recombination=kw["recombination"], nbsim=kw.get("nbsim", 500))
        for key in ("tau0", "seed"):
            if key in kw:
                meta[key] = kw[key]
        np.savez_compressed(OUT / f"{name}.npz", **arrays, **{f"meta_{k}": np.asarray(v) for k, v in meta.items()})
        print(f"{name}: {len(idx)} patches, ranks {np.bincount(arrays['patch_rank'])}")


if __name__ == "__main__":
    main()
