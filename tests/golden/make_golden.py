"""Generate the golden fixtures by running the reference package itself.

Run in a checkout that has the reference sources (``--ref`` points at the
reference project root; its ``src/`` is put on ``sys.path`` with a stub
``patch_denoise._version``). The GPU test machines never run this script: they
only read the ``.npz`` files it writes next to itself.

Each case stores the (float32-representable) input, the reference outputs
(denoised volume and weights, both as float32/complex64), the selected patch
indices and, recorded by wrapping ``_patch_processing``, the per-patch
``(maxidx, noise_var)`` the reference computes. Inputs are rounded to float32
first and the reference then runs on their float64 (complex128) copies, so the
stored input is exactly what the reference saw.

    python tests/golden/make_golden.py --ref /path/to/patch-denoising
"""

from __future__ import annotations

import argparse
import pathlib
import sys
import types

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from patch_denoising_b200.synthetic import ellipsoid_mask, lowrank_volume  # noqa: E402


def _import_reference(ref_root):
    stub = types.ModuleType("patch_denoise._version")
    stub.version = stub.__version__ = "0.0.0"
    sys.modules["patch_denoise._version"] = stub
    sys.path.insert(0, str(pathlib.Path(ref_root) / "src"))
    from patch_denoise.simulation.activations import add_frames
    from patch_denoise.simulation.noise import add_temporal_gaussian_noise
    from patch_denoise.simulation.phantom import g_factor_map, mr_shepp_logan_t2_star
    from patch_denoise.space_time import lowrank

    return types.SimpleNamespace(
        lowrank=lowrank,
        add_frames=add_frames,
        add_noise=add_temporal_gaussian_noise,
        g_factor_map=g_factor_map,
        phantom=mr_shepp_logan_t2_star,
    )


def _run(ref, method, data, patch, overlap, recombination, mask=None, mask_threshold=50,
         seed=None, **kw):
    lr = ref.lowrank
    if method == "mp-pca":
        den = lr.MPPCADenoiser(patch, overlap, threshold_scale=kw.pop("threshold_scale", 1.0),
                               recombination=recombination)
    elif method == "hybrid-pca":
        den = lr.HybridPCADenoiser(patch, overlap, recombination=recombination)
    elif method == "raw":
        den = lr.RawSVDDenoiser(patch, overlap, threshold_value=kw.pop("threshold_value"),
                                recombination=recombination)
    elif method == "nordic":
        den = lr.NordicDenoiser(patch, overlap, recombination=recombination)
    elif method == "optimal":
        den = lr.OptimalSVDDenoiser(patch, overlap, loss=kw.pop("loss"),
                                    recombination=recombination)
    else:
        raise ValueError(method)
    rec = {}
    inner = den._patch_processing

    def recording(patch_arr, patch_idx=None, **pkw):
        res = inner(patch_arr, patch_idx=patch_idx, **pkw)
        rec[int(patch_idx)] = (int(res[1]), float(res[2]))
        return res

    den._patch_processing = recording
    if seed is not None:
        np.random.seed(seed)
    out, weights, _, _ = den.denoise(data, mask=mask, mask_threshold=mask_threshold,
                                     progbar=False, **kw)
    idx = np.array(sorted(rec), dtype=np.int64)
    extra = {}
    if method in ("raw", "nordic"):
        extra["threshold"] = np.float64(den._threshold)
    if method == "optimal":
        extra["mp_median"] = np.float64(den.input_denoising_kwargs["mp_median"])
    return dict(
        out=np.asarray(out).astype(np.complex64 if np.iscomplexobj(out) else np.float32),
        weights=np.asarray(weights, dtype=np.float32),
        patches=idx,
        patch_rank=np.array([rec[i][0] for i in idx], dtype=np.int64),
        patch_noise=np.array([rec[i][1] for i in idx], dtype=np.float64),
        **extra,
    )


def _cases(ref):
    """(name, input, call kwargs) for every fixture."""
    shape = (10, 9, 8, 20)
    x, _ = lowrank_volume(shape, 3, amplitude=20.0, sigma_space=3.0, noise=1.0, seed=11)
    xc, _ = lowrank_volume(shape, 3, amplitude=20.0, sigma_space=3.0, noise=1.0, seed=12,
                           complex_valued=True)
    mask3 = ellipsoid_mask(shape[:-1], fill=0.6, seed=3)
    rng = np.random.default_rng(5)
    mask4 = rng.random(shape) < 0.7
    nmap = 0.8 + 0.4 * rng.random(shape[:-1])
    p, o = 4, 2
    cases = []
    for rec in ("weighted", "average", "center"):
        cases.append((f"mppca_{rec}", x, dict(method="mp-pca", patch=p, overlap=o,
                                              recombination=rec, threshold_scale=1.0)))
    cases += [
        ("mppca_mask3_tau23", x, dict(method="mp-pca", patch=p, overlap=o, recombination="weighted",
                                      threshold_scale=2.3, mask=mask3, mask_threshold=50)),
        ("mppca_mask4", x, dict(method="mp-pca", patch=p, overlap=o, recombination="weighted",
                                mask=mask4, mask_threshold=30)),
        ("mppca_timetiled", x, dict(method="mp-pca", patch=(4, 4, 4, 12), overlap=(2, 2, 2, 6),
                                    recombination="weighted")),
        ("hybrid_scalar", x, dict(method="hybrid-pca", patch=p, overlap=o,
                                  recombination="weighted", noise_std=1.0)),
        ("hybrid_map_average", x, dict(method="hybrid-pca", patch=p, overlap=o,
                                       recombination="average", noise_std=nmap)),
        ("raw_weighted", x, dict(method="raw", patch=p, overlap=o, recombination="weighted",
                                 threshold_value=12.0)),
        ("raw_center", x, dict(method="raw", patch=p, overlap=o, recombination="center",
                               threshold_value=12.0)),
        ("nordic_weighted", x, dict(method="nordic", patch=p, overlap=o, recombination="weighted",
                                    noise_std=1.0, seed=1234)),
        ("opt_fro", x, dict(method="optimal", patch=p, overlap=o, recombination="weighted",
                            loss="fro")),
        ("opt_nuc", x, dict(method="optimal", patch=p, overlap=o, recombination="weighted",
                            loss="nuc")),
        ("opt_ope", x, dict(method="optimal", patch=p, overlap=o, recombination="weighted",
                            loss="ope")),
        ("opt_fro_prior_average", x, dict(method="optimal", patch=p, overlap=o,
                                          recombination="average", loss="fro", noise_std=nmap)),
        ("opt_ope_center", x, dict(method="optimal", patch=p, overlap=o, recombination="center",
                                   loss="ope")),
        ("cplx_mppca", xc, dict(method="mp-pca", patch=p, overlap=o, recombination="weighted",
                                threshold_scale=1.0)),
        ("cplx_raw", xc, dict(method="raw", patch=p, overlap=o, recombination="weighted",
                              threshold_value=15.0)),
        ("cplx_nordic", xc, dict(method="nordic", patch=p, overlap=o, recombination="weighted",
                                 noise_std=1.0, seed=99)),
        ("cplx_opt_fro", xc, dict(method="optimal", patch=p, overlap=o, recombination="weighted",
                                  loss="fro")),
    ]
    # The reference's own test fixture: 2D Shepp-Logan T2* slice x 20 frames,
    # Gaussian noise scaled by the Hamming g-factor map (RandomState(42)).
    ph = ref.add_frames(ref.phantom(64)[32], 20)
    g_map = ref.g_factor_map(ph.shape[:-1])
    noisy = ref.add_noise(ph, sigma=1, rng=np.random.RandomState(42), g_factor_map=g_map)
    cases += [
        ("phantom_mppca", noisy, dict(method="mp-pca", patch=6, overlap=5,
                                      recombination="weighted", threshold_scale=2.3)),
        ("phantom_opt_nuc_prior", noisy, dict(method="optimal", patch=10, overlap=9,
                                              recombination="weighted", loss="nuc",
                                              noise_std=1.414 * g_map)),
    ]
    return cases


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="reference project root")
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    ref = _import_reference(args.ref)
    for name, data, kw in _cases(ref):
        if args.only and args.only != name:
            continue
        kw = dict(kw)
        method = kw.pop("method")
        patch = kw.pop("patch")
        overlap = kw.pop("overlap")
        recomb = kw.pop("recombination")
        data32 = np.asarray(data).astype(np.complex64 if np.iscomplexobj(data) else np.float32)
        data64 = data32.astype(np.complex128 if np.iscomplexobj(data) else np.float64)
        res = _run(ref, method, data64, patch, overlap, recomb, **kw)
        meta = dict(method=method, patch=np.array(patch), overlap=np.array(overlap),
                    recombination=recomb)
        for key in ("threshold_scale", "threshold_value", "loss", "mask_threshold", "seed"):
            if key in kw:
                meta[key] = kw[key]
        arrays = {"input": data32, **res}
        if "mask" in kw and kw["mask"] is not None:
            arrays["mask"] = kw["mask"]
        if "noise_std" in kw:
            ns = kw["noise_std"]
            arrays["noise_std"] = np.asarray(ns, dtype=np.float64)
        np.savez_compressed(HERE / f"{name}.npz", **arrays,
                            **{f"meta_{k}": np.asarray(v) for k, v in meta.items()})
        print(f"{name}: {len(res['patches'])} patches, ranks {np.bincount(res['patch_rank'])}")


if __name__ == "__main__":
    main()
