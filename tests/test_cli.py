"""Command-line front end: argument parsing on CPU, one end-to-end run on the GPU."""

from __future__ import annotations

import argparse

import numpy as np
import pytest

from patch_denoising_b200.bindings import cli


def _npy(tmp_path, name, arr):
    p = tmp_path / name
    np.save(p, arr)
    return p


def test_patch_shape_and_overlap_forms(tmp_path):
    f = _npy(tmp_path, "x.npy", np.zeros((4, 4, 4, 5), np.float32))
    a = cli.parse_args([str(f), "--method", "mp-pca", "--patch-shape", "5x5x3", "--patch-overlap", "2"])
    assert a.patch_shape == (5, 5, 3) and a.patch_overlap == 2 and a.extra == {}
    a = cli.parse_args([str(f), "--conf", "nordic_7_3_weighted_20", "--extra", "threshold_scale=1.5", "tag=x"])
    assert a.conf == "nordic_7_3_weighted_20" and a.extra == {"threshold_scale": 1.5, "tag": "x"}


def test_method_and_conf_are_exclusive(tmp_path):
    f = _npy(tmp_path, "x.npy", np.zeros((4, 4, 4, 5), np.float32))
    with pytest.raises(SystemExit):
        cli.parse_args([str(f), "--method", "mp-pca", "--conf", "mp-pca_5_2_weighted_10"])
    with pytest.raises(SystemExit):
        cli.parse_args([str(tmp_path / "missing.npy"), "--method", "mp-pca"])
    with pytest.raises(argparse.ArgumentTypeError):
        cli._positive_int("-3")


def test_npy_mask_and_noise_map_requirement(tmp_path):
    f = _npy(tmp_path, "x.npy", np.zeros((4, 4, 4, 5), np.float32))
    m = _npy(tmp_path, "m.npy", np.ones((4, 4, 4), np.uint8))
    a = cli.parse_args([str(f), str(tmp_path / "o.npy"), "--method", "mp-pca", "--mask", str(m)])
    mask, aff = cli._mask(a)
    assert mask.dtype == bool and mask.shape == (4, 4, 4) and aff is None
    with pytest.raises(RuntimeError, match="noise map"):
        cli.main([str(f), str(tmp_path / "o.npy"), "--method", "nordic"])


@pytest.mark.gpu
def test_cli_end_to_end_matches_the_api(tmp_path):
    from patch_denoising_b200 import mp_pca
    from patch_denoising_b200.synthetic import lowrank_volume

    x, _ = lowrank_volume((14, 14, 10, 30), 3, seed=5)
    f = _npy(tmp_path, "x.npy", x)
    out_file = cli.main([str(f), str(tmp_path / "out" / "d.npy"), "--method", "mp-pca", "--patch-shape", "5",
                         "--patch-overlap", "2", "--mask-threshold", "10", "--nan-to-num", "0"])
    got = np.load(out_file)
    want, _, _, _ = mp_pca(x, 5, 2, mask_threshold=10)
    np.testing.assert_array_equal(np.isnan(got), np.isnan(want))
    ok = ~np.isnan(want)
    assert np.linalg.norm(got[ok] - want[ok]) <= 1e-6 * np.linalg.norm(want[ok])
