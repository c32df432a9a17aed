"""BIDS app (bindings/cli.py:510-667): discovery, naming and masking on CPU,
one whole run over a small dataset on the GPU."""

from __future__ import annotations

import json

import numpy as np
import pytest

from patch_denoising_b200.bindings import bids
from patch_denoising_b200.synthetic import ellipsoid_mask, lowrank_volume


def _dataset(root):
    """Two subjects: sub-01 with two tasks, sub-02 with a session; .npy runs."""
    runs = {}
    mask = ellipsoid_mask((16, 16, 12), fill=0.5, seed=1)
    for rel, seed in [("sub-01/func/sub-01_task-rest_bold.npy", 1),
                      ("sub-01/func/sub-01_task-motor_run-2_bold.npy", 2),
                      ("sub-02/ses-a/func/sub-02_ses-a_task-rest_bold.npy", 3)]:
        x, _ = lowrank_volume((16, 16, 12, 30), 3, seed=seed)
        x = x + 200.0 * mask[..., None]  # bright brain on a dark background
        p = root / rel
        p.parent.mkdir(parents=True, exist_ok=True)
        np.save(p, x.astype(np.float32))
        runs[rel] = x
    (root / "sub-01" / "anat").mkdir(parents=True)
    np.save(root / "sub-01" / "anat" / "sub-01_T1w.npy", np.zeros((4, 4, 4), np.float32))
    return runs, mask


def test_names_and_discovery(tmp_path):
    _dataset(tmp_path)
    ents, suffix, ext = bids.parse_bids_name("sub-02_ses-a_task-rest_run-3_bold.nii.gz")
    assert ents == {"sub": "02", "ses": "a", "task": "rest", "run": "3"} and suffix == "bold" and ext == ".nii.gz"
    assert bids.bids_name(dict(ents, desc="denoised"), "std", ".npy") == \
        "sub-02_ses-a_task-rest_run-3_desc-denoised_std.npy"
    assert bids.subjects(tmp_path) == ["01", "02"]
    assert bids.subjects(tmp_path, ["sub-02"]) == ["02"]
    assert [f.name for f in bids.bold_runs(tmp_path, "01")] == ["sub-01_task-motor_run-2_bold.npy",
                                                                 "sub-01_task-rest_bold.npy"]
    assert [f.name for f in bids.bold_runs(tmp_path, "01", {"task": ["rest"]})] == ["sub-01_task-rest_bold.npy"]
    assert bids.bold_runs(tmp_path, "02", {"ses": ["b"]}) == []


def test_epi_mask_finds_the_bright_region():
    mask = ellipsoid_mask((20, 20, 16), fill=0.4, seed=2)
    x, _ = lowrank_volume((20, 20, 16, 12), 2, seed=4)
    got = bids.epi_mask(x + 300.0 * mask[..., None])
    assert (got == mask).mean() > 0.97


def test_dataset_description_is_appended(tmp_path):
    d = bids.update_dataset_description(tmp_path)
    assert d["DatasetType"] == "derivative" and len(d["GeneratedBy"]) == 1
    d = bids.update_dataset_description(tmp_path)
    assert len(json.loads((tmp_path / "dataset_description.json").read_text())["GeneratedBy"]) == 2


def test_noise_methods_need_a_noise_map(tmp_path):
    _dataset(tmp_path / "in")
    with pytest.raises(RuntimeError, match="noise map"):
        bids.bids_app([str(tmp_path / "in"), str(tmp_path / "out"), "participant", "--method", "nordic"])


@pytest.mark.gpu
def test_bids_app_denoises_every_selected_run(tmp_path):
    from patch_denoising_b200 import mp_pca

    runs, _ = _dataset(tmp_path / "in")
    out = tmp_path / "out"
    written = bids.bids_app([str(tmp_path / "in"), str(out), "participant", "--method", "mp-pca",
                             "--patch-shape", "5", "--patch-overlap", "2", "--task-label", "rest"])
    assert sorted(p.relative_to(out).as_posix() for p in written) == [
        "sub-01/sub-01_task-rest_desc-denoised_bold.npy",
        "sub-02/ses-a/sub-02_ses-a_task-rest_desc-denoised_bold.npy"]
    for rel in ("sub-01/func/sub-01_task-rest_bold.npy", "sub-02/ses-a/func/sub-02_ses-a_task-rest_bold.npy"):
        x = runs[rel]
        stem = rel.split("/")[-1].replace("_bold.npy", "")
        sub_dir = out / "/".join(rel.split("/")[:-2])
        mask = np.load(sub_dir / f"{stem}_desc-denoised_mask.npy").astype(bool)
        got = np.load(sub_dir / f"{stem}_desc-denoised_bold.npy")
        assert (sub_dir / f"{stem}_desc-denoised_std.npy").exists()
        want, _, _, _ = mp_pca(x, 5, 2, mask=mask, mask_threshold=10)
        np.testing.assert_array_equal(np.isnan(got), np.isnan(want))
        ok = ~np.isnan(want)
        assert np.linalg.norm(got[ok] - want[ok]) <= 1e-6 * np.linalg.norm(want[ok])
