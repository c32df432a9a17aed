"""BIDS app: denoise every BOLD run of a BIDS dataset (bindings/cli.py:137-200, 510-667).

``patch-denoise-bids bids_dir output_dir participant [--participant-label ...]
[--session-label ...] [--task-label ...] [--method ... | --conf ...]``: for each
subject (every ``sub-*`` folder, or the given labels) and each
``func/*_bold.nii[.gz]`` run (``*_bold.npy`` too, for data held as NumPy arrays),
optionally filtered by task and session, it

* computes a brain mask of the run: nilearn's ``NiftiMasker(mask_strategy="epi")``
  as the reference when nilearn is installed and the run is NIfTI, else
  ``epi_mask`` below, and saves it as ``..._desc-denoised_mask``;
* denoises the run with the chosen method (``DENOISER_MAP``, the GPU path) and
  saves ``..._desc-denoised_bold`` and the noise map ``..._desc-denoised_std``
  under ``output_dir/sub-<label>[/ses-<label>]``;
* records itself in ``output_dir/dataset_description.json`` (appended to an
  existing ``GeneratedBy`` list, as the reference).

File discovery, entity parsing and output naming are written here (the reference
uses nilearn's BIDS helpers, which are not needed for this).
"""

from __future__ import annotations

import argparse
import json
import logging
import re
from pathlib import Path

import numpy as np

from .. import __version__
from .cli import NOISE_METHODS, ToDict, _tuple_positive_int
from .utils import DENOISER_MAP, DenoiseParameters, load_as_array, save_array

# BIDS entity order of file names (the specification's entity table)
ENTITY_ORDER = ("sub", "ses", "task", "acq", "ce", "rec", "dir", "run", "mod", "echo", "flip", "inv", "mt", "part",
                "recording", "space", "res", "den", "label", "desc")
BOLD_EXTENSIONS = (".nii.gz", ".nii", ".npy")


def bids_parser():
    """Arguments of the BIDS app (the reference's ``_bids_parser`` plus the denoising options)."""
    p = argparse.ArgumentParser(formatter_class=argparse.ArgumentDefaultsHelpFormatter)
    p.add_argument("bids_dir", type=Path, help="The directory with the input dataset formatted according to BIDS.")
    p.add_argument("output_dir", type=Path, help="The directory where the output files should be stored.")
    p.add_argument("analysis_level", choices=["participant"],
                   help="Level of the analysis that will be performed. Only participant level is available.")
    p.add_argument("--participant-label", "--participant_label", nargs="+",
                   help="Participant label(s) without 'sub-'; default: every subject.")
    p.add_argument("--session-label", "--session_label", nargs="+", help="Session label(s) without 'ses-'.")
    p.add_argument("--task-label", "--task_label", nargs="+", help="Task label(s) without 'task-'.")
    p.add_argument("--bids-filter-file", type=Path, default=None,
                   help="JSON file of entity filters for the 'bold' query, e.g. {\"bold\": {\"run\": \"1\"}}.")
    p.add_argument("--version", action="version", version=__version__)
    p.add_argument("--gpu", action="store_true", help="Use GPU for computation if available.")
    den = p.add_argument_group("Denoising parameters")
    exclusive = den.add_mutually_exclusive_group(required=True)
    exclusive.add_argument("--method", choices=DENOISER_MAP, default="optimal-fro", help="Denoising method.")
    exclusive.add_argument("--conf", default=None,
                           help="<name>_<patch-size>_<patch-overlap>_<recombination>_<mask_threshold>.")
    den.add_argument("--patch-shape", default=11, type=lambda s: _tuple_positive_int(s, True), metavar="INT")
    den.add_argument("--patch-overlap", default=5, type=lambda s: _tuple_positive_int(s, True), metavar="INT")
    den.add_argument("--recombination", default="weighted", choices=["mean", "weighted"])
    den.add_argument("--mask-threshold", default=10, type=int, metavar="INT")
    den.add_argument("--extra", metavar="key=value", default=None, nargs="+", action=ToDict)
    p.add_argument("-v", "--verbose", action="count", default=0, help="Increase verbosity level.")
    return p


def split_extension(path):
    name = Path(path).name
    for ext in BOLD_EXTENSIONS:
        if name.endswith(ext):
            return name[: -len(ext)], ext
    stem = Path(name).stem
    return stem, name[len(stem):]


def parse_bids_name(path):
    """``sub-01_ses-a_task-rest_run-2_bold.nii.gz`` -> ({entity: label}, suffix, extension)."""
    base, ext = split_extension(path)
    parts = base.split("_")
    entities = {}
    for part in parts[:-1]:
        key, sep, val = part.partition("-")
        if not sep:
            raise ValueError(f"not a BIDS entity: {part!r} in {Path(path).name}")
        entities[key] = val
    return entities, parts[-1], ext


def bids_name(entities, suffix, ext):
    """A BIDS file name with the entities in the specification's order."""
    known = [k for k in ENTITY_ORDER if k in entities]
    other = [k for k in entities if k not in ENTITY_ORDER]
    return "_".join([f"{k}-{entities[k]}" for k in known + other] + [suffix]) + ext


def subjects(bids_dir, labels=None):
    if labels:
        return [str(lab).removeprefix("sub-") for lab in labels]
    return sorted(p.name.removeprefix("sub-") for p in Path(bids_dir).iterdir() if p.is_dir()
                  and p.name.startswith("sub-"))


def bold_runs(bids_dir, subject, filters=None):
    """Every ``func/*_bold.<ext>`` run of a subject (any session) whose entities match ``filters``."""
    root = Path(bids_dir) / f"sub-{subject}"
    files = []
    for f in sorted(root.glob("**/func/*_bold*")):
        base, ext = split_extension(f)
        if ext not in BOLD_EXTENSIONS:
            continue
        ents, suffix, _ = parse_bids_name(f)
        if suffix != "bold":
            continue
        if all(str(ents.get(k)) in [str(v) for v in (vals if isinstance(vals, (list, tuple)) else [vals])]
               for k, vals in (filters or {}).items()):
            files.append(f)
    return files


def epi_mask(data, lower=0.2, upper=0.85, opening=2):
    """Brain mask of an EPI series: the mean image thresholded at the least
    dense point of its intensity histogram between the ``lower`` and ``upper``
    fractions of the sorted intensities (T. Nichols' heuristic), then a
    morphological opening and the largest connected component."""
    from scipy import ndimage

    mean = np.abs(np.asarray(data)).mean(axis=-1) if np.ndim(data) == 4 else np.abs(np.asarray(data))
    vals = np.sort(mean[mean != 0].ravel())
    if vals.size < 3:
        return np.zeros(mean.shape, dtype=bool)
    lo = int(lower * vals.size)
    hi = max(lo + 1, min(int(upper * vals.size), vals.size - 1))
    gaps = np.diff(vals[lo : hi + 1])
    k = int(np.argmax(gaps)) + lo
    mask = mean >= 0.5 * (vals[k] + vals[k + 1])
    if opening:
        mask = ndimage.binary_opening(mask, iterations=opening)
    lab, n = ndimage.label(mask)
    if n > 1:
        sizes = ndimage.sum(mask, lab, index=np.arange(1, n + 1))
        mask = lab == (int(np.argmax(sizes)) + 1)
    return mask


def _mask_of(run, data, verbose):
    """(mask, affine): nilearn's EPI masker for a NIfTI run when nilearn is installed, else epi_mask."""
    if ".nii" in "".join(Path(run).suffixes):
        try:
            from nilearn.maskers import NiftiMasker
        except ImportError:
            pass
        else:
            masker = NiftiMasker(verbose=verbose, mask_strategy="epi")
            masker.fit(str(run))
            return masker.mask_img_.get_fdata().astype(bool), masker.mask_img_.affine, masker
    return epi_mask(data), None, None


def update_dataset_description(output_dir):
    """Add this tool to ``GeneratedBy`` of the derivative dataset description."""
    ds_json = Path(output_dir) / "dataset_description.json"
    generated = {"Name": "patch-denoise", "Version": __version__,
                 "Description": "A dataset denoised with patch-denoise.",
                 "CodeURL": "https://github.com/paquiteau/patch-denoising"}
    if ds_json.exists():
        desc = json.loads(ds_json.read_text())
        if desc.get("GeneratedBy"):
            desc["GeneratedBy"].append(generated)
    else:
        desc = {"BIDSVersion": "1.9.0", "DatasetType": "derivative", "GeneratedBy": [generated]}
    ds_json.write_text(json.dumps(desc, indent=4, sort_keys=True))
    return desc


def bids_app(argv=None):
    """Denoise every selected BOLD run; returns the list of denoised files."""
    args = bids_parser().parse_args(argv)
    kwargs = args.extra or {}
    levels = [logging.WARNING, logging.INFO, logging.DEBUG]
    logging.basicConfig(level=levels[min(args.verbose, len(levels) - 1)])
    filters = {}
    if args.task_label:
        filters["task"] = args.task_label
    if args.session_label:
        filters["ses"] = args.session_label
    if args.bids_filter_file is not None:
        spec = json.loads(Path(args.bids_filter_file).read_text())
        filters.update(spec.get("bold", spec))
    if args.conf is not None:
        d = DenoiseParameters.from_str(args.conf)
        args.method, args.patch_shape, args.patch_overlap = d.method, d.patch_shape, d.patch_overlap
        args.recombination, args.mask_threshold = d.recombination, d.mask_threshold
    if args.method in NOISE_METHODS:
        # the BIDS app has no noise-map input (the reference raises here too)
        raise RuntimeError("A noise map must be specified for this method.")
    func = DENOISER_MAP.get(args.method)
    if func is None:
        raise ValueError(f"Method {args.method} is not supported.")
    out_root = Path(args.output_dir)
    out_root.mkdir(exist_ok=True, parents=True)
    update_dataset_description(out_root)
    written = []
    for sub in subjects(args.bids_dir, args.participant_label):
        for run in bold_runs(args.bids_dir, sub, filters):
            ents, _, ext = parse_bids_name(run)
            out_dir = out_root / f"sub-{ents['sub']}"
            if "ses" in ents:
                out_dir = out_dir / f"ses-{ents['ses']}"
            out_dir.mkdir(exist_ok=True, parents=True)
            ents = dict(ents, desc="denoised")
            out_bold = out_dir / bids_name(ents, "bold", ext)
            out_mask = out_dir / bids_name(ents, "mask", ext)
            out_std = out_dir / bids_name(ents, "std", ext)
            data, affine = load_as_array(run)
            mask, mask_affine, masker = _mask_of(run, data, args.verbose)
            if masker is not None:
                masker.generate_report().save_as_html(out_mask.with_suffix(".html"))
                masker.mask_img_.to_filename(out_mask)
            else:
                save_array(mask.astype(np.uint8), affine, out_mask)
            if args.gpu:
                from ..gpu import main_gpu

                denoised, _, noise_std_map = main_gpu(args, data, mask, None, **kwargs)
            else:
                denoised, _, noise_std_map, _ = func(data, patch_shape=args.patch_shape,
                                                     patch_overlap=args.patch_overlap, mask=mask,
                                                     mask_threshold=args.mask_threshold,
                                                     recombination=args.recombination, **kwargs)
            save_array(denoised, affine if affine is not None else mask_affine, out_bold)
            save_array(noise_std_map, affine if affine is not None else mask_affine, out_std)
            logging.info("denoised %s -> %s", run, out_bold)
            written.append(out_bold)
    return written


if __name__ == "__main__":
    bids_app()
