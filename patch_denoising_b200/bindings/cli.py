"""Command-line front end (bindings/cli.py:115-507, the non-BIDS ``patch-denoise``).

Same arguments, configuration strings and outputs as the reference's CLI; the
denoising runs on the GPU in both branches (``--gpu`` goes through ``main_gpu``,
the default through ``DENOISER_MAP``, as in the reference).

The reference computes the brain mask with nilearn's ``NiftiMasker`` (EPI
strategy) on the NIfTI input and saves it with an HTML report next to the
output. Here that happens when nilearn is installed; without nilearn (or for
``.npy`` inputs, which nilearn cannot read) ``--mask`` takes a ``.npy`` mask
file and no mask means every voxel.

    python -m patch_denoising_b200.bindings.cli noisy.npy denoised.npy --method mp-pca
"""

from __future__ import annotations

import argparse
import logging
import re
from functools import partial
from pathlib import Path

import numpy as np

from .. import __version__
from .utils import DENOISER_MAP, DenoiseParameters, load_as_array, load_complex_nifti, save_array

DENOISER_NAMES = ", ".join(d for d in DENOISER_MAP if d)
NOISE_METHODS = ("nordic", "hybrid-pca", "adaptive-qut", "optimal-fro-noise")


def _path_exists(path, parser):
    if path is None or not Path(path).exists():
        raise parser.error(f"Path does not exist: <{path}>.")
    return Path(path).absolute()


def _is_file(path, parser):
    path = _path_exists(path, parser)
    if not path.is_file():
        raise parser.error(f"Path should point to a file (or symlink of file): <{path}>.")
    return path


def _is_file_or_value(path, parser, *values):
    if path in values:
        return path
    return _is_file(path, parser)


def _positive_int(string, is_parser=True):
    """An integer >= 0 (cli.py:65-76)."""
    error = argparse.ArgumentTypeError if is_parser else ValueError
    try:
        value = int(string)
    except ValueError:
        raise error("Argument must be a nonnegative integer.") from None
    if value < 0:
        raise error("Int argument must be nonnegative.")
    return value


def _tuple_positive_int(string, is_parser=True):
    """``11`` or ``11x11x11`` (any non-digit separator) (cli.py:79-88)."""
    sep = re.search(r"\D", string)
    if sep is not None:
        return tuple(_positive_int(s, is_parser=is_parser) for s in string.split(sep.group(0)))
    return _positive_int(string, is_parser=is_parser)


class ToDict(argparse.Action):
    """``key=value`` pairs to a dict, float-like values as floats (cli.py:91-112)."""

    def __call__(self, parser, namespace, values, option_string=None):  # noqa: ARG002
        d = {}
        for spec in values:
            try:
                key, value = spec.split("=")
            except ValueError:
                raise ValueError("Extra arguments must be in the form key=value.") from None
            try:
                value = float(value)
            except ValueError:
                pass
            d[key] = value
        setattr(namespace, self.dest, d)


def get_parser():
    """The argument parser of ``patch-denoise`` (cli.py:115-369)."""
    parser = argparse.ArgumentParser(formatter_class=argparse.ArgumentDefaultsHelpFormatter)
    is_file = partial(_is_file, parser=parser)
    parser.add_argument("input_file", help="Input (noisy) file.", type=is_file)
    parser.add_argument("output_file", nargs="?", default=None, type=Path,
                        help="Output (denoised) file.\nDefault is D<input_file_name>.")
    parser.add_argument("--version", action="version", version=__version__)
    parser.add_argument("--gpu", action="store_true", help="Use GPU for computation if available.")
    den = parser.add_argument_group("Denoising parameters")
    exclusive = den.add_mutually_exclusive_group(required=True)
    exclusive.add_argument("--method", choices=DENOISER_MAP, default="optimal-fro",
                           help=f"Denoising method. Available denoising methods:\n  {DENOISER_NAMES}.")
    tuple_int = partial(_tuple_positive_int, is_parser=True)
    den.add_argument("--patch-shape", default=11, type=tuple_int, metavar="INT", help="Patch shape.")
    den.add_argument("--patch-overlap", default=5, type=tuple_int, metavar="INT", help="Patch overlap.")
    den.add_argument("--recombination", default="weighted", choices=["mean", "weighted"],
                     help="Recombination method.")
    den.add_argument("--mask-threshold", default=10, type=int, metavar="INT", help="Mask threshold.")
    exclusive.add_argument("--conf", default=None,
                           help="Denoising configuration "
                                "<name>_<patch-size>_<patch-overlap>_<recombination>_<mask_threshold>.")
    den.add_argument("--extra", metavar="key=value", default=None, nargs="+", action=ToDict,
                     help="extra key=value arguments for denoising methods.")
    data = parser.add_argument_group("Additional input data")
    data.add_argument("--mask", metavar="FILE|auto", default=None,
                      type=lambda path: _is_file_or_value(path, parser, "auto"),
                      help="mask file, if auto, it would be determined from the average image.")
    data.add_argument("--noise-map", metavar="FILE", default=None, type=is_file, help="noise map estimation file")
    data.add_argument("--input-phase", metavar="FILE", default=None, type=is_file,
                      help="Phase of the input data, in radians.")
    data.add_argument("--noise-map-phase", metavar="FILE", default=None, type=is_file,
                      help="Phase component of the noise map, in radians.")
    misc = parser.add_argument_group("Miscellaneous options")
    misc.add_argument("--output-noise-map", metavar="FILE", default=None, type=Path,
                      help="Output name for calculated noise map")
    misc.add_argument("--nan-to-num", metavar="VALUE", default=None, type=float,
                      help="Replace NaN by the provided value.")
    misc.add_argument("-v", "--verbose", action="count", default=0, help="Increase verbosity level.")
    return parser


def parse_args(argv=None):
    """Parse arguments and set the logging level (cli.py:372-384)."""
    args = get_parser().parse_args(argv)
    if not args.extra:
        args.extra = {}
    levels = [logging.WARNING, logging.INFO, logging.DEBUG]
    logging.basicConfig(level=levels[min(args.verbose, len(levels) - 1)])
    return args


def _mask(args):
    """(mask array or None, mask affine): nilearn's EPI masker when it can run, else a .npy mask."""
    if args.mask is not None and args.mask != "auto" and Path(args.mask).suffix == ".npy":
        return np.load(args.mask).astype(bool), None
    try:
        from nilearn.maskers import NiftiMasker
    except ImportError:
        if args.mask == "auto":
            raise RuntimeError("--mask auto needs nilearn, which is not installed") from None
        logging.warning("nilearn is not installed: denoising every voxel (give --mask FILE.npy to restrict)")
        return None, None
    if ".nii" not in Path(args.input_file).suffixes:
        if args.mask == "auto":
            raise RuntimeError("--mask auto needs a NIfTI input")
        return None, None
    masker = NiftiMasker(verbose=args.verbose, mask_strategy="epi")
    if args.mask != "auto" and args.mask is not None:
        masker.mask_img = args.mask
    masker.fit(args.input_file)
    if args.output_file is not None:
        masker.generate_report().save_as_html(Path(args.output_file).with_suffix(".html"))
        masker.mask_img_.to_filename(args.output_file.with_stem("mask_" + args.output_file.stem))
    return masker.mask_img_.get_fdata().astype(bool), masker.mask_img_.affine


def main(argv=None):
    """Command line entry point (cli.py:387-507)."""
    args = parse_args(argv)
    if args.output_file is None:
        args.output_file = Path(args.input_file).with_name("D" + Path(args.input_file).name)
    if args.input_phase is not None:
        input_data, affine = load_complex_nifti(args.input_file, args.input_phase)
    else:
        input_data, affine = load_as_array(args.input_file)
    kwargs = args.extra
    if args.nan_to_num is not None:
        input_data = np.nan_to_num(input_data, nan=args.nan_to_num)
    logging.info("Input data shape: %s", input_data.shape)
    n_nans = int(np.isnan(input_data).sum())
    if n_nans > 0:
        logging.warning("%d/%d voxels are NaN. You might want to use --nan-to-num=<value>", n_nans, input_data.size)
    mask, affine_mask = _mask(args)

    if args.noise_map is not None and args.noise_map_phase is not None:
        noise_map, affine_noise_map = load_complex_nifti(args.noise_map, args.noise_map_phase)
    elif args.noise_map is not None:
        noise_map, affine_noise_map = load_as_array(args.noise_map)
    elif args.noise_map_phase is not None:
        raise ValueError("The phase component of the noise map has been provided, but not the magnitude.")
    else:
        noise_map = affine_noise_map = None
    if affine is not None:
        if affine_mask is not None and not np.allclose(affine, affine_mask):
            logging.warning("Affine matrix of input and mask does not match")
        if affine_noise_map is not None and not np.allclose(affine, affine_noise_map):
            logging.warning("Affine matrix of input and noise map does not match")

    if args.conf is not None:
        d = DenoiseParameters.from_str(args.conf)
        args.method, args.patch_shape, args.patch_overlap = d.method, d.patch_shape, d.patch_overlap
        args.recombination, args.mask_threshold = d.recombination, d.mask_threshold
    Path(args.output_file).parent.mkdir(exist_ok=True, parents=True)

    if args.gpu:
        from ..gpu import main_gpu

        denoised, _, noise_std_map = main_gpu(args, input_data, mask, noise_map, **kwargs)
    else:
        if args.method in NOISE_METHODS:
            if noise_map is None:
                raise RuntimeError("A noise map must be specified for this method.")
            kwargs["noise_std"] = noise_map
        func = DENOISER_MAP.get(args.method, None)
        if func is None:
            raise ValueError(f"Method {args.method} is not supported.")
        denoised, _, noise_std_map, _ = func(input_data, patch_shape=args.patch_shape,
                                             patch_overlap=args.patch_overlap, mask=mask,
                                             mask_threshold=args.mask_threshold,
                                             recombination=args.recombination, **kwargs)
    save_array(denoised, affine, args.output_file)
    save_array(noise_std_map, affine, args.output_noise_map)
    return args.output_file


if __name__ == "__main__":
    main()
