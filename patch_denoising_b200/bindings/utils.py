"""Method registry, configuration strings and array I/O (bindings/utils.py:20-173)."""

from __future__ import annotations

import logging
import pathlib
from dataclasses import dataclass

import numpy as np

from ..denoise import (
    adaptive_thresholding,
    hybrid_pca,
    mp_pca,
    nordic,
    optimal_thresholding,
    raw_svt,
)

DENOISER_MAP = {
    None: None,
    "mp-pca": mp_pca,
    "hybrid-pca": hybrid_pca,
    "raw": raw_svt,
    "optimal-fro": lambda *args, **kwargs: optimal_thresholding(*args, loss="fro", **kwargs),
    "optimal-fro-noise": lambda *args, **kwargs: optimal_thresholding(*args, loss="fro", **kwargs),
    "optimal-nuc": lambda *args, **kwargs: optimal_thresholding(*args, loss="nuc", **kwargs),
    "optimal-ope": lambda *args, **kwargs: optimal_thresholding(*args, loss="ope", **kwargs),
    "nordic": nordic,
    "adaptive-qut": lambda *args, **kwargs: adaptive_thresholding(*args, method="qut", **kwargs),
}

_RECOMBINATION = {"w": "weighted", "c": "center", "a": "average"}


@dataclass
class DenoiseParameters:
    """Denoising configuration, serialisable as ``method_patch_overlap_recomb_maskthr``."""

    method: str | None = None
    patch_shape: int | tuple = 11
    patch_overlap: int | tuple = 0
    recombination: str = "weighted"
    mask_threshold: int = 10

    @property
    def pretty_name(self):
        """Configuration string of these parameters."""
        if self.method:
            name = self.method
            for attr in ["patch_shape", "patch_overlap", "recombination", "mask_threshold"]:
                if getattr(self, attr):
                    name += f"_{getattr(self, attr)}"
        else:
            name = "noisy"
        return name

    @property
    def pretty_par(self):
        """Short form of the patch parameters."""
        return f"{self.patch_shape}_{self.patch_overlap}{self.recombination[0]}"

    @classmethod
    def get_str(cls, **kwargs):
        """Configuration string from keyword arguments."""
        return cls(**kwargs).pretty_name

    @classmethod
    def from_str(cls, config_str):
        """Parse a configuration string (bindings/utils.py:84-109)."""
        if "noisy" in config_str:
            return DenoiseParameters(method=None, patch_shape=None, patch_overlap=None, recombination=None,
                                     mask_threshold=None)
        conf = config_str.split("_")
        d = DenoiseParameters()
        if conf:
            d.method = conf.pop(0)
        if conf:
            d.patch_shape = int(conf.pop(0))
        if conf:
            d.patch_overlap = int(conf.pop(0))
        if conf:
            d.recombination = conf.pop(0)
        if conf:
            d.mask_threshold = int(conf.pop(0))
        return d

    def __str__(self):
        return self.pretty_name


def load_as_array(input):
    """Load ``.npy`` (or NIfTI when nibabel is installed); returns (array, affine)."""
    if input is None:
        return None, None
    input = pathlib.Path(input)
    if input.suffix == ".npy":
        return np.load(input), None
    if ".nii" in input.suffixes:
        try:
            import nibabel as nib
        except ImportError as exc:  # pragma: no cover - depends on the environment
            raise ValueError("NIfTI input needs nibabel, which is not installed") from exc
        nii = nib.load(input)
        return nii.get_fdata(dtype=np.float32), nii.affine
    raise ValueError("Unsupported file format. use numpy or nifti formats.")


def save_array(data, affine, filename):
    """Save to ``.npy`` (or NIfTI when nibabel is installed)."""
    if filename is None:
        return None
    filename = pathlib.Path(filename)
    if ".nii" in filename.suffixes:
        import nibabel as nib

        if affine is None:
            affine = np.eye(len(data.shape))
        nib.Nifti1Image(data, affine).to_filename(filename)
    elif filename.suffix == ".npy":
        np.save(filename, data)
    return filename


def load_complex_nifti(mag_file, phase_file, filename=None):  # pragma: no cover - needs nibabel
    """Magnitude + phase images -> complex array (bindings/utils.py:147-173)."""
    mag, mag_affine = load_as_array(mag_file)
    phase, phase_affine = load_as_array(phase_file)
    if mag_affine is not None and phase_affine is not None and not np.allclose(mag_affine, phase_affine):
        logging.warning("Affine matrices for magnitude and phase are not the same")
    img = mag * np.exp(1j * phase)
    if filename is not None:
        np.save(filename, img)
    return img, mag_affine
