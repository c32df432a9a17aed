"""CPU oracle for the space-time low-rank denoising path. TEST INFRASTRUCTURE ONLY.

This module restates, in NumPy + SciPy (``scipy.linalg.eigh`` / ``svd`` and
``scipy.integrate.quad``, SciPy 1.18.1 -- the same third-party LAPACK calls the
reference makes), the algorithm of paquiteau/patch-denoising's ``space_time``
package. Every function names the reference lines it follows (paths are relative
to the reference project root). It is the checker for the CUDA path and the timed
CPU reference arm of ``bench.py``; the product package never imports it.

Parity pin: ``tests/test_oracle_golden.py`` checks this module against
``tests/golden/*.npz``, which ``tests/golden/make_golden.py`` produced by running
the reference package itself on seeded inputs.

Beyond the reference, the oracle
  * records the per-patch ``(maxidx, noise_var)`` that every reference
    ``_patch_processing`` returns but ``denoise`` drops, and fills the voxel rank
    and noise maps from them (the reference returns all-zero maps);
  * records a per-patch decision margin (relative distance of the closest
    threshold comparison), so tests can name near-threshold ties;
  * accepts ``rank_override`` = {patch index: maxidx} to replay a decision taken
    by another implementation at a near-tie, so outputs can be compared exactly.
"""

from __future__ import annotations

import numpy as np
from scipy.integrate import quad
from scipy.linalg import eigh, svd

METHODS = ("mp-pca", "hybrid-pca", "raw", "nordic", "optimal")

# --------------------------------------------------------------------------- #
# Patch geometry                                                              #
# --------------------------------------------------------------------------- #


def patch_params(data_shape, patch_shape, patch_overlap):
    """int / list / tuple -> full patch shape and overlap (time axis appended).

    Follows ``src/patch_denoise/space_time/base.py:359-384``.
    """
    res = []
    for p in (patch_shape, patch_overlap):
        if isinstance(p, list):
            p = tuple(p)
        elif isinstance(p, (int, np.integer)):
            p = (p,) * (len(data_shape) - 1)
        if len(p) == len(data_shape) - 1:
            p = (*p, data_shape[-1])
        res.append(tuple(int(v) for v in p))
    return res[0], res[1]


def grid_geometry(data_shape, p_s, p_o):
    """Patch grid of the strided sliding view: (effective patch, step, grid).

    Follows ``space_time/base.py:37-82``: step = patch - overlap is taken before
    the patch is clamped to the array; a dimension whose (clamped) patch covers
    the whole axis has a single grid position; there is no trailing partial
    patch. A zero step on a covered axis gives NumPy's ``x // 0 == 0`` (one grid
    position), which is mirrored here.
    """
    ps = np.asarray(p_s, dtype=np.int64)
    step = ps - np.asarray(p_o, dtype=np.int64)
    if np.any(step < 0):
        raise ValueError("overlap should be smaller than patch on every dimension.")
    if ps.size != len(data_shape) or step.size != len(data_shape):
        raise ValueError("patch shape and overlap must match the input dimensions")
    ps = np.minimum(ps, data_shape)
    grid = []
    for n, p, s in zip(data_shape, ps, step):
        if p < n:
            grid.append(int((n - p) // s + 1) if s > 0 else 1)
        else:
            grid.append(1)
    return tuple(int(v) for v in ps), tuple(int(v) for v in step), tuple(grid)


def _patch_slices(idx, ps, step, grid):
    """Slices of the linear patch ``idx`` (``space_time/base.py:89-103``)."""
    g = np.unravel_index(idx, grid)
    return tuple(slice(int(gi) * s, int(gi) * s + p) for gi, p, s in zip(g, ps, step))


def _broadcast_mask(mask, data_shape):
    """Mask normalisation of ``space_time/base.py:202-211``."""
    if mask is None:
        return np.full(data_shape, True)
    mask = np.asarray(mask)
    if mask.shape == tuple(data_shape):
        return mask
    if mask.shape == tuple(data_shape[:-1]):
        return np.broadcast_to(mask[..., None], data_shape)
    raise ValueError(f"Mask shape {mask.shape} is incompatible with input {data_shape}.")


def select_patches(mask4d, ps, step, grid, mask_threshold):
    """Indices of the patches whose mask fill is strictly above the threshold.

    Follows ``space_time/base.py:220-227``: ``100 * sum(pm) / pm.size > thr``.
    """
    n_patches = int(np.prod(grid))
    keep = np.zeros(n_patches, dtype=bool)
    for i in range(n_patches):
        pm = mask4d[_patch_slices(i, ps, step, grid)]
        if 100 * np.sum(pm) / pm.size > mask_threshold:
            keep[i] = True
    return np.nonzero(keep)[0]


# --------------------------------------------------------------------------- #
# Per-patch linear algebra                                                    #
# --------------------------------------------------------------------------- #


def svd_analysis(x):
    """Centred thin SVD, ``space_time/utils.py:58-78``."""
    mean = np.mean(x, axis=0)
    xc = x - mean
    u, s, vt = svd(xc, full_matrices=False)
    return u, s, vt, mean


def svd_synthesis(u, s, vt, mean, k):
    """``U[:, :k] (s[:k] Vt[:k]) + mean``, ``space_time/utils.py:81-99``."""
    return (u[:, :k] @ (s[:k, None] * vt[:k, :])) + mean


def eig_analysis(x, max_eig_val=10):
    """Top eigenpairs of the centred autocorrelation, ``space_time/utils.py:102-137``.

    ``C = Xc^H Xc / (M - 1)`` (T x T); LAPACK ``?syevx/?heevx`` restricted to the
    ``max_eig_val`` largest eigenvalues, returned in ascending order.
    """
    mean = np.mean(x, axis=0)
    xc = x - mean
    m = xc.shape[0]
    n = mean.shape[0]
    vals, vecs = eigh(
        xc.conj().T @ xc / (m - 1),
        driver="evx",
        subset_by_index=(n - max_eig_val, n - 1),
    )
    return xc, vals, vecs, mean


def eig_synthesis(xc, vecs, mean, k):
    """Projection on the last ``k`` eigenvector columns, ``space_time/utils.py:140-146``."""
    vecs = vecs.copy()
    vecs[:, :-k] = 0
    return ((xc @ vecs) @ vecs.conj().T) + mean


def marchenko_pastur_median(beta, eps=1e-7):
    """Median of the Marchenko-Pastur law by 5-point dichotomy.

    Follows ``space_time/utils.py:149-204``: up to 20 rounds, the CDF at each of
    the 5 ``linspace`` points is a ``quad`` integral of the density from the lower
    edge; the bracket shrinks to the points on either side of 1/2.
    """
    if not (0 <= beta <= 1):
        raise ValueError("Aspect Ratio should be between 0 and 1")
    hi_edge = (1 + np.sqrt(beta)) ** 2
    lo_edge = (1 - np.sqrt(beta)) ** 2

    def density(t):
        if hi_edge >= t >= lo_edge:
            return np.sqrt((hi_edge - t) * (t - lo_edge)) / (2 * np.pi * t * beta)
        return 0

    lo, hi = lo_edge, hi_edge
    moved = True
    rounds = 0
    while moved and (hi - lo) > eps and rounds < 20:
        moved = False
        pts = np.linspace(lo, hi, 5)
        cdf = np.array([quad(density, lo_edge, p)[0] for p in pts])
        if np.any(cdf < 0.5):
            lo = np.max(pts[cdf < 0.5])
            moved = True
        if np.any(cdf > 0.5):
            hi = np.min(pts[cdf > 0.5])
            moved = True
        rounds += 1
    return (lo + hi) / 2


def nordic_threshold(p_s, n_frames, noise_std, n_iter_threshold=10, rng=None):
    """Monte-Carlo NORDIC threshold, ``space_time/lowrank.py:221-242``.

    ``noise_std * mean_n max sigma(randn(prod(p_s), T))``; ``prod(p_s)`` includes
    the time extent of the patch. ``rng`` defaults to NumPy's global generator,
    as in the reference.
    """
    gen = np.random if rng is None else rng
    acc = 0
    for _ in range(n_iter_threshold):
        acc = acc + max(svd(gen.randn(int(np.prod(p_s)), n_frames), compute_uv=False))
    acc /= n_iter_threshold
    if isinstance(noise_std, np.ndarray):
        noise_std = np.mean(noise_std)
    if not isinstance(noise_std, (float, np.floating)):
        raise ValueError(
            "For NORDIC the noise level must be either an"
            " array or a float specifying the std in the volume."
        )
    return noise_std * acc


# --------------------------------------------------------------------------- #
# Threshold rules (one patch)                                                 #
# --------------------------------------------------------------------------- #


def _rel(a, b):
    den = max(abs(float(a)), abs(float(b)), 1e-300)
    return abs(float(a) - float(b)) / den


def _mppca_patch(x, threshold_scale, override=None):
    """``MPPCADenoiser._patch_processing``, ``space_time/lowrank.py:42-63``."""
    xc, lam, vecs, mean = eig_analysis(x)
    n_eig = len(lam)
    n_rows = len(x)
    n_vec = len(vecs)
    margin = np.inf
    k = 0
    crit = np.mean(lam)
    crit = crit * (4 * np.sqrt((n_eig - k + 1) / n_rows))
    while k < n_eig:
        rhs = lam[n_eig - 1 - k] - lam[0]
        margin = min(margin, _rel(crit, rhs))
        if not crit < rhs:
            break
        k += 1
        with np.errstate(invalid="ignore", divide="ignore"):
            crit = np.mean(lam[: n_eig - k]) if n_eig - k > 0 else np.float64("nan")
        crit = crit * (4 * np.sqrt((n_vec - k + 1) / n_rows))
    with np.errstate(invalid="ignore", divide="ignore"):
        var_noise = np.mean(lam[: n_eig - k]) if n_eig - k > 0 else lam.dtype.type("nan")
    cut = var_noise * threshold_scale**2
    rank = np.sum(lam > cut)  # np.int64, as in the reference (sets theta's promotion)
    for v in lam:
        margin = min(margin, _rel(v, cut))
    if override is not None:
        rank = np.int64(override)
    if rank == 0:
        new = np.zeros_like(x) + mean
    else:
        new = eig_synthesis(xc, vecs, mean, rank)
    return new, rank, var_noise, margin


def _hybrid_patch(x, varest, override=None):
    """``HybridPCADenoiser._patch_processing``, ``space_time/lowrank.py:104-119``."""
    xc, lam, vecs, mean = eig_analysis(x)
    n_eig = len(lam)
    margin = np.inf
    k = 0
    var_noise = np.mean(lam)
    while True:
        margin = min(margin, _rel(var_noise, varest))
        if not (var_noise > varest and k < n_eig - 2):
            break
        k += 1
        var_noise = np.mean(lam[: n_eig - k])
    rank = k if override is None else int(override)
    if rank == 0:
        new = np.zeros_like(x) + mean
    else:
        new = eig_synthesis(xc, vecs, mean, rank)
    return new, rank, var_noise, margin


def _raw_patch(x, threshold, override=None):
    """``RawSVDDenoiser._patch_processing``, ``space_time/lowrank.py:170-184``."""
    u, s, vt, mean = svd_analysis(x)
    rank = np.sum(s > threshold)  # np.int64, as in the reference
    margin = min((_rel(v, threshold) for v in s), default=np.inf)
    if override is not None:
        rank = np.int64(override)
    if rank == 0:
        new = np.zeros_like(x) + mean
    else:
        s = s.copy()
        s[s < threshold] = 0
        new = svd_synthesis(u, s, vt, mean, rank)
    return new, rank, np.nan, margin


def _opt_loss_x(y, beta):
    """Eq. (8) of Gavish-Donoho, ``space_time/lowrank.py:250-255``."""
    tmp = y**2 - beta - 1
    return np.sqrt(0.5 * (tmp + np.sqrt((tmp**2) - (4 * beta)))) * (y >= (1 + np.sqrt(beta)))


def _opt_ope_shrink(s, beta=1):
    """``space_time/lowrank.py:258-260``."""
    return np.maximum(_opt_loss_x(s, beta), 0)


def _opt_nuc_shrink(s, beta=1):
    """``space_time/lowrank.py:263-269``."""
    tmp = _opt_loss_x(s, beta)
    return np.maximum(0, (tmp**4 - (np.sqrt(beta) * tmp * s) - beta)) / ((tmp**2) * s)


def _opt_fro_shrink(s, beta=1):
    """``space_time/lowrank.py:272-280`` (the square root covers the quotient)."""
    return np.sqrt(np.maximum((((s**2) - beta - 1) ** 2 - 4 * beta), 0) / s)


SHRINKERS = {"fro": _opt_fro_shrink, "nuc": _opt_nuc_shrink, "ope": _opt_ope_shrink}


def _optimal_patch(x, loss, mp_median, sigma_prior=None, override=None):
    """``OptimalSVDDenoiser._patch_processing``, ``space_time/lowrank.py:379-407``."""
    u, s, vt, mean = svd_analysis(x)
    n_rows, n_cols = x.shape
    if sigma_prior is not None:
        sigma = sigma_prior
    else:
        sigma = np.median(s) / np.sqrt(n_cols * mp_median)
    scale = np.sqrt(n_cols) * sigma
    beta = n_cols / n_rows
    with np.errstate(invalid="ignore", divide="ignore"):
        shrunk = scale * SHRINKERS[loss](s / scale, beta=beta)
    shrunk[np.isnan(shrunk)] = 0
    # margin: relative distance of y to the decision edges of the shrinker
    y = s / scale
    margin = np.inf
    edge_hi = 1 + np.sqrt(beta)
    for v in y:
        margin = min(margin, _rel(v, edge_hi))
        if loss == "fro":
            margin = min(margin, _rel((v**2 - beta - 1) ** 2, 4 * beta))
    if np.any(shrunk):
        rank = np.max(np.nonzero(shrunk)) + 1  # np.int64, as in the reference
    else:
        rank = 0
    if override is not None:
        rank = np.int64(override) if override else 0
        shrunk = shrunk.copy()
        shrunk[rank:] = 0
    if rank == 0:
        new = np.zeros_like(x) + mean
    else:
        new = svd_synthesis(u, shrunk, vt, mean, rank)
    return new, rank, np.nan, margin


# --------------------------------------------------------------------------- #
# Driver                                                                      #
# --------------------------------------------------------------------------- #


def _prior_patches(noise_std, data_shape):
    """``noise_std**2`` broadcast over time (``space_time/lowrank.py:94-100``)."""
    if isinstance(noise_std, (float, np.floating)):
        var = noise_std**2 * np.ones(data_shape[:-1])
    else:
        var = noise_std**2
    return np.broadcast_to(var[..., None], data_shape)


def denoise(
    method,
    data,
    patch_shape,
    patch_overlap,
    recombination="weighted",
    mask=None,
    mask_threshold=50,
    *,
    threshold_scale=1.0,
    threshold_value=1.0,
    noise_std=None,
    loss="fro",
    eps_marshenko_pastur=1e-7,
    n_iter_threshold=10,
    nordic_rng=None,
    threshold=None,
    rank_override=None,
):
    """Whole-volume denoising: ``BaseSpaceTimeDenoiser.denoise`` + method setup.

    Follows ``space_time/base.py:177-270`` for the driver and
    ``space_time/lowrank.py`` for the method set-up (``HybridPCADenoiser.denoise``
    :76-102, ``RawSVDDenoiser.denoise`` :142-168, ``NordicDenoiser.denoise``
    :197-246, ``OptimalSVDDenoiser.denoise`` :318-377).

    ``threshold`` (raw / nordic) replaces the computed singular-value threshold.
    Returns a dict with the reference outputs ``out``, ``weights`` and the
    extension outputs ``noise_map``, ``rank_map``, ``patches``, ``patch_rank``,
    ``patch_noise``, ``patch_margin``, ``threshold``, ``mp_median``.
    """
    if method not in METHODS:
        raise ValueError(f"unknown method {method}")
    if recombination not in ("weighted", "average", "center"):
        raise ValueError("recombination must be one of 'weighted', 'average', 'center'")
    data = np.asarray(data)
    data_shape = data.shape
    p_s, p_o = patch_params(data_shape, patch_shape, patch_overlap)
    ps, step, grid = grid_geometry(data_shape, p_s, p_o)
    if tuple(ps) != tuple(p_s):
        raise ValueError("patch larger than the input along some axis")
    n_rows = int(np.prod(p_s[:-1]))

    # ---- method set-up -------------------------------------------------------
    prior = None
    mp_med = None
    thr = None
    if method == "hybrid-pca":
        prior = _prior_patches(1.0 if noise_std is None else noise_std, data_shape)
    elif method == "raw":
        thr = threshold_value * threshold_scale if threshold is None else threshold
    elif method == "nordic":
        if threshold is None:
            thr = nordic_threshold(
                p_s, data_shape[-1], 1.0 if noise_std is None else noise_std,
                n_iter_threshold, nordic_rng,
            )
        else:
            thr = threshold
    elif method == "optimal":
        mp_med = marchenko_pastur_median(p_s[-1] / np.prod(p_s[:-1]), eps=eps_marshenko_pastur)
        if noise_std is not None:
            prior = _prior_patches(noise_std, data_shape)

    # ---- driver (base.py:193-270) ------------------------------------------
    out = np.zeros(data_shape, dtype=data.dtype)
    weights = np.zeros(data_shape, dtype=np.float32)
    noise_acc = np.zeros(data_shape, dtype=np.float64)
    rank_map = np.zeros(data_shape, dtype=np.int32)
    noise_center = np.zeros(data_shape, dtype=np.float32)
    mask4d = _broadcast_mask(mask, data_shape)
    center = tuple(p // 2 for p in p_s)
    sel = select_patches(mask4d, ps, step, grid, mask_threshold)
    ranks = np.zeros(len(sel), dtype=np.int64)
    noises = np.zeros(len(sel), dtype=np.float64)
    margins = np.zeros(len(sel), dtype=np.float64)
    override = rank_override or {}

    for j, i in enumerate(sel):
        sl = _patch_slices(i, ps, step, grid)
        x = data[sl].reshape(n_rows, -1)
        ov = override.get(int(i))
        if method == "mp-pca":
            new, rank, nvar, marg = _mppca_patch(x, threshold_scale, ov)
        elif method == "hybrid-pca":
            new, rank, nvar, marg = _hybrid_patch(x, np.mean(prior[sl]), ov)
        elif method in ("raw", "nordic"):
            new, rank, nvar, marg = _raw_patch(x, thr, ov)
        else:
            sig = None if prior is None else np.mean(np.sqrt(prior[sl]))
            new, rank, nvar, marg = _optimal_patch(x, loss, mp_med, sig, ov)
        ranks[j], noises[j], margins[j] = rank, nvar, marg
        new = np.reshape(new, p_s)
        corner = tuple(s.start for s in sl)
        cpos = tuple(c + o for c, o in zip(corner, center))
        if recombination == "center":
            out[sl][center] = new[center]
            if not np.isnan(nvar):
                noise_center[cpos] = nvar
        elif recombination == "weighted":
            theta = 1 / (2 + rank)
            out[sl] += new * theta
            weights[sl] += theta
            if not np.isnan(nvar):
                noise_acc[sl] += theta * nvar
        else:
            out[sl] += new
            weights[sl] += 1
            if not np.isnan(nvar):
                noise_acc[sl] += nvar
        # rank map: maxidx at the spatial centre, over the patch's time span
        rsl = tuple(slice(c, c + 1) for c in cpos[:-1]) + (sl[-1],)
        np.maximum(rank_map[rsl], rank, out=rank_map[rsl])

    with np.errstate(invalid="ignore", divide="ignore"):
        if recombination in ("average", "weighted"):
            out /= weights
            noise_map = (noise_acc / weights).astype(np.float32)
        else:
            noise_map = noise_center
    out[~mask4d] = 0
    noise_map[~mask4d] = 0
    return {
        "out": out,
        "weights": weights,
        "noise_map": noise_map,
        "rank_map": rank_map,
        "patches": sel,
        "patch_rank": ranks,
        "patch_noise": noises,
        "patch_margin": margins,
        "threshold": thr,
        "mp_median": mp_med,
    }


# --------------------------------------------------------------------------- #
# Noise map from a noise-only sequence                                        #
# --------------------------------------------------------------------------- #
def patch_locs(p_shape, p_ovl, v_shape):
    """Top-left corners of all patches (space_time/utils.py:8-55, ``get_patch_locs``).

    Per axis: ``arange(0, v - p, p - o)`` plus the last index ``v - p`` when the
    range stops short of it; an axis with ``v <= p`` gives an empty range, on
    which the reference's ``range_[-1]`` raises IndexError, as here.
    """
    if len(v_shape) != len(p_shape) or len(v_shape) != len(p_ovl):
        raise ValueError(f"Dimension mismatch between the arguments. {p_shape}{p_ovl}, {v_shape}")
    ranges = []
    for v_s, p_s, p_o in zip(v_shape, p_shape, p_ovl):
        if p_o >= p_s:
            raise ValueError("Overlap should be a non-negative integer smaller than patch_size")
        last = v_s - p_s
        r = np.arange(0, last, p_s - p_o, dtype=np.int32)
        if r[-1] < last:  # IndexError on an empty range, as in the reference
            r = np.append(r, last)
        ranges.append(r)
    grids = np.meshgrid(*ranges, indexing="ij")
    return np.stack([g.reshape(-1) for g in grids], axis=1)


def estimate_noise(noise_sequence, block_size=1):
    """Noise map of a noise-only sequence (space_time/utils.py:207-242).

    For every block of ``block_size`` voxels per spatial axis (overlap
    ``block_size - 1``: every position), the voxel at the block's centre
    (top-left + ``block_size // 2``) gets the population standard deviation of
    all the block's samples over all frames. Computed in float64. Voxels no
    block centres on are left at 0 (the reference leaves ``np.empty`` content
    there, which is undefined).
    """
    x = np.asarray(noise_sequence)
    x = x.astype(np.complex128 if np.iscomplexobj(x) else np.float64)
    v_shape = x.shape[:-1]
    b = int(block_size)
    out = np.zeros(v_shape)
    p_shape = (b,) * len(v_shape)
    for tl in patch_locs(p_shape, (b - 1,) * len(v_shape), v_shape):
        sl = tuple(slice(t, t + b) for t in tl)
        ctr = tuple(int(t) + b // 2 for t in tl)
        out[ctr] = np.std(x[sl])
    return out


def estimate_noise_covered(v_shape, block_size):
    """Boolean map of the voxels ``estimate_noise`` writes (the block centres)."""
    b = int(block_size)
    cov = np.zeros(v_shape, dtype=bool)
    sl = tuple(slice(b // 2, v - b + b // 2 + 1) for v in v_shape)
    cov[sl] = True
    return cov
