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
from scipy.optimize import minimize

METHODS = ("mp-pca", "hybrid-pca", "raw", "nordic", "optimal", "adaptive")

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
# Adaptive trace-norm shrinkage (AdaptiveDenoiser)                            #
# --------------------------------------------------------------------------- #
def sure_atn_cost(x_shape, method, s, gamma, sigma, tau):
    """``_sure_atn_cost``, ``space_time/lowrank.py:410-447``: the (G)SURE cost of
    the shrinkage d = s max(1 - (tau/s)^gamma, 0). For "qut" the variable is
    log(gamma - 1), else log tau; the divergence matrix D is float32, as there."""
    n_rows, n_cols = x_shape
    if method == "qut":
        gamma = np.exp(gamma) + 1
    else:
        tau = np.exp(tau)
    s2 = s**2
    d_hat = s * np.maximum(1 - (tau / s) ** gamma, 0)
    sd = s * d_hat
    dmat = np.zeros((len(s), len(s)), dtype=np.float32)
    for i in range(len(s)):
        gap = s2[i] - s2
        gap[i] = np.inf
        dmat[i, :] = sd[i] / gap
    grad = (1 + (gamma - 1) * (tau / s) ** gamma) * (s >= tau)
    div = np.sum(grad + abs(n_rows - n_cols) * d_hat / s) + 2 * np.sum(dmat)
    rss = np.sum((d_hat - s) ** 2)
    if method == "gsure":
        return rss / (1 - div / n_rows / n_cols) ** 2
    return sigma**2 * (-n_rows * n_cols + 2 * div) + rss


def atn_shrink(s, gamma, tau):
    """``_atn_shrink``, ``space_time/lowrank.py:459-461``."""
    return s * np.maximum(1 - (tau / s) ** gamma, 0)


def qut_level(x_shape, nbsim, rng=None):
    """The QUT quantile for a unit noise estimate: ``_get_gamma_tau_qut``'s
    ``maxd`` draws and quantile (``space_time/lowrank.py:466-475``) divided by stdest."""
    rng = np.random if rng is None else rng
    maxd = np.ones(nbsim)
    for i in range(nbsim):
        maxd[i] = np.max(svd(rng.randn(*x_shape), compute_uv=False, overwrite_a=True))
    return np.quantile(maxd, 1 - 1 / np.sqrt(np.log(max(*x_shape))))


def atn_cost64(s, si, x_shape, lt, gamma, sigma, gsure):
    """The (G)SURE cost of ``sure_atn_cost`` at log tau = ``lt`` in float64, with
    sum_ij D_ij = sum_i s_i d_i si_i (si_i = sum_{j != i} 1 / (s_i^2 - s_j^2)):
    the form the library evaluates on the device."""
    n_rows, n_cols = x_shape
    tau = np.exp(lt)
    s, si = s[s > 0], si[s > 0]  # zero singular values add nothing (their terms vanish as s -> 0)
    r = np.exp(gamma * (lt - np.log(s)))
    d_hat = s * np.maximum(1 - r, 0)
    div = np.sum((1 + (gamma - 1) * r) * (s >= tau) + abs(n_rows - n_cols) * d_hat / s) + 2 * np.sum(s * d_hat * si)
    rss = np.sum((d_hat - s) ** 2)
    if gsure:
        return rss / (1 - div / n_rows / n_cols) ** 2
    return sigma**2 * (2 * div - n_rows * n_cols) + rss


def _brent_min(f, a, b, tol=1e-10):
    """Brent's minimisation on [a, b] (golden section with parabolic steps; Brent 1973, ch. 5)."""
    cg = 0.3819660112501051
    x = w = v = a + cg * (b - a)
    fx = fw = fv = f(x)
    d = e = 0.0
    for _ in range(200):
        m = 0.5 * (a + b)
        tol1 = tol * abs(x) + 1e-12
        tol2 = 2 * tol1
        if abs(x - m) <= tol2 - 0.5 * (b - a):
            break
        golden = True
        if abs(e) > tol1:
            r = (x - w) * (fx - fv)
            q = (x - v) * (fx - fw)
            pp = (x - v) * q - (x - w) * r
            q = 2 * (q - r)
            if q > 0:
                pp = -pp
            else:
                q = -q
            e_old, e = e, d
            if abs(pp) < abs(0.5 * q * e_old) and q * (a - x) < pp < q * (b - x):
                d = pp / q
                if (x + d) - a < tol2 or b - (x + d) < tol2:
                    d = tol1 if x < m else -tol1
                golden = False
        if golden:
            e = (b - x) if x < m else (a - x)
            d = cg * e
        u = x + d if abs(d) >= tol1 else x + (tol1 if d > 0 else -tol1)
        fu = f(u)
        if fu <= fx:
            if u < x:
                b = x
            else:
                a = x
            v, fv, w, fw, x, fx = w, fw, x, fx, u, fu
        else:
            if u < x:
                a = u
            else:
                b = u
            if fu <= fw or w == x:
                v, fv, w, fw = w, fw, u, fu
            elif fu <= fv or v == x or v == w:
                v, fv = u, fu
    return x


def line_search_min(f, x0, lo=-700.0, hi=700.0):
    """The library's minimisation from x0 on [lo, hi]: forward-difference slope
    (step 1.49e-8), first trial step -g min(1, 1.01/|g|) (as BFGS's first
    line-search point), golden growth while the cost falls, then Brent inside
    the bracket."""
    h = 1.4901161193847656e-08
    x0 = min(max(x0, lo), hi)
    fa = f(x0)
    g = (f(x0 + h) - fa) / h
    if not abs(g) > 0:
        return x0
    a, b = x0, min(max(x0 - g * min(1.0, 1.01 / abs(g)), lo), hi)
    if b == a:
        return x0
    fb = f(b)
    if fb < fa:
        c = min(max(b + 1.618033988749895 * (b - a), lo), hi)
        fc = f(c)
        for _ in range(60):
            if not (fc < fb and c != b and lo < c < hi):
                break
            a, fa, b, fb = b, fb, c, fc
            c = min(max(b + 1.618033988749895 * (b - a), lo), hi)
            fc = f(c)
        return _brent_min(f, min(a, c), max(a, c))
    return _brent_min(f, min(a, b), max(a, b))


def _adaptive_patch(x, stdest, method, gamma0, tau0, nbsim, qlevel=None, rng=None, override=None,
                    optimizer="bfgs"):
    """``AdaptiveDenoiser._patch_processing`` with ``_get_gamma_tau`` /
    ``_get_gamma_tau_qut`` (``space_time/lowrank.py:464-533, 607-636``).
    ``qlevel`` replaces the per-patch QUT draws (tau = stdest * qlevel).
    ``optimizer="bfgs"``: scipy's BFGS on the float32-D cost, as the reference.
    ``optimizer="search"``: the library's line search + Brent on the float64 cost
    (``atn_cost64``), a deterministic function of the singular values."""
    u, s, vt, mean = svd_analysis(x)
    if optimizer == "search":
        s = s.astype(np.float64)  # the cost in float64 whatever the patch's precision
        if x.shape[0] <= x.shape[1]:
            # a centred M x T patch with M <= T has rank M - 1 at most: its last
            # singular values are zero (rounding leaves them tiny), as the library takes them
            s = s.copy()
            s[x.shape[0] - 1 :] = 0.0
        s2 = s**2
        with np.errstate(divide="ignore"):
            si = np.array([np.sum(1.0 / (s2[k] - np.delete(s2, k))) if s[k] > 0 else 0.0 for k in range(len(s))])
        gs = method == "gsure"
        if method == "qut":
            tau = stdest * qlevel
            if isinstance(gamma0, (float, np.floating)):
                gamma = gamma0
            else:
                lt = np.log(tau)
                gamma = np.exp(line_search_min(lambda g: atn_cost64(s, si, x.shape, lt, np.exp(g) + 1, stdest, gs),
                                               0.0)) + 1
        else:
            pos = s[s > 0]
            med = np.median(s)
            x0 = (np.log(med) if med > 0 else np.log(pos[-1]) - 10.0) if tau0 is None else tau0
            lo, hi = np.log(pos[-1]) - 10.0, np.log(s[0]) + 10.0  # the library's bounds on log tau
            best = np.inf
            gamma, tau = gamma0[0], np.exp(x0)
            for g in gamma0:
                xt = line_search_min(lambda t: atn_cost64(s, si, x.shape, t, g, stdest, gs), x0, lo, hi)  # noqa: B023
                cost = atn_cost64(s, si, x.shape, xt, g, stdest, gs)
                if cost < best:
                    gamma, tau, best = g, np.exp(xt), cost
        return _adaptive_finish(x, u, s, vt, mean, gamma, tau, override)
    if method == "qut":
        if qlevel is None:
            rng = np.random if rng is None else rng
            maxd = np.ones(nbsim)
            for i in range(nbsim):
                maxd[i] = np.max(svd(rng.randn(*x.shape) * stdest, compute_uv=False, overwrite_a=True))
            tau = np.quantile(maxd, 1 - 1 / np.sqrt(np.log(max(*x.shape))))
        else:
            tau = stdest * qlevel
        if isinstance(gamma0, (float, np.floating)):
            gamma = gamma0
        else:
            res = minimize(lambda g: sure_atn_cost(x.shape, "qut", s, g, stdest, tau), 0)
            gamma = np.exp(res.x) + 1
    else:
        x0 = np.log(np.median(s)) if tau0 is None else tau0
        best = np.inf
        for g in gamma0:
            res = minimize(lambda t: sure_atn_cost(x.shape, method, s, g, stdest, t), x0)  # noqa: B023
            cost = sure_atn_cost(x.shape, method, s, g, stdest, res.x)
            if cost < best:
                gamma, tau, best = g, np.exp(res.x), cost
    return _adaptive_finish(x, u, s, vt, mean, gamma, tau, override)


def _adaptive_finish(x, u, s, vt, mean, gamma, tau, override):
    """Shrink, maxidx, synthesis (``space_time/lowrank.py:626-636``); margin =
    relative distance of the closest singular value to tau."""
    shrunk = atn_shrink(s, gamma, tau)
    with np.errstate(invalid="ignore", divide="ignore"):
        margin = float(np.min(np.abs(s / np.asarray(tau).reshape(-1)[0] - 1))) if len(s) else np.inf
    rank = np.max(np.nonzero(shrunk)) + 1 if np.any(shrunk) else 0
    if override is not None:
        rank = np.int64(override) if override else 0
        shrunk = shrunk.copy()
        shrunk[rank:] = 0
    new = np.zeros_like(x) + mean if rank == 0 else svd_synthesis(u, shrunk, vt, mean, rank)
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
    adaptive_method="sure",
    gamma0=None,
    tau0=None,
    nbsim=500,
    qut_level=None,
    adaptive_rng=None,
    optimizer="bfgs",
):
    """Whole-volume denoising: ``BaseSpaceTimeDenoiser.denoise`` + method setup.

    Follows ``space_time/base.py:177-270`` for the driver and
    ``space_time/lowrank.py`` for the method set-up (``HybridPCADenoiser.denoise``
    :76-102, ``RawSVDDenoiser.denoise`` :142-168, ``NordicDenoiser.denoise``
    :197-246, ``OptimalSVDDenoiser.denoise`` :318-377, ``AdaptiveDenoiser.denoise``
    :563-605 with ``adaptive_method``, ``gamma0``, ``tau0``, ``nbsim``; ``qut_level``
    replaces the per-patch QUT draws; ``optimizer`` as for ``_adaptive_patch``).

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
    elif method == "adaptive":
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
        elif method == "adaptive":
            new, rank, nvar, marg = _adaptive_patch(x, np.sqrt(np.mean(prior[sl])), adaptive_method, gamma0, tau0,
                                                    nbsim, qut_level, adaptive_rng, ov, optimizer)
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
