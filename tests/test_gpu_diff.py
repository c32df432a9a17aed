"""Gradients of the differentiable low-rank denoiser (``lowrank_denoise``).

The CUDA backward (``pd_lowrank_backward``) is checked three ways:
* against torch.linalg.svd autograd on an FP64 torch restatement of the same
  map (patch gather, centring, SVD, shrinkage, recombination, normalisation);
* against central finite differences (step 1e-3) of the FP64 oracle's forward
  along 64 seeded random directions, and in threshold_scale;
* a 20-step Monte-Carlo SURE tuning loop must lower the SURE estimate and the
  true error against the clean signal.
"""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

import oracle
from patch_denoising_b200 import _engine
from patch_denoising_b200.space_time import lowrank_denoise, sure_tune_threshold
from patch_denoising_b200.synthetic import lowrank_volume, radial_noise_map

pytestmark = pytest.mark.gpu

SHAPE = (10, 9, 8, 20)
PATCH, OVERLAP = 4, 2  # M = 64 > T = 20, 36 patches
DEV = torch.device("cuda", 0)


def _volume(seed=3):
    nmap = radial_noise_map(SHAPE[:-1], base=2.0, extra=1.0)
    x, clean = lowrank_volume(SHAPE, 3, amplitude=20.0, noise=1.0, noise_map=nmap, seed=seed)
    return x, clean, nmap


def _patch_index(shape, patch, overlap):
    """Flat indices (patches, M, T) of every patch's Casorati matrix (rows in C
    order over the spatial patch), as the library's geometry."""
    g = _engine.geometry(shape, (patch,) * 3 + (shape[-1],), (overlap,) * 3 + (shape[-1],))
    X, Y, Z, T = shape
    idx = []
    for gi in range(int(g.grid[0])):
        for gj in range(int(g.grid[1])):
            for gk in range(int(g.grid[2])):
                o = (gi * int(g.step[0]), gj * int(g.step[1]), gk * int(g.step[2]))
                rows = []
                for i in range(patch):
                    for j in range(patch):
                        for k in range(patch):
                            v = ((o[0] + i) * Y + (o[1] + j)) * Z + (o[2] + k)
                            rows.append(v * T + np.arange(T))
                idx.append(np.stack(rows))
    return torch.from_numpy(np.stack(idx)).to(DEV)


def _torch_reference(x, scale, nmap, shrink, recombination, ranks=None):
    """The map in FP64 torch with torch.linalg.svd (autograd through the SVD)."""
    X, Y, Z, T = x.shape
    I = _patch_index(tuple(x.shape), PATCH, OVERLAP)
    P = x.reshape(-1)[I]  # (np, M, T)
    mu = P.mean(1, keepdim=True)
    U, S, Vh = torch.linalg.svd(P - mu, full_matrices=False)
    M = P.shape[1]
    if shrink == "soft":
        vox = I[:, :, 0] // T
        stdest = torch.sqrt((nmap.reshape(-1)[vox] ** 2).mean(1))
        tau = scale * stdest * (math.sqrt(M) + math.sqrt(T))
        St = torch.relu(S - tau[:, None])
        rank = (St > 0).sum(1).detach()
    else:
        keep = torch.arange(S.shape[1], device=DEV)[None, :] < ranks[:, None]
        St = S * keep
        rank = ranks
    Yp = U @ torch.diag_embed(St) @ Vh + mu
    theta = torch.ones_like(rank, dtype=x.dtype) if recombination == "average" else 1.0 / (2.0 + rank.to(x.dtype))
    th = theta[:, None, None].expand_as(Yp)
    acc = torch.zeros(x.numel(), dtype=x.dtype, device=DEV).index_add(0, I.reshape(-1), (th * Yp).reshape(-1))
    W = torch.zeros(x.numel(), dtype=x.dtype, device=DEV).index_add(0, I.reshape(-1), th.reshape(-1))
    return (acc / W).reshape(x.shape)


def _mp_ranks(x, scale):
    res = _engine.run("mp-pca", torch.from_numpy(x).to(DEV), (PATCH,) * 3 + (SHAPE[-1],),
                      (OVERLAP,) * 3 + (SHAPE[-1],), "weighted", None, 50, threshold_scale=scale)
    return res.patch_rank.long()


@pytest.mark.parametrize("shrink,recombination", [("soft", "average"), ("soft", "weighted"), ("hard", "weighted"),
                                                  ("hard", "average")])
def test_gradients_match_torch_svd_autograd(shrink, recombination):
    x, _, nmap = _volume()
    scale = 0.6
    w = torch.from_numpy(np.random.default_rng(1).standard_normal(SHAPE)).to(DEV)
    # ours (FP32 kernels)
    xt = torch.from_numpy(x).to(DEV).requires_grad_(True)
    st = torch.tensor(scale, device=DEV, requires_grad=True)
    out = lowrank_denoise(xt, PATCH, OVERLAP, st, nmap, shrink=shrink, recombination=recombination)
    fin = torch.isfinite(out)
    loss = (torch.where(fin, out, torch.zeros_like(out)).double() * w).sum()
    loss.backward()
    # FP64 torch reference
    x64 = torch.from_numpy(x.astype(np.float64)).to(DEV).requires_grad_(True)
    s64 = torch.tensor(scale, dtype=torch.float64, device=DEV, requires_grad=True)
    ranks = _mp_ranks(x, scale) if shrink == "hard" else None
    ref = _torch_reference(x64, s64, torch.from_numpy(nmap).to(DEV), shrink, recombination, ranks)
    np.testing.assert_array_equal(torch.isfinite(ref).cpu().numpy(), fin.cpu().numpy())
    rl = (torch.where(torch.isfinite(ref), ref, torch.zeros_like(ref)) * w).sum()
    rl.backward()
    assert abs(float(loss.detach()) - float(rl.detach())) <= 1e-5 * abs(float(rl.detach()))
    gx, rx = xt.grad.double(), x64.grad
    err = float(torch.linalg.vector_norm(gx - rx) / torch.linalg.vector_norm(rx))
    print(f"{shrink} {recombination}: input-gradient rel-L2 {err:.2e}")
    assert err <= 1e-4
    if shrink == "soft":
        assert abs(float(st.grad) - float(s64.grad)) <= 1e-4 * abs(float(s64.grad))
    else:
        assert float(st.grad) == 0.0


def _oracle_loss(x64, scale, nmap, w, recombination):
    p_s = (PATCH,) * 3 + (SHAPE[-1],)
    M, T = PATCH**3, SHAPE[-1]
    level = scale * (math.sqrt(M) + math.sqrt(T))
    r = oracle.denoise("adaptive", x64, PATCH, OVERLAP, recombination=recombination, adaptive_method="qut",
                       noise_std=nmap, gamma0=1.0, qut_level=level, nbsim=1)
    out = r["out"]
    assert tuple(p_s[:-1]) == (PATCH,) * 3
    fin = np.isfinite(out)
    return float((np.where(fin, out, 0.0) * w).sum())


@pytest.mark.parametrize("recombination", ["average", "weighted"])
def test_gradients_match_finite_differences(recombination):
    """64 seeded directions d (unit RMS per voxel-frame), central differences
    with step 1e-3 of the FP64 oracle's loss; agreement to 1e-3 of the typical
    directional derivative. threshold_scale: central difference at 1e-6."""
    x, _, nmap = _volume(seed=5)
    scale = 0.7
    rng = np.random.default_rng(2)
    w = rng.standard_normal(SHAPE)
    xt = torch.from_numpy(x).to(DEV).requires_grad_(True)
    st = torch.tensor(scale, device=DEV, requires_grad=True)
    out = lowrank_denoise(xt, PATCH, OVERLAP, st, nmap, shrink="soft", recombination=recombination)
    fin = torch.isfinite(out)
    (torch.where(fin, out, torch.zeros_like(out)).double() * torch.from_numpy(w).to(DEV)).sum().backward()
    g = xt.grad.double().cpu().numpy()
    x64 = x.astype(np.float64)
    h = 1e-3
    fd, ad = [], []
    for _ in range(64):
        d = rng.standard_normal(SHAPE)
        lp = _oracle_loss(x64 + h * d, scale, nmap, w, recombination)
        lm = _oracle_loss(x64 - h * d, scale, nmap, w, recombination)
        fd.append((lp - lm) / (2 * h))
        ad.append(float((g * d).sum()))
    fd, ad = np.array(fd), np.array(ad)
    typ = float(np.sqrt(np.mean(fd**2)))
    worst = float(np.max(np.abs(fd - ad)) / typ)
    print(f"{recombination}: worst |FD - backward| / rms(FD) over 64 directions: {worst:.2e}")
    assert worst <= 1e-3
    # threshold_scale: a 1e-3 step moves tau across some singular values of the
    # 36 patches, where the soft threshold has a kink (and, weighted, theta
    # jumps); a 1e-6 relative step stays inside one smooth piece in FP64
    hs = 1e-6 * scale
    fds = (_oracle_loss(x64, scale + hs, nmap, w, recombination)
           - _oracle_loss(x64, scale - hs, nmap, w, recombination)) / (2 * hs)
    assert abs(float(st.grad) - fds) <= 1e-3 * abs(fds)


def test_sure_tuning_lowers_the_risk():
    """20 Monte-Carlo SURE steps from an over-smoothing threshold lower the SURE
    estimate, and the true error against the clean signal falls with it."""
    x, clean = lowrank_volume((16, 16, 12, 40), 4, amplitude=20.0, noise=2.0, seed=9)
    y = torch.from_numpy(x).to(DEV)
    scale, hist = sure_tune_threshold(y, 2.0, 5, 3, init_scale=2.5, steps=20, lr=0.1)
    assert hist[-1][1] < hist[0][1]

    def mse(s):
        with torch.no_grad():
            out = lowrank_denoise(y, 5, 3, s, 2.0)
        fin = torch.isfinite(out)
        c = torch.from_numpy(clean).to(DEV)
        return float(((out - c)[fin] ** 2).mean())

    print(f"SURE tuning: scale 2.5 -> {scale:.3f}, SURE {hist[0][1]:.4g} -> {hist[-1][1]:.4g}, "
          f"MSE {mse(2.5):.4g} -> {mse(scale):.4g}")
    assert mse(scale) < mse(2.5)
