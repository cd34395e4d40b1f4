"""Transmural coordinate with the reference's signature and formulation
(coordinates/functions/generate_transmural_coordinate.py:83-286 of the
HrdayaPy project): the Laplace equation on the myocardial voxels of S,
phi = 1 on voxels labelled +1 (epicardium), phi = 0 on voxels labelled -1
(endocardium), zero-flux faces elsewhere (a face to a voxel outside S
contributes nothing, so it does not inflate the diagonal), solved by CG
from the distance-ratio guess d_endo / (d_endo + d_epi).

This is set-up, run once per geometry on the device: the graph Laplacian
is applied matrix-free from a six-neighbour table, and the Dirichlet
voxels are eliminated (their values enter the right-hand side), which
leaves a symmetric positive-definite system for Jacobi-preconditioned CG
with FP64 dot products, stopped on the relative residual like the
reference (tol relative to the initial residual).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np


def generate_transmural_coordinate(S, surface_label, device="cuda", tol=1e-6, maxiter=10_000,
                                   save_path=None):
    """phi (Nx, Ny, Nz) float32 in [0, 1], NaN outside S."""
    import torch
    from scipy.ndimage import distance_transform_edt
    if save_path is not None:
        save_path = Path(save_path).with_suffix(".npy")
        if save_path.exists():
            return np.load(save_path)
    S = np.asarray(S)
    surface_label = np.asarray(surface_label)
    if S.shape != surface_label.shape:
        raise ValueError(f"S {S.shape} and surface_label {surface_label.shape} differ in shape")
    dev = torch.device(device) if isinstance(device, str) else device
    if dev.type == "cuda" and not torch.cuda.is_available():
        raise RuntimeError("generate_transmural_coordinate: no CUDA device")
    shape = S.shape
    vox = np.argwhere(S == 1)
    N = len(vox)
    idx = -np.ones(shape, np.int64)
    idx[vox[:, 0], vox[:, 1], vox[:, 2]] = np.arange(N)
    lab = surface_label[vox[:, 0], vox[:, 1], vox[:, 2]]
    is_dir = lab != 0
    # EDT warm start, as the reference (generate_transmural_coordinate.py:250-262)
    d_endo = distance_transform_edt(surface_label != -1)
    d_epi = distance_transform_edt(surface_label != 1)
    den = d_endo + d_epi
    guess = np.where(den > 0, d_endo / np.where(den > 0, den, 1.0), 0.5).astype(np.float32)
    guess[surface_label == -1] = 0.0
    guess[surface_label == 1] = 1.0
    nb = np.full((N, 6), -1, np.int64)
    for q, d in enumerate(((-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1))):
        n_ = vox + np.array(d)
        inb = np.all((n_ >= 0) & (n_ < np.array(shape)), 1)
        nc = np.clip(n_, 0, np.array(shape) - 1)
        nb[:, q] = np.where(inb, idx[nc[:, 0], nc[:, 1], nc[:, 2]], -1)
    dirv = np.where(lab == 1, 1.0, 0.0).astype(np.float32)       # Dirichlet values
    nb_t = torch.as_tensor(nb, device=dev)
    has = nb_t >= 0
    nbc = nb_t.clamp(min=0)
    free = torch.as_tensor(~is_dir, device=dev)
    dir_t = torch.as_tensor(dirv, device=dev)
    deg = has.sum(1).to(torch.float32)
    # unknowns: the free voxels; a Dirichlet neighbour moves to the RHS
    nb_free = has & free[nbc]
    rhs = torch.where(free, ((dir_t[nbc] * (has & ~free[nbc])).sum(1)), torch.zeros_like(deg))

    def A(x):                     # x is zero on Dirichlet voxels
        return torch.where(free, deg * x - (x[nbc] * nb_free).sum(1), torch.zeros_like(x))

    x = torch.as_tensor(guess[vox[:, 0], vox[:, 1], vox[:, 2]], device=dev)
    x = torch.where(free, x, torch.zeros_like(x))
    minv = torch.where(free & (deg > 0), 1.0 / deg.clamp(min=1.0), torch.zeros_like(deg))
    r = rhs - A(x)
    r0 = float(torch.linalg.vector_norm(r.double()))
    z = minv * r
    p = z.clone()
    rz = torch.dot(r.double(), z.double())
    for _ in range(int(maxiter)):
        if r0 == 0.0 or float(torch.linalg.vector_norm(r.double())) < tol * r0:
            break
        Ap = A(p)
        pap = torch.dot(p.double(), Ap.double())
        if float(pap) <= 0.0:
            break
        alpha = rz / pap
        x = x + alpha.float() * p
        r = r - alpha.float() * Ap
        z = minv * r
        rz_new = torch.dot(r.double(), z.double())
        p = z + (rz_new / rz).float() * p
        rz = rz_new
    phi_flat = torch.where(free, x, dir_t).cpu().numpy()
    phi = np.full(shape, np.nan, np.float32)
    phi[vox[:, 0], vox[:, 1], vox[:, 2]] = phi_flat
    np.clip(phi, 0.0, 1.0, out=phi)
    if save_path is not None:
        save_path.parent.mkdir(parents=True, exist_ok=True)
        np.save(save_path, phi)
    return phi
