"""ORACLE -- test infrastructure, not product code.

FP64 CPU restatement of HrdayaPy's torso forward solve, used only by tests/,
``__graft_entry__.smoke()`` (as the checker) and bench.py's CPU-baseline leg.

* :func:`assemble_stiffness` -- ecg/functions/build_torso_grid.py:276-397
  (harmonic-mean face conductance / h^2, air skipped; with psi_vol the
  smoothed-boundary path, the face conductance times the harmonic mean of
  psi)
* :func:`surface_ids`        -- build_torso_grid.py:469-488
* :func:`pin_row`            -- build_torso_grid.py:616-623
* :func:`heart_laplacian`    -- ecg/functions/compute_bspm.py:88-119
* :func:`projection_map`     -- compute_bspm.py:126-157
* :func:`frame_rhs`          -- solve_frame's source construction,
  compute_bspm.py:381-419 (in FP64)
* :func:`solve`              -- the pinned system A x = b (compute_bspm.py:327-336)
  solved to machine precision (sparse LU), the reference the GPU PCG is
  judged against
* :func:`pcg_reference`      -- _pcg_gpu (compute_bspm.py:164-263) in FP64
  numpy, with its rms / p99 / linf stopping statistics
* :func:`pinned_csr`, :func:`pcg_fp64` -- the pinned system in CSR form
  without a LIL round trip, and _pcg_gpu's Jacobi-CG run in FP64 in C
  (torso_oracle.c, pthreads) to a relative true residual: the FP64
  solution the GPU's potentials are judged against at full torso size, and
  the reference method timed on the host cores

Pinned by tests/test_oracle_golden.py against tests/golden/torso.npz.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
from scipy import ndimage as ndi
from scipy.sparse.linalg import splu


def assemble_stiffness(sigma_vol, h_m, active_mask, psi_vol=None):
    """psi_vol: the smoothed-boundary domain function, or None (sharp).
    With psi every face conductance is (psi_face * sigma_face) / h^2, psi_face
    the harmonic mean of the two cells' psi (build_torso_grid.py:340-378)."""
    ni, nj, nk = sigma_vol.shape
    flat = np.where(active_mask.ravel())[0]
    N = len(flat)
    id_map = np.full(sigma_vol.size, -1, np.int64)
    id_map[flat] = np.arange(N)
    sig = sigma_vol.ravel().astype(np.float64)
    psi = None if psi_vol is None else np.asarray(psi_vol, np.float64).ravel()
    i, j, k = np.unravel_index(flat, sigma_vol.shape)
    rows, cols, vals = [], [], []
    diag = np.zeros(N)
    for di, dj, dk in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
        a, b, c = i + di, j + dj, k + dk
        inb = (a >= 0) & (a < ni) & (b >= 0) & (b < nj) & (c >= 0) & (c < nk)
        r = np.where(inb)[0]
        fn = (a[r] * nj + b[r]) * nk + c[r]
        sk, sn = sig[flat[r]], sig[fn]
        ok = sk + sn >= 1e-30
        if psi_vol is not None:
            pk_, pn_ = psi[flat[r]], psi[fn]
            ok &= ~((pk_ <= 0.0) & (pn_ <= 0.0))
        r, fn, sk, sn = r[ok], fn[ok], sk[ok], sn[ok]
        if psi_vol is None:
            g = (2.0 * sk * sn) / (sk + sn) / (h_m ** 2)
        else:
            pk_, pn_ = psi[flat[r]], psi[fn]
            ps = pk_ + pn_
            pf = np.where(ps < 1e-30, 0.0, (2.0 * pk_ * pn_) / np.where(ps < 1e-30, 1.0, ps))
            g = pf * ((2.0 * sk * sn) / (sk + sn)) / (h_m ** 2)
        np.add.at(diag, r, g)
        act = active_mask.ravel()[fn]
        rows.append(r[act]); cols.append(id_map[fn[act]]); vals.append(-g[act])
    rows.append(np.arange(N)); cols.append(np.arange(N)); vals.append(diag)
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(N, N))
    return A, flat, id_map


def surface_ids(label_vol, active_mask, id_map):
    is_air = label_vol == 0
    dil = ndi.binary_dilation(is_air, structure=ndi.generate_binary_structure(3, 1))
    surf_flat = np.where((active_mask & dil).ravel())[0]
    return surf_flat, id_map[surf_flat]


def pin_row(tissue_mask, id_map):
    interior = np.where(tissue_mask.ravel())[0]
    return int(id_map[int(interior[len(interior) // 2])])


def heart_laplacian(vox_idx, n_nodes):
    ijk = vox_idx.astype(np.int64)
    off = ijk - ijk.min(axis=0)
    shape = tuple((off.max(axis=0) + 2).tolist())
    lookup = np.full(shape, -1, np.int64)
    lookup[off[:, 0], off[:, 1], off[:, 2]] = np.arange(n_nodes)
    rows, cols = [], []
    for d in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
        n_ = off + np.array(d)
        inb = np.all((n_ >= 0) & (n_ < np.array(shape)), axis=1)
        kk = np.where(inb)[0]
        nn = lookup[n_[inb, 0], n_[inb, 1], n_[inb, 2]]
        ok = nn >= 0
        rows.append(kk[ok]); cols.append(nn[ok])
    r = np.concatenate(rows); c = np.concatenate(cols)
    Koff = sp.csr_matrix((np.ones(len(r)), (r, c)), shape=(n_nodes, n_nodes))
    deg = np.asarray(Koff.sum(axis=1)).ravel()
    return Koff - sp.diags(deg, format="csr")


def projection_map(coords_mm, R, t, scale, origin, dx, active_id_map, shape):
    torso = (R @ (coords_mm * scale).T).T + t
    ijk = np.floor((torso - origin) / dx).astype(np.int64)
    ni, nj, nk = shape
    inb = ((ijk[:, 0] >= 0) & (ijk[:, 0] < ni) & (ijk[:, 1] >= 0) & (ijk[:, 1] < nj) &
           (ijk[:, 2] >= 0) & (ijk[:, 2] < nk))
    proj = np.full(len(coords_mm), -1, np.int64)
    flat = (ijk[inb, 0] * nj + ijk[inb, 1]) * nk + ijk[inb, 2]
    cand = active_id_map[flat]
    proj[np.where(inb)[0][cand >= 0]] = cand[cand >= 0]
    return proj, proj >= 0


def frame_rhs(K, Vm_mV, proj, valid, n_rows, pin, sigma_i, h_fine_m, dx_mm, psi_row=None):
    """FP64 restatement of solve_frame's b (compute_bspm.py:381-419); with a
    smoothed boundary b is weighted by psi per row (:413-414)."""
    V = np.asarray(Vm_mV, np.float64) * 1e-3
    Iv = (K @ V)[valid] * (sigma_i / h_fine_m ** 2)
    src = Iv - Iv.mean()
    b = np.zeros(n_rows)
    np.add.at(b, proj[valid], src)
    b /= (dx_mm / (h_fine_m * 1e3)) ** 3
    if psi_row is not None:
        b *= np.asarray(psi_row, np.float64)
    b[pin] = 0.0
    return b


def pinned(A, pin):
    A = A.tolil()
    A[pin, :] = 0.0
    A[:, pin] = 0.0
    A[pin, pin] = 1.0
    return A.tocsc()


class Solver:
    """Direct FP64 solve of the pinned system (factorised once)."""

    def __init__(self, A, pin):
        self.pin = pin
        self.Ap = pinned(A, pin)
        self.lu = splu(self.Ap)

    def solve(self, b):
        b = np.array(b, np.float64)
        b[self.pin] = 0.0
        return self.lu.solve(b)


def pcg_reference(A_pinned, b, x0=None, tol_mV=0.01, max_iter=500, metric="rms"):
    """_pcg_gpu restated in FP64 numpy: returns (x, n_iter, stat_mV)."""
    Minv = 1.0 / np.where(np.abs(A_pinned.diagonal()) > 1e-30, A_pinned.diagonal(), 1.0)
    N = len(b)
    tol_v = tol_mV * 1e-3

    def stat(z):
        if metric == "rms":
            return np.linalg.norm(z) / np.sqrt(N)
        if metric == "p99":    # torch.quantile(|z|, 0.99), linear interpolation
            return np.quantile(np.abs(z), 0.99)
        return np.abs(z).max()

    x = np.zeros(N) if x0 is None else np.array(x0, np.float64)
    r = b - A_pinned @ x if x0 is not None else np.array(b, np.float64)
    z = Minv * r
    p = z.copy()
    rz = r @ z
    for i in range(max_iter):
        Ap = A_pinned @ p
        pAp = p @ Ap
        if abs(pAp) < 1e-30:
            break
        a = rz / pAp
        x = x + a * p
        r = r - a * Ap
        z = Minv * r
        e = stat(z)
        if e < tol_v:
            return x, i + 1, e * 1e3
        rz_new = r @ z
        p = z + (rz_new / rz) * p
        rz = rz_new
    return x, max_iter, stat(Minv * r) * 1e3


def pinned_csr(A, pin):
    """The pinned system of make_gpu_solver (compute_bspm.py:327-336): row
    and column ``pin`` zeroed, 1 on its diagonal; CSR, without a LIL round
    trip (fast at millions of rows)."""
    A = sp.csr_matrix(A)
    n = A.shape[0]
    keep = np.ones(n)
    keep[pin] = 0.0
    D = sp.diags(keep, format="csr")
    Ap = (D @ A @ D).tocsr()
    Ap = Ap + sp.csr_matrix(([1.0], ([pin], [pin])), shape=(n, n))
    Ap.sort_indices()
    return Ap.tocsr()


def pcg_fp64(A_pinned, b, x0=None, tol=1e-10, max_iter=20000):
    """Jacobi-PCG in FP64 (orc_csr_pcg) from x0 to ||b - A x|| <= tol ||b||
    (true residual).  Returns (x, iterations, true relative residual,
    restarts)."""
    import ctypes
    from .mono import lib
    L = lib()
    if not hasattr(L, "_pcg_typed"):
        P = ctypes.c_void_p
        L.orc_csr_pcg.argtypes = [ctypes.c_int64, P, P, P, P, P, P, ctypes.c_double,
                                  ctypes.c_int64, P]
        L.orc_csr_pcg.restype = ctypes.c_int
        L._pcg_typed = True
    A = sp.csr_matrix(A_pinned)
    ptr = np.ascontiguousarray(A.indptr, np.int64)
    idx = np.ascontiguousarray(A.indices, np.int32)
    val = np.ascontiguousarray(A.data, np.float64)
    d = A.diagonal()
    minv = np.where(np.abs(d) > 1e-30, 1.0 / np.where(d == 0, 1.0, d), 0.0)
    bb = np.ascontiguousarray(b, np.float64)
    x = np.zeros(A.shape[0]) if x0 is None else np.array(x0, np.float64)
    out = np.zeros(3)
    c = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    rc = L.orc_csr_pcg(A.shape[0], c(ptr), c(idx), c(val), c(minv), c(bb), c(x), float(tol),
                       int(max_iter), c(out))
    if rc != 0:
        raise MemoryError("orc_csr_pcg: out of host memory")
    return x, int(out[0]), float(out[1]), int(out[2])
