"""Torso forward solve on the GPU (libhrdaya_b200 hp_torso_*), plus the
host-side geometry it needs: heart neighbour table, projection of heart
voxels onto torso rows (compute_bspm.py:88-157), surface rows, pinned row
(build_torso_grid.py:469-488, :616-623), electrode read-out and leads.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .. import _lib

RULES = {"rel": 0, "rms": 1, "linf": 2, "p99": 3}


def heart_neighbours(vox_idx: np.ndarray) -> np.ndarray:
    """(N, 6) face-neighbour node ids (-1 = none) of the heart voxels; the
    graph Laplacian K of build_heart_laplacian (compute_bspm.py:88-119) is
    K V = sum_n (V_n - V_i) over these neighbours."""
    ijk = np.asarray(vox_idx, np.int64)
    off = ijk - ijk.min(axis=0)
    shape = tuple((off.max(axis=0) + 3).tolist())
    lookup = np.full(shape, -1, np.int64)
    lookup[off[:, 0] + 1, off[:, 1] + 1, off[:, 2] + 1] = np.arange(len(ijk))
    nbr = np.empty((len(ijk), 6), np.int32)
    for q, d in enumerate(((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1))):
        n_ = off + 1 + np.array(d)
        nbr[:, q] = lookup[n_[:, 0], n_[:, 1], n_[:, 2]]
    return nbr


def projection_map(coords_mm, R, t, scale, origin, dx, active_id_map, shape):
    """Heart node -> torso row via R (s x) + t and floor((. - origin) / dx)
    (compute_bspm.py:126-157); -1 where the node misses the active torso."""
    torso = (np.asarray(R, np.float64) @ (np.asarray(coords_mm, np.float64) * float(scale)).T).T \
        + np.asarray(t, np.float64)
    ijk = np.floor((torso - np.asarray(origin, np.float64)) / float(dx)).astype(np.int64)
    ni, nj, nk = shape
    inb = ((ijk[:, 0] >= 0) & (ijk[:, 0] < ni) & (ijk[:, 1] >= 0) & (ijk[:, 1] < nj) &
           (ijk[:, 2] >= 0) & (ijk[:, 2] < nk))
    proj = np.full(len(torso), -1, np.int64)
    flat = (ijk[inb, 0] * nj + ijk[inb, 1]) * nk + ijk[inb, 2]
    cand = np.asarray(active_id_map)[flat]
    idx = np.where(inb)[0]
    proj[idx[cand >= 0]] = cand[cand >= 0]
    return proj.astype(np.int32), proj >= 0


def surface_ids(labels, active_mask, id_map):
    """Tissue voxels with an air face neighbour (build_torso_grid.py:469-488)."""
    from scipy import ndimage as ndi
    air = np.asarray(labels) == 0
    dil = ndi.binary_dilation(air, structure=ndi.generate_binary_structure(3, 1))
    flat = np.where((np.asarray(active_mask) & dil).ravel())[0].astype(np.int32)
    return flat, np.asarray(id_map)[flat]


def pin_row(tissue_mask, id_map) -> int:
    interior = np.where(np.asarray(tissue_mask).ravel())[0]
    return int(np.asarray(id_map)[int(interior[len(interior) // 2])])


def labels_from_grid(grid):
    """Material labels (uint8) and their conductivities from a grid dict:
    either our own ("labels", "sigma_table") or the reference's
    ("sigma_vol" + "active_mask"), whose distinct conductivities become
    materials."""
    if "labels" in grid and "sigma_table" in grid:
        return np.asarray(grid["labels"], np.uint8), np.asarray(grid["sigma_table"], np.float64)
    sig = np.asarray(grid["sigma_vol"], np.float64)
    act = np.asarray(grid["active_mask"], bool)
    vals = np.unique(sig[act])
    if len(vals) + 1 > 16:
        raise ValueError(f"{len(vals)} distinct conductivities; at most 15 are supported")
    lab = np.zeros(sig.shape, np.uint8)
    lab[act] = (np.searchsorted(vals, sig[act]) + 1).astype(np.uint8)
    return lab, np.concatenate([[0.0], vals])


def psi_from_grid(grid):
    """The smoothed-boundary domain function of a grid built with
    use_sbm=True (float32, grid shape), else None."""
    if bool(grid.get("use_sbm", False)) and "psi_vol" in grid:
        return np.ascontiguousarray(grid["psi_vol"], np.float32)
    return None


class TorsoSolver:
    """Owns one hp_torso handle.  psi: the smoothed-boundary domain function
    (labels' shape, > 0 exactly on the labelled cells) or None."""

    def __init__(self, labels, sigma_table, dx_mm, pin, heart_nbr, proj, sigma_i, h_fine_mm,
                 read_rows, stream=None, psi=None):
        torch = _lib.require_cuda()
        L = _lib.lib()
        labels = np.ascontiguousarray(labels, np.uint8)
        sig = np.ascontiguousarray(sigma_table, np.float64)
        nbr = np.ascontiguousarray(heart_nbr, np.int32)
        proj = np.ascontiguousarray(proj, np.int32)
        read = np.ascontiguousarray(read_rows, np.int64)
        d = _lib.HpTorsoDesc()
        d.ni, d.nj, d.nk = labels.shape
        d.h_m = float(dx_mm) * 1e-3
        d.label = _lib.ptr(labels)
        d.n_materials = len(sig)
        d.sigma = _lib.ptr(sig)
        d.pin_row = int(pin)
        d.n_heart = len(proj)
        d.heart_nbr = _lib.ptr(nbr)
        d.proj = _lib.ptr(proj)
        h_fine_m = float(h_fine_mm) * 1e-3
        d.coeff = float(sigma_i) / h_fine_m ** 2
        d.n_expected = float((float(dx_mm) / float(h_fine_mm)) ** 3)
        d.n_read = len(read)
        d.read_rows = _lib.ptr(read)
        if psi is not None:
            psi = np.ascontiguousarray(psi, np.float32)
            if psi.shape != labels.shape:
                raise ValueError(f"psi {psi.shape} and labels {labels.shape} differ in shape")
            d.psi = _lib.ptr(psi)
        if stream is None:
            self._torch_stream = torch.cuda.Stream()
            stream = C.c_void_p(self._torch_stream.cuda_stream)
        self.stream = stream
        h = C.c_void_p()
        _lib.check(L.hp_torso_create(C.byref(d), C.byref(h), self.stream), "hp_torso_create")
        self.h = h
        self.sigma_table = sig
        self.h_m = d.h_m
        self.n_read = len(read)
        self.n_heart = len(proj)
        self.n_rows = int(L.hp_torso_rows(h))

    def solve_frame(self, vm, tol=1e-6, rule="rel", max_iter=2000, out=None):
        """vm: (n_heart,) mV, numpy (host) or a CUDA tensor (device).
        Returns (read-out potentials in mV, HpSolveStats)."""
        if rule not in RULES:
            raise ValueError(f"rule must be one of {sorted(RULES)}, got {rule!r}")
        L = _lib.lib()
        st = _lib.HpSolveStats()
        on_dev = 0
        if hasattr(vm, "data_ptr"):
            assert vm.is_cuda and vm.dtype.itemsize == 4 and vm.is_contiguous()
            vptr, on_dev = C.c_void_p(vm.data_ptr()), 1
        else:
            vm = np.ascontiguousarray(vm, np.float32)
            if vm.shape != (self.n_heart,):
                raise ValueError(f"Vm frame has shape {vm.shape}, expected ({self.n_heart},)")
            vptr = _lib.ptr(vm)
        out_dev = 0
        if out is None:
            out = np.empty(self.n_read, np.float32)
        if hasattr(out, "data_ptr"):
            optr, out_dev = C.c_void_p(out.data_ptr()), 1
        else:
            optr = _lib.ptr(out)
        _lib.check(L.hp_torso_solve_frame(self.h, vptr, on_dev, optr, out_dev, float(tol),
                                          RULES[rule], int(max_iter), C.byref(st), self.stream),
                   "hp_torso_solve_frame")
        return out, st

    def solution(self):
        x = np.empty(self.n_rows, np.float64)
        _lib.check(_lib.lib().hp_torso_copy_solution(self.h, _lib.ptr(x), self.stream),
                   "hp_torso_copy_solution")
        return x

    def rhs(self):
        b = np.empty(self.n_rows, np.float32)
        _lib.check(_lib.lib().hp_torso_copy_rhs(self.h, _lib.ptr(b), self.stream),
                   "hp_torso_copy_rhs")
        return b

    def reset(self):
        _lib.check(_lib.lib().hp_torso_reset(self.h), "hp_torso_reset")

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().hp_torso_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------------
# electrodes and leads
# --------------------------------------------------------------------------

LEADS = ["I", "II", "III", "aVR", "aVL", "aVF", "V1", "V2", "V3", "V4", "V5", "V6"]
ELECTRODES = ["RA", "LA", "RL", "LL", "V1", "V2", "V3", "V4", "V5", "V6"]


def twelve_lead(phi_e):
    """Standard 12 leads from the 10 electrode potentials (rows in ELECTRODES
    order; any trailing axis is time).  Wilson central terminal
    WCT = (RA + LA + LL) / 3."""
    e = {n: np.asarray(phi_e[i]) for i, n in enumerate(ELECTRODES)}
    wct = (e["RA"] + e["LA"] + e["LL"]) / 3.0
    out = [e["LA"] - e["RA"], e["LL"] - e["RA"], e["LL"] - e["LA"],
           e["RA"] - 0.5 * (e["LA"] + e["LL"]), e["LA"] - 0.5 * (e["RA"] + e["LL"]),
           e["LL"] - 0.5 * (e["RA"] + e["LA"])]
    out += [e[f"V{k}"] - wct for k in range(1, 7)]
    return np.stack(out)


def nearest_surface_rows(points_mm, surface_xyz, surface_rows):
    from scipy.spatial import cKDTree
    _, k = cKDTree(np.asarray(surface_xyz, np.float64)).query(np.asarray(points_mm, np.float64))
    return np.asarray(surface_rows)[k]
