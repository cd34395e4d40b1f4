"""compute_torso_grid / load_torso_grid with the reference's signatures
(ecg/torso_grid.py:26-103, ecg/functions/build_torso_grid.py:495-758).

The grid dict carries the reference's keys (shape, dx_mm, origin_mm,
sigma_vol, active_mask, tissue_mask, active_ids, active_id_map,
surface_flat, surface_rows, surface_xyz, pin_row, use_sbm) plus the material
labels and their conductivities ("labels", "sigma_table") that the GPU
operator works from.  The stiffness matrix is never assembled (the solve is
matrix-free), so there is no A_scipy / solve_fn; the smoothed-boundary
method (use_sbm=True) is not implemented.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from . import torso as T


def voxel_ids_to_xyz(flat, shape, dx_mm, origin):
    i, j, k = np.unravel_index(np.asarray(flat, np.int64), shape)
    return np.stack([i, j, k], 1).astype(np.float64) * float(dx_mm) + np.asarray(origin, np.float64)


def torso_grid_from_labels(labels, sigma_map, dx_mm, origin_mm=(0.0, 0.0, 0.0), save_path=None,
                           verbose=False):
    """Grid dict from a label volume (0 = air) and label -> sigma [S/m]."""
    labels = np.asarray(labels)
    shape = labels.shape
    keys = sorted(int(k) for k in sigma_map)
    if 0 in keys:
        keys.remove(0)
    if len(keys) + 1 > 16:
        raise ValueError("at most 15 tissue labels are supported")
    lab = np.zeros(shape, np.uint8)
    table = [0.0]
    sigma_vol = np.zeros(shape, np.float64)
    for m, key in enumerate(keys, start=1):
        sel = labels == key
        lab[sel] = m
        table.append(float(sigma_map[key]))
        sigma_vol[sel] = float(sigma_map[key])
    unknown = (labels != 0) & (lab == 0)
    if unknown.any():
        raise ValueError(f"labels {np.unique(labels[unknown])} have no conductivity in sigma_map")
    tissue = labels != 0
    active_flat = np.where(tissue.ravel())[0].astype(np.int32)
    id_map = np.full(labels.size, -1, np.int32)
    id_map[active_flat] = np.arange(len(active_flat), dtype=np.int32)
    pin = T.pin_row(tissue, id_map)
    surf_flat, surf_rows = T.surface_ids(labels, tissue, id_map)
    origin = np.asarray(origin_mm, np.float64)
    grid = dict(shape=shape, dx_mm=float(dx_mm), origin_mm=origin, sigma_vol=sigma_vol,
                active_mask=tissue, tissue_mask=tissue, active_ids=active_flat,
                active_id_map=id_map, surface_flat=surf_flat, surface_rows=surf_rows,
                surface_xyz=voxel_ids_to_xyz(surf_flat, shape, dx_mm, origin), pin_row=pin,
                use_sbm=False, labels=lab, sigma_table=np.asarray(table))
    if save_path is not None:
        np.savez(str(save_path), shape=np.array(shape, np.int32), dx_mm=np.float64(dx_mm),
                 origin_mm=origin, sigma_vol=sigma_vol.astype(np.float32), active_mask=tissue,
                 tissue_mask=tissue, active_ids=active_flat, active_id_map=id_map,
                 surface_flat=surf_flat, surface_rows=surf_rows,
                 surface_xyz=grid["surface_xyz"].astype(np.float32), pin_row=np.int32(pin),
                 use_sbm=False, labels=lab, sigma_table=np.asarray(table))
    return grid


def compute_torso_grid(torso_nrrd_path=None, sigma_map=None, *, dx_coarse_mm=1.5, verbose=True,
                       save_path=None, use_sbm=False, labels=None, spacing_mm=None,
                       origin_mm=None, **_unused):
    """Label volume (from a torso NRRD, resampled to dx_coarse_mm by
    nearest neighbour as the reference does, or given directly as
    ``labels`` at dx_coarse_mm) -> grid dict."""
    if use_sbm:
        raise NotImplementedError("use_sbm=True (smoothed boundary method) is not implemented")
    if sigma_map is None:
        raise ValueError("sigma_map is required")
    if labels is None:
        try:
            import nrrd
        except ImportError as e:
            raise ImportError("reading a torso NRRD needs pynrrd; pass labels= instead") from e
        from scipy import ndimage as ndi
        data, hdr = nrrd.read(str(torso_nrrd_path))
        sp = np.abs(np.diag(np.asarray(hdr["space directions"], np.float64)))
        origin_mm = np.asarray(hdr.get("space origin", np.zeros(3)), np.float64)
        labels = ndi.zoom(data.astype(np.float32), sp / dx_coarse_mm, order=0).astype(np.int32)
    return torso_grid_from_labels(labels, sigma_map, dx_coarse_mm,
                                  origin_mm if origin_mm is not None else (0.0, 0.0, 0.0),
                                  save_path=save_path, verbose=verbose)


def load_torso_grid(out_path, torso_nrrd_path=None, sigma_map=None, dx_coarse_mm=None,
                    verbose=True):
    data = np.load(str(out_path))
    g = {k: data[k] for k in data.files}
    g["shape"] = tuple(np.asarray(g["shape"]).tolist())
    g["dx_mm"] = float(g["dx_mm"])
    g["pin_row"] = int(g["pin_row"])
    g["use_sbm"] = bool(g.get("use_sbm", False))
    return g
