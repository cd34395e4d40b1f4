"""compute_torso_grid / load_torso_grid with the reference's signatures
(ecg/torso_grid.py:26-103, ecg/functions/build_torso_grid.py:495-758).

The grid dict carries the reference's keys (shape, dx_mm, origin_mm,
sigma_vol, active_mask, tissue_mask, active_ids, active_id_map,
surface_flat, surface_rows, surface_xyz, pin_row, use_sbm, and psi_vol with
the smoothed boundary) plus the material labels and their conductivities
("labels", "sigma_table") that the GPU operator works from.  The stiffness
matrix is never assembled (the solve is matrix-free), so there is no
A_scipy / solve_fn.

Smoothed boundary method (use_sbm=True, build_torso_grid.py:130-206,
:564-585): a domain function psi is built from the FINE segmentation, the
system spans the cells with psi > 0 (a band beyond the tissue included),
the band takes the material of its nearest tissue voxel, and the GPU
operator weights every face by the harmonic mean of psi (hp_torso_create's
psi).  Surface nodes and the pinned node stay on the true tissue.
"""
from __future__ import annotations

import numpy as np

from . import torso as T


def voxel_ids_to_xyz(flat, shape, dx_mm, origin):
    i, j, k = np.unravel_index(np.asarray(flat, np.int64), shape)
    return np.stack([i, j, k], 1).astype(np.float64) * float(dx_mm) + np.asarray(origin, np.float64)


def smoothed_domain(volume_fine, spacing_fine, dx_coarse_mm, coarse_shape,
                    interface_width_mm=3.0, psi_cutoff=1e-3):
    """Domain function psi on the coarse grid (build_torso_grid.py:130-186):
    the signed distance to the torso surface of the fine segmentation (mm,
    positive inside), psi = (1 + tanh(3 d / width)) / 2, resampled linearly
    by spacing_fine / dx_coarse_mm, cropped or zero-padded to coarse_shape,
    and 0 below psi_cutoff (those cells leave the system)."""
    from scipy import ndimage as ndi
    inside = np.asarray(volume_fine) != 0
    sp = np.asarray(spacing_fine, np.float64)
    d = ndi.distance_transform_edt(inside, sampling=sp) - \
        ndi.distance_transform_edt(~inside, sampling=sp)
    psi_f = 0.5 * (1.0 + np.tanh(3.0 * d / float(interface_width_mm)))
    psi_c = ndi.zoom(psi_f, sp / float(dx_coarse_mm), order=1)
    out = np.zeros(tuple(coarse_shape), np.float64)
    n = tuple(min(a, b) for a, b in zip(psi_c.shape, coarse_shape))
    out[:n[0], :n[1], :n[2]] = psi_c[:n[0], :n[1], :n[2]]
    out[out < psi_cutoff] = 0.0
    return out


def extend_to_band(values, tissue_mask, active_mask):
    """values (labels or conductivities) carried from the nearest tissue
    voxel into the band active_mask & ~tissue_mask (build_torso_grid.py:
    189-206, constant extrapolation by the Euclidean distance transform's
    nearest-feature indices)."""
    from scipy import ndimage as ndi
    out = np.array(values, copy=True)
    band = np.asarray(active_mask) & ~np.asarray(tissue_mask)
    if not band.any():
        return out
    _, idx = ndi.distance_transform_edt(~np.asarray(tissue_mask), return_indices=True)
    out[band] = np.asarray(values)[tuple(ix[band] for ix in idx)]
    return out


def torso_grid_from_labels(labels, sigma_map, dx_mm, origin_mm=(0.0, 0.0, 0.0), save_path=None,
                           verbose=False, psi_vol=None):
    """Grid dict from a coarse label volume (0 = air) and label -> sigma
    [S/m]; psi_vol (coarse shape) selects the smoothed boundary."""
    labels = np.asarray(labels)
    shape = labels.shape
    keys = sorted(int(k) for k in sigma_map)
    if 0 in keys:
        keys.remove(0)
    if len(keys) + 1 > 16:
        raise ValueError("at most 15 tissue labels are supported")
    tissue = labels != 0
    if psi_vol is not None:
        psi_vol = np.asarray(psi_vol, np.float64)
        if psi_vol.shape != shape:
            raise ValueError(f"psi_vol {psi_vol.shape} and labels {shape} differ in shape")
        active = psi_vol > 0.0
        ext = extend_to_band(labels, tissue, active)
        ext[~active] = 0
    else:
        active, ext = tissue, labels
    lab = np.zeros(shape, np.uint8)
    table = [0.0]
    sigma_vol = np.zeros(shape, np.float64)
    for m, key in enumerate(keys, start=1):
        sel = ext == key
        lab[sel] = m
        table.append(float(sigma_map[key]))
        sigma_vol[sel] = float(sigma_map[key])
    unknown = (ext != 0) & (lab == 0)
    if unknown.any():
        raise ValueError(f"labels {np.unique(ext[unknown])} have no conductivity in sigma_map")
    active_flat = np.where(active.ravel())[0].astype(np.int32)
    id_map = np.full(labels.size, -1, np.int32)
    id_map[active_flat] = np.arange(len(active_flat), dtype=np.int32)
    pin = T.pin_row(tissue, id_map)
    surf_flat, surf_rows = T.surface_ids(labels, tissue, id_map)
    origin = np.asarray(origin_mm, np.float64)
    sbm = psi_vol is not None
    grid = dict(shape=shape, dx_mm=float(dx_mm), origin_mm=origin, sigma_vol=sigma_vol,
                active_mask=active, tissue_mask=tissue, active_ids=active_flat,
                active_id_map=id_map, surface_flat=surf_flat, surface_rows=surf_rows,
                surface_xyz=voxel_ids_to_xyz(surf_flat, shape, dx_mm, origin), pin_row=pin,
                use_sbm=sbm, labels=lab, sigma_table=np.asarray(table))
    if sbm:
        grid["psi_vol"] = psi_vol
    if verbose:
        print(f"  torso grid {shape} @ {dx_mm} mm: {len(active_flat):,} rows"
              + (f" ({int((active & ~tissue).sum()):,} smoothed-boundary band cells)" if sbm else ""))
    if save_path is not None:
        extra = {"psi_vol": psi_vol.astype(np.float32)} if sbm else {}
        np.savez(str(save_path), shape=np.array(shape, np.int32), dx_mm=np.float64(dx_mm),
                 origin_mm=origin, sigma_vol=sigma_vol.astype(np.float32), active_mask=active,
                 tissue_mask=tissue, active_ids=active_flat, active_id_map=id_map,
                 surface_flat=surf_flat, surface_rows=surf_rows,
                 surface_xyz=grid["surface_xyz"].astype(np.float32), pin_row=np.int32(pin),
                 use_sbm=sbm, labels=lab, sigma_table=np.asarray(table), **extra)
    return grid


def _resample_labels(volume, spacing, dx_coarse_mm):
    """Nearest-neighbour resampling to dx_coarse_mm (build_torso_grid.py:260-270)."""
    from scipy import ndimage as ndi
    zoom = np.asarray(spacing, np.float64) / float(dx_coarse_mm)
    return ndi.zoom(np.asarray(volume).astype(np.float32), zoom, order=0).astype(np.int32)


def compute_torso_grid(torso_nrrd_path=None, sigma_map=None, *, dx_coarse_mm=2.0, verbose=True,
                       save_path=None, use_sbm=False, sbm_interface_width_mm=3.0,
                       sbm_psi_cutoff=1e-3, labels=None, spacing_mm=None, origin_mm=None,
                       **_unused):
    """Grid dict from a torso segmentation: a NRRD file, or ``labels`` with
    their voxel size ``spacing_mm`` (resampled to dx_coarse_mm by nearest
    neighbour as the reference does), or ``labels`` already at dx_coarse_mm
    (spacing_mm None; no smoothed boundary, which needs the fine volume)."""
    if sigma_map is None:
        raise ValueError("sigma_map is required")
    fine, spacing = None, None
    if labels is None:
        try:
            import nrrd
        except ImportError as e:
            raise ImportError("reading a torso NRRD needs pynrrd; pass labels= instead") from e
        data, hdr = nrrd.read(str(torso_nrrd_path))
        if "space directions" in hdr:
            spacing = np.linalg.norm(np.asarray(hdr["space directions"], np.float64), axis=1)
            origin_mm = np.asarray(hdr.get("space origin", np.zeros(3)), np.float64)
        elif "spacings" in hdr:
            spacing = np.asarray(hdr["spacings"], np.float64)
        else:
            spacing = np.ones(3)
        fine = np.asarray(data, np.int32)
    elif spacing_mm is not None:
        fine = np.asarray(labels)
        spacing = np.broadcast_to(np.asarray(spacing_mm, np.float64), (3,))
    if fine is not None:
        coarse = _resample_labels(fine, spacing, dx_coarse_mm)
    else:
        coarse = np.asarray(labels)
    psi = None
    if use_sbm:
        if fine is None:
            raise ValueError("use_sbm=True builds psi from the fine segmentation: pass the NRRD "
                             "path, or labels with their spacing_mm")
        psi = smoothed_domain(fine, spacing, dx_coarse_mm, coarse.shape,
                              interface_width_mm=sbm_interface_width_mm, psi_cutoff=sbm_psi_cutoff)
    return torso_grid_from_labels(coarse, sigma_map, dx_coarse_mm,
                                  origin_mm if origin_mm is not None else (0.0, 0.0, 0.0),
                                  save_path=save_path, verbose=verbose, psi_vol=psi)


def load_torso_grid(out_path, torso_nrrd_path=None, sigma_map=None, dx_coarse_mm=None,
                    verbose=True):
    data = np.load(str(out_path))
    g = {k: data[k] for k in data.files}
    g["shape"] = tuple(np.asarray(g["shape"]).tolist())
    g["dx_mm"] = float(g["dx_mm"])
    g["pin_row"] = int(g["pin_row"])
    g["use_sbm"] = bool(g.get("use_sbm", False))
    if "psi_vol" in g:
        g["psi_vol"] = g["psi_vol"].astype(np.float64)
    return g
