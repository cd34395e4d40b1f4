"""compute_bspm / run_bspm_loop with the reference's signatures
(ecg/bspm.py:33-145, ecg/functions/compute_bspm.py:445-670).

Per frame: the heart source (sigma_i / h^2) K Vm, de-meaned over the
projected nodes, scattered onto torso rows and divided by the expected
number of fine voxels per coarse voxel; then Jacobi-PCG warm-started from
the previous frame -- all on the GPU (hp_torso_solve_frame).  cg_metric
'rms' / 'p99' / 'linf' keep the reference's absolute-mV stop on z = M^-1 r
(p99: the 0.99 quantile of |z| with torch.quantile's linear
interpolation, decided exactly on the device); the extra metric 'rel' stops
on the FP64 true relative residual (cg_tol_rel).  A grid built with
use_sbm=True solves the smoothed-boundary system (psi-weighted faces and
right-hand side, compute_bspm.py:413-414, :542-546).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from . import torso as T
from .._spacing import resolve_voxel_size

DEFAULT_SIGMA_I = 0.2625
DEFAULT_H_FINE_MM = 0.4


def run_bspm_loop(vm_snapshots_path, grid, registration, sigma_i, h_fine_mm, out_path,
                  cg_tol_mV=0.01, cg_max_iter=500, cg_metric="rms", t_window=None, verbose=True,
                  full_field_frames=None, full_field_out_path=None, cg_tol_rel=1e-6,
                  electrodes_mm=None, return_stats=False):
    if cg_metric not in ("rms", "linf", "rel", "p99"):
        raise ValueError(f"metric must be one of 'rms', 'p99', 'linf', got {cg_metric!r}")
    snap = np.load(str(vm_snapshots_path))
    Vm_all = snap["Vm"].astype(np.float32)
    coords = snap["coords_mm"].astype(np.float64)
    vox = snap["vox_idx"].astype(np.int32)
    time_ms = snap["time_vm"].astype(np.float64)
    if t_window is not None:
        keep = (time_ms >= t_window[0]) & (time_ms <= t_window[1])
        if not keep.any():
            raise ValueError(f"t_window={t_window} selected 0 frames out of "
                             f"[{time_ms.min():.1f}, {time_ms.max():.1f}] ms available.")
        Vm_all, time_ms = Vm_all[keep], time_ms[keep]
    n_frames = Vm_all.shape[0]
    labels, table = T.labels_from_grid(grid)
    proj, valid = T.projection_map(coords, registration["R"], registration["t"],
                                   float(registration["scale"]), grid["origin_mm"],
                                   grid["dx_mm"], grid["active_id_map"], grid["shape"])
    surf_rows = np.asarray(grid["surface_rows"], np.int64)
    read = [surf_rows]
    n_el = 0
    if electrodes_mm is not None:
        el_rows = T.nearest_surface_rows(electrodes_mm, grid["surface_xyz"], surf_rows)
        read.append(el_rows)
        n_el = len(el_rows)
    full_set = sorted(set(int(f) for f in full_field_frames)) if full_field_frames is not None else []
    if full_set and full_field_out_path is None:
        raise ValueError("full_field_frames given but full_field_out_path is None")
    if full_set and (min(full_set) < 0 or max(full_set) >= n_frames):
        raise ValueError("full_field_frames contains indices outside the frame range")
    solver = T.TorsoSolver(labels, table, grid["dx_mm"], grid["pin_row"],
                           T.heart_neighbours(vox), proj, sigma_i, h_fine_mm,
                           np.concatenate(read), psi=T.psi_from_grid(grid))
    tol = cg_tol_rel if cg_metric == "rel" else cg_tol_mV
    try:
        solver.solve_frame(Vm_all[0], tol, cg_metric, cg_max_iter)   # warm-up, as the reference
        N_surf = len(surf_rows)
        bspm = np.zeros((N_surf, n_frames), np.float32)
        el = np.zeros((n_el, n_frames), np.float32)
        iters = np.zeros(n_frames, np.int32)
        rel = np.zeros(n_frames)
        full = np.zeros((len(grid["active_ids"]), len(full_set)), np.float32) if full_set else None
        for f in range(n_frames):
            out, st = solver.solve_frame(Vm_all[f], tol, cg_metric, cg_max_iter)
            bspm[:, f] = out[:N_surf]
            el[:, f] = out[N_surf:]
            iters[f] = st.iterations
            rel[f] = st.rel_residual
            if f in full_set:
                full[:, full_set.index(f)] = solver.solution() * 1e3
    finally:
        solver.close()
    if full_set:
        np.savez(str(full_field_out_path), phi_full=full, frame_indices=np.array(full_set, np.int64),
                 time_ms=time_ms[full_set], active_ids=np.asarray(grid["active_ids"], np.int32),
                 shape=np.array(grid["shape"], np.int32), dx_mm=np.float64(grid["dx_mm"]),
                 origin_mm=np.asarray(grid["origin_mm"], np.float64))
    np.savez(str(out_path), surface_xyz=np.asarray(grid["surface_xyz"], np.float32),
             surface_flat=np.asarray(grid["surface_flat"], np.int32), dx_mm=np.float64(grid["dx_mm"]),
             bspm_signal=bspm, time_ms=time_ms.astype(np.float64),
             reg_R=np.asarray(registration["R"], np.float64),
             reg_t=np.asarray(registration["t"], np.float64),
             reg_scale=np.float64(registration["scale"]),
             reg_dice=np.float64(float(registration.get("dice", np.nan))),
             sigma_i=np.float64(sigma_i), h_fine_mm=np.float64(h_fine_mm))
    if return_stats:
        return bspm, dict(iterations=iters, rel_residual=rel, electrodes=el)
    return bspm


def compute_bspm(vm_snapshots_path, grid, registration, *, anatomy=None, sigma_i=DEFAULT_SIGMA_I,
                 h_fine_mm=DEFAULT_H_FINE_MM, cg_tol_mV=0.01, cg_max_iter=500, cg_metric="rms",
                 t_window=None, verbose=True, save_path=None, full_field_frames=None,
                 full_field_save_path=None, **extra):
    if save_path is None:
        raise ValueError("compute_bspm requires save_path (run_bspm_loop writes results "
                         "incrementally as it solves).")
    h_fine_mm = resolve_voxel_size(h_fine_mm, anatomy, param_name="h_fine_mm")
    return run_bspm_loop(Path(vm_snapshots_path), grid, registration, sigma_i, h_fine_mm,
                         Path(save_path), cg_tol_mV=cg_tol_mV, cg_max_iter=cg_max_iter,
                         cg_metric=cg_metric, t_window=t_window, verbose=verbose,
                         full_field_frames=full_field_frames,
                         full_field_out_path=(Path(full_field_save_path)
                                              if full_field_save_path is not None else None),
                         **extra)


def load_bspm(path):
    path = Path(path).with_suffix(".npz")
    if not path.exists():
        raise FileNotFoundError(f"No saved BSPM at {path}")
    z = np.load(str(path))
    return {k: z[k] for k in z.files}
