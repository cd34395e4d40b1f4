"""compute_coupled / run_coupled with the signatures of the reference's
hrdayapy/simulation/coupled.py:33-131 and
simulation/functions/purkinje_myocardium_pipeline.py:1030-1069.

The time loop runs on the GPU (libhrdaya_b200): theta = 0 the fused explicit
step, 0 < theta <= 1 (default 0.5, as the reference) the theta-scheme with a
CG solve per step (cg_tol, cg_max_iter).  Extra keyword arguments act_threshold /
deact_threshold / max_events control the in-loop activation recording whose
tables are added to the returned dict ("activation_times", ...).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from .. import monodomain
from .._spacing import resolve_voxel_size


def run_coupled(nodes, elements, activation_times, S, Z, phi, *, voxel_size=0.4, dx_p=0.2,
                sigma_P=0.225, sigma_M=6.5625e-5, Cm=0.01, A_P=133.33, A_M=0.14, R_P=0.015,
                dt=0.1, T=400.0, theta=0.5, stim_protocol=None, ectopic_region=None,
                stim_len_mm=2.0, c_pmj=0.05, n_pmj=1, cg_tol=1e-5, cg_max_iter=100,
                n_frames=100, device=None, dtype=None, out_npz=None, phi_endo_max=0.35,
                phi_epi_min=0.65, vm_save_dt=None, out_vm_npz=None, vm_tmp_dir=None,
                act_threshold=-40.0, deact_threshold=-40.0, max_events=4, brick=None):
    return monodomain.run(
        nodes, elements, activation_times, S, Z, phi, anisotropic=False, theta=theta,
        dtype=dtype, device=device, n_frames=n_frames, out_npz=out_npz, out_vm_npz=out_vm_npz,
        vm_save_dt=vm_save_dt, vm_tmp_dir=vm_tmp_dir, cg_tol=cg_tol, cg_max_iter=cg_max_iter,
        voxel_size=voxel_size, dx_p=dx_p, sigma_P=sigma_P, sigma_M=sigma_M, Cm=Cm, A_P=A_P,
        A_M=A_M, R_P=R_P, dt=dt, T=T, stim_protocol=stim_protocol,
        ectopic_region=ectopic_region, stim_len_mm=stim_len_mm, c_pmj=c_pmj, n_pmj=n_pmj,
        phi_endo_max=phi_endo_max, phi_epi_min=phi_epi_min, act_threshold=act_threshold,
        deact_threshold=deact_threshold, max_events=max_events, brick=brick)


def compute_coupled(nodes, elements, act_times, S, Z, phi, *, anatomy=None, stim_protocol=None,
                    ectopic_region=None, voxel_size=0.4, dx_p: float = 0.2,
                    sigma_P: float = 0.45, sigma_M: float = 1.31e-4, Cm: float = 0.01,
                    A_P: float = 133.33, A_M: float = 0.14, R_P: float = 0.015,
                    dt: float = 0.1, T: float = 400.0, theta: float = 0.5,
                    stim_len_mm: float = 2.0, c_pmj: float = 0.05, n_pmj: int = 1,
                    cg_tol: float = 1e-5, cg_max_iter: int = 500, n_frames: int = 100,
                    device=None, phi_endo_max: float = 0.35, phi_epi_min: float = 0.65,
                    save_path=None, vm_save_dt=None, vm_save_path=None, vm_tmp_dir=None,
                    **extra):
    voxel_size = resolve_voxel_size(voxel_size, anatomy, param_name="voxel_size")
    return run_coupled(
        nodes=nodes, elements=elements, activation_times=act_times, S=S, Z=Z, phi=phi,
        voxel_size=voxel_size, dx_p=dx_p, sigma_P=sigma_P, sigma_M=sigma_M, Cm=Cm, A_P=A_P,
        A_M=A_M, R_P=R_P, dt=dt, T=T, theta=theta, stim_protocol=stim_protocol,
        ectopic_region=ectopic_region, stim_len_mm=stim_len_mm, c_pmj=c_pmj, n_pmj=n_pmj,
        cg_tol=cg_tol, cg_max_iter=cg_max_iter, n_frames=n_frames, device=device,
        out_npz=save_path, phi_endo_max=phi_endo_max, phi_epi_min=phi_epi_min,
        vm_save_dt=vm_save_dt, out_vm_npz=vm_save_path, vm_tmp_dir=vm_tmp_dir, **extra)


def load_coupled(path):
    path = Path(path).with_suffix(".npz")
    if not path.exists():
        raise FileNotFoundError(f"No saved coupled simulation at {path}")
    z = np.load(path)
    return {k: z[k] for k in z.files}
