"""Generate the golden fixtures in this directory by running the UPSTREAM
HrdayaPy code itself (loaded from its source tree by _refload.py).

Run once in a container that has the upstream sources:

    python tests/golden/make_golden.py

Fixtures (all seeded, small enough to commit):

* ttp06_cells.npz   -- one step of gpu_ttp06._currents_and_gates (FP64) on
                       random physiological states, all three phenotypes.
* ttp06_pacing.npz  -- single-cell 1-beat pacing trace (experiment_1 recipe:
                       52 pA/pF for 1 ms, dt 0.02 ms), all three phenotypes.
* mono_iso.npz      -- run_coupled at theta=0, FP64, on a 16x16x4 slab with
                       an inert Purkinje stub (c_pmj=0), corner stimulus.
* mono_aniso.npz    -- anisotropic solver at theta=0, FP64, on a 12x10x6 slab
                       with a seeded fibre field, three phenotypes, a small
                       coupled Purkinje tree (root stimulus, c_pmj=0.01 mS)
                       and a myocardial focus stimulated at t = 1 ms.
                       Also the theta=0.5 activation map for the scheme gap.
* act_maps_iso.npz  -- compute_activation_maps + save_activation_maps on the
                       snapshots (every 0.5 ms) of a 340 ms run_coupled on
                       the isotropic slab (activation and repolarisation),
                       and on a seeded chattering trace with debounce.
* pmj_exp4.npz      -- the upstream Experiment 4 core
                       (experiments/experiment_3/experiment_common.py
                       run_directional) on its slab + fibre at dx 0.25 mm:
                       orthodromic capture and block, antidromic capture.
* torso.npz         -- _assemble_stiffness / _find_surface_ids on a small
                       synthetic torso, build_heart_laplacian /
                       build_projection_map, and solve_frame on one Vm frame.
* transmural.npz    -- generate_transmural_coordinate on a small truncated
                       ellipsoidal shell (epicardium +1, endocardium -1,
                       a Neumann base plane).
* bspm_loop.npz     -- the upstream chain end to end: run_coupled (theta 0,
                       FP64) writes vm_snapshots.npz of a 24x24x8 slab at
                       0.5 mm (1 ms frames), run_bspm_loop solves every frame
                       on the small torso of torso.npz and writes bspm.npz;
                       both files' arrays (vm_*, out_*) and their dtypes.
"""
from __future__ import annotations

import contextlib
import io
import sys
import tempfile
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import _refload  # noqa: E402

ref = _refload.load()
STATE_INIT = np.array([138.4, 10.355, 0.00013, 0.00448, 0.476, 0.0087, 0.00155,
                       0.7573, 0.7225, 3.164e-5, 0.8009, 0.9778, 0.9953, 0.3212,
                       2.235e-8, 3.715, 0.9068, 0.00036])


def quiet(fn, *a, **k):
    with contextlib.redirect_stdout(io.StringIO()):
        return fn(*a, **k)


def ttp06_cells():
    rng = np.random.default_rng(1234)
    g = ref.gpu_ttp06
    out = {}
    for key, cls in (("endo", g.EndoTTP06), ("mid", g.MidTTP06), ("epi", g.EpiTTP06)):
        n = 256
        V = rng.uniform(-95.0, 50.0, n)
        V[:4] = [-40.0, -40.0 + 1e-9, 15.0, -86.709]      # branch points / CaL guard
        st = np.tile(STATE_INIT, (n, 1))
        gates = [3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 16]
        st[:, gates] = rng.uniform(0.0, 1.0, (n, len(gates)))
        conc = [0, 1, 2, 15, 17]
        st[:, conc] *= rng.uniform(0.7, 1.3, (n, len(conc)))
        I, st2 = cls().step(torch.tensor(V), torch.tensor(st), 0.02, 0.0)
        out[f"{key}_V"] = V
        out[f"{key}_state"] = st
        out[f"{key}_Iion"] = I.numpy()
        out[f"{key}_state_out"] = st2.numpy()
    np.savez_compressed(HERE / "ttp06_cells.npz", **out)


def ttp06_pacing():
    g = ref.gpu_ttp06
    dt, n_steps, stim_steps = 0.02, 20000, 50
    out = {"dt": dt}
    for key, cls in (("endo", g.EndoTTP06), ("mid", g.MidTTP06), ("epi", g.EpiTTP06)):
        m = cls()
        st = m.init_state_tensor(1, torch.device("cpu"), torch.float64)
        V = torch.full((1,), -86.709, dtype=torch.float64)
        trace = np.empty(n_steps)
        for k in range(n_steps):
            Is = 52.0 if k < stim_steps else 0.0
            I, st = m.step(V, st, dt, Is)
            V = V + dt * (Is - I)
            trace[k] = V.item()
        out[f"{key}_V"] = trace[::25].copy()          # every 0.5 ms
        out[f"{key}_V_fine"] = trace[:500].copy()     # first 10 ms, every step
        out[f"{key}_state_end"] = st.numpy()[0]
    np.savez_compressed(HERE / "ttp06_pacing.npz", **out)


def _stub(nx, ny, nz):
    nodes = np.array([[ny + 8.0, nx + 8.0, nz + 8.0], [ny + 8.0, nx + 8.0, nz + 12.0]])
    return nodes, np.array([[0, 1]]), np.array([0.0, 1.0])


def mono_iso():
    nx, ny, nz = 16, 16, 4
    h, dt, T = 0.25, 0.02, 20.0
    S = np.ones((nx, ny, nz), np.uint8)
    phi = np.ones(S.shape, np.float32)
    ect = np.zeros(S.shape, bool)
    ect[:4, :4, :] = True
    nodes, el, act = _stub(nx, ny, nz)
    prot = [dict(name="corner", target="ectopic", amp=0.52, dur=1.0, onset=0.0)]
    out = {}
    for theta in (0.0, 0.5):
        with tempfile.TemporaryDirectory() as td:
            vm_path = Path(td) / "vm.npz"
            quiet(ref.pipeline.run_coupled, nodes, el, act, S, S.copy(), phi,
                  voxel_size=h, dx_p=0.25, sigma_P=0.0, sigma_M=0.13, Cm=0.01, A_P=133.33,
                  A_M=140.0, R_P=0.015, dt=dt, T=T, theta=theta, stim_protocol=prot,
                  ectopic_region=ect, stim_len_mm=1.0, c_pmj=0.0, n_pmj=1,
                  cg_tol=1e-12, cg_max_iter=200, n_frames=10, device="cpu",
                  dtype=torch.float64, vm_save_dt=dt, out_vm_npz=vm_path)
            snap = quiet(ref.load_vm_snapshots.load_vm_snapshots, vm_path)
            maps = quiet(ref.activation_maps.compute_activation_maps, snap, S,
                         act_threshold=-20.0, deact_threshold=-20.0)
            tag = "" if theta == 0.0 else "_cn"
            out["act" + tag] = maps.activation_times
            if theta == 0.0:
                out["Vm_sub"] = np.asarray(snap.Vm)[::25].copy()
                out["time_sub"] = np.asarray(snap.time_vm)[::25].copy()
                out["Vm_last"] = np.asarray(snap.Vm)[-1].copy()
                out["n_frames"] = np.int64(snap.n_frames)
                out["vox_idx"] = np.asarray(snap.vox_idx)
    out.update(h=h, dt=dt, T=T, nx=nx, ny=ny, nz=nz)
    np.savez_compressed(HERE / "mono_iso.npz", **out)


def aniso_case():
    """Geometry shared with the tests (restated there from these numbers)."""
    nx, ny, nz = 12, 10, 6
    rng = np.random.default_rng(7)
    S = np.ones((nx, ny, nz), np.uint8)
    S[0, 0, :] = 0                                   # a notch: masked-out voxels
    S[nx - 1, ny - 1, nz - 1] = 0
    ii, jj, kk = np.indices(S.shape)
    phi = (kk / (nz - 1)).astype(np.float32)         # endo at k=0 .. epi at k=nz-1
    phi[S == 0] = np.nan
    a = 0.4 * ii + 0.3 * jj + rng.uniform(0, 0.2, S.shape)
    b = 0.5 * kk / nz
    f = np.stack([np.cos(a) * np.cos(b), np.sin(a) * np.cos(b), np.sin(b)], -1)
    f /= np.linalg.norm(f, axis=-1, keepdims=True)
    fibre = f.astype(np.float32)
    # small Purkinje tree in (x,y,z) = (col,row,depth) voxel units, sitting
    # just below the k=0 face (endocardium side)
    nodes = np.array([[1.0, 1.0, -2.0], [4.0, 5.0, -1.0], [8.0, 3.0, -0.5],
                      [3.0, 9.0, -0.5], [7.0, 10.0, -0.6]])
    el = np.array([[0, 1], [1, 2], [1, 3], [3, 4]])
    act = np.array([0.0, 1.0, 2.0, 2.0, 3.0])
    return S, phi, fibre, nodes, el, act


def mono_aniso():
    S, phi, fibre, nodes, el, act = aniso_case()
    h, dt, T = 0.4, 0.02, 20.0
    ect = np.zeros(S.shape, bool)
    ect[8:12, 6:10, 3:6] = True
    prot = [dict(name="av_node", target="root", amp=12.0, dur=2.0, onset=0.0),
            dict(name="focus", target="ectopic", amp=1.0, dur=2.0, onset=1.0)]
    kw = dict(voxel_size=h, dx_p=0.2, sigma_P=0.45, sigma_l=0.34, sigma_t=0.06,
              Cm=0.01, A_M=140.0, R_P=0.015, dt=dt, T=T, stim_protocol=prot,
              ectopic_region=ect,
              stim_len_mm=0.5, c_pmj=0.01, n_pmj=2, cg_tol=1e-12, cg_max_iter=200,
              n_frames=10, device="cpu", dtype=torch.float64, phi_endo_max=0.3,
              phi_epi_min=0.7, vm_save_dt=dt)
    out = {}
    for theta in (0.0, 0.5):
        with tempfile.TemporaryDirectory() as td:
            vm_path = Path(td) / "vm.npz"
            res = quiet(ref.aniso.purkinje_myocardium_anisotropic_solver, nodes, el, act,
                        S, S.copy(), phi, fibre, theta=theta, out_vm_npz=vm_path,
                        frame_save_dt=dt, anim_tmp_dir=td, **kw)
            snap = quiet(ref.load_vm_snapshots.load_vm_snapshots, vm_path)
            maps = quiet(ref.activation_maps.compute_activation_maps, snap, S,
                         act_threshold=-20.0, deact_threshold=-20.0)
            tag = "" if theta == 0.0 else "_cn"
            out["act" + tag] = maps.activation_times
            if theta == 0.0:
                out["Vm_sub"] = np.asarray(snap.Vm)[::25].copy()
                out["time_sub"] = np.asarray(snap.time_vm)[::25].copy()
                out["Vm_last"] = np.asarray(snap.Vm)[-1].copy()
                bm = res["branch_map"]
                Vp = np.zeros((len(res["times"]), len(res["comp_nodes"])), np.float32)
                for b, arr in zip(bm, res["branch_frames_p"]):
                    Vp[:, np.asarray(b)] = np.asarray(arr)
                out["Vp_sub"] = Vp[::25].copy()
                out["n_comp"] = np.int64(len(res["comp_nodes"]))
                out["vox_idx"] = np.asarray(snap.vox_idx)
    out.update(h=h, dt=dt, T=T)
    np.savez_compressed(HERE / "mono_aniso.npz", **out)


def torso_case():
    """Small synthetic torso: elliptic cylinder, two lungs, a blood pool.
    Labels: 0 air, 1 bulk, 2 lung, 3 blood."""
    ni, nj, nk = 22, 18, 24
    ii, jj, kk = np.indices((ni, nj, nk)).astype(np.float64)
    ci, cj = (ni - 1) / 2, (nj - 1) / 2
    lab = np.zeros((ni, nj, nk), np.int32)
    body = ((ii - ci) / 10.0) ** 2 + ((jj - cj) / 8.0) ** 2 <= 1.0
    body &= (kk >= 1) & (kk <= nk - 2)
    lab[body] = 1
    for sgn in (-1, 1):
        lung = ((ii - ci - sgn * 5) / 3.5) ** 2 + ((jj - cj) / 4.5) ** 2 + ((kk - 13) / 7) ** 2 <= 1
        lab[lung & body] = 2
    blood = ((ii - ci) / 2.0) ** 2 + ((jj - cj - 1) / 2.0) ** 2 + ((kk - 10) / 2.5) ** 2 <= 1
    lab[blood & body] = 3
    return lab


def torso():
    btg = ref.build_torso_grid
    cb = ref.compute_bspm
    lab = torso_case()
    dx = 1.5
    sig_map = {1: 0.2, 2: 0.05, 3: 0.7}
    sigma = np.zeros(lab.shape)
    for k, v in sig_map.items():
        sigma[lab == k] = v
    active = lab != 0
    active_flat = np.where(active.ravel())[0].astype(np.int32)
    id_map = np.full(lab.size, -1, np.int32)
    id_map[active_flat] = np.arange(len(active_flat), dtype=np.int32)
    A = btg._assemble_stiffness(sigma, dx * 1e-3, active, active_flat, id_map)
    surf_flat, surf_rows = btg._find_surface_ids(lab, active, id_map)
    interior = np.where(active.ravel())[0]
    pin_flat = int(interior[len(interior) // 2])
    pin_row = int(id_map[pin_flat])
    # heart: fine voxels (0.5 mm) of a thick spherical shell inside the torso
    h_f = 0.5
    origin = np.zeros(3)
    gi, gj, gk = np.indices((36, 30, 36))
    cen = np.array([17.5, 14.5, 17.5])
    r = np.sqrt((gi - cen[0]) ** 2 + (gj - cen[1]) ** 2 + (gk - cen[2]) ** 2)
    shell = (r >= 9) & (r <= 14)
    vox = np.argwhere(shell).astype(np.int32)
    coords = (vox[:, [1, 0, 2]].astype(np.float64)) * h_f
    # registration: heart coords (x,y,z) -> torso mm; place shell centre near
    # the torso centre (ijk convention of the coarse grid)
    R = np.eye(3)
    t = np.array([8.0, 6.0, 12.0])
    K = cb.build_heart_laplacian(vox, len(vox), h_f)
    proj, valid = quiet(cb.build_projection_map, coords, R, t, 1.0, origin, dx,
                        id_map, lab.shape)
    # one Vm frame: a planar wavefront through the shell
    rng = np.random.default_rng(3)
    x = vox[:, 0].astype(np.float64)
    Vm = (-85.0 + 110.0 / (1.0 + np.exp(-(x - 17.0) / 1.5)) + rng.normal(0, 0.5, len(vox)))
    Vm = Vm.astype(np.float32)
    solve, iters = quiet(cb.make_gpu_solver, A, pin_row, proj, valid, cb._scipy_csr_to_torch(
        K, torch.device("cpu"), torch.float32), 0.2625, h_f * 1e-3, dx, surf_rows,
        len(active_flat), torch.device("cpu"), cg_tol_mV=1e-7, cg_max=5000, cg_metric="linf")
    phi_s, n_it, res_mV, phi_full = quiet(solve, Vm, capture_full=True)
    A = A.tocsr()
    np.savez_compressed(
        HERE / "torso.npz", labels=lab, dx=dx, sigma_keys=np.array(list(sig_map)),
        sigma_vals=np.array(list(sig_map.values())), A_indptr=A.indptr, A_indices=A.indices,
        A_data=A.data, surf_flat=surf_flat, surf_rows=surf_rows, pin_row=pin_row,
        heart_vox=vox, h_fine=h_f, reg_t=t, K_indptr=K.indptr, K_indices=K.indices,
        K_data=K.data, proj=proj, valid=valid, Vm=Vm, phi_surf_ref=phi_s,
        phi_full_ref=phi_full, ref_iters=n_it)


def sbm_case():
    """Fine (0.75 mm) segmentation of a small torso for the smoothed-boundary
    method: elliptic cylinder with two lungs and a blood pool, boundaries
    placed off the coarse (1.5 mm) grid.  Labels: 0 air, 1 bulk, 2 lung,
    3 blood."""
    ni, nj, nk = 44, 36, 48
    x, y, z = (np.indices((ni, nj, nk)).astype(np.float64) + 0.5) * 0.75
    cx, cy = ni * 0.75 / 2, nj * 0.75 / 2
    lab = np.zeros((ni, nj, nk), np.int32)
    body = ((x - cx) / 14.6) ** 2 + ((y - cy) / 11.3) ** 2 <= 1.0
    body &= (z >= 2.2) & (z <= 33.4)
    lab[body] = 1
    for sgn in (-1, 1):
        lung = (((x - cx - sgn * 7.6) / 5.1) ** 2 + ((y - cy) / 6.4) ** 2
                + ((z - 19.0) / 10.2) ** 2 <= 1)
        lab[lung & body] = 2
    blood = ((x - cx) / 3.1) ** 2 + ((y - cy - 1.4) / 2.9) ** 2 + ((z - 15.2) / 3.6) ** 2 <= 1
    lab[blood & body] = 3
    return lab, 0.75


def sbm():
    """The upstream smoothed-boundary set-up and stiffness on sbm_case, and a
    frame solved by the upstream GPU solver loop (on the CPU) with its
    psi-weighted right-hand side."""
    btg = ref.build_torso_grid
    cb = ref.compute_bspm
    fine, sp_f = sbm_case()
    spacing = np.full(3, sp_f)
    dx = 1.5
    sig_map = {1: 0.2, 2: 0.05, 3: 0.7}
    coarse = btg._resample_labels(fine, spacing, dx)
    sigma = np.zeros(coarse.shape)
    for k, v in sig_map.items():
        sigma[coarse == k] = v
    tissue = coarse != 0
    psi = btg.compute_smoothed_domain(fine, spacing, dx, coarse.shape, interface_width_mm=3.0,
                                      psi_cutoff=1e-3)
    active = psi > 0.0
    sigma_ext = btg.extend_conductivity(sigma, tissue, active)
    active_flat = np.where(active.ravel())[0].astype(np.int32)
    id_map = np.full(coarse.size, -1, np.int32)
    id_map[active_flat] = np.arange(len(active_flat), dtype=np.int32)
    A = btg._assemble_stiffness(sigma_ext, dx * 1e-3, active, active_flat, id_map, psi_vol=psi)
    interior = np.where(tissue.ravel())[0]
    pin_row = int(id_map[int(interior[len(interior) // 2])])
    surf_flat, surf_rows = btg._find_surface_ids(coarse, tissue, id_map)
    # heart shell and wavefront as in torso(), registered into this torso
    h_f = 0.5
    gi, gj, gk = np.indices((36, 30, 36))
    cen = np.array([17.5, 14.5, 17.5])
    r = np.sqrt((gi - cen[0]) ** 2 + (gj - cen[1]) ** 2 + (gk - cen[2]) ** 2)
    vox = np.argwhere((r >= 9) & (r <= 14)).astype(np.int32)
    coords = (vox[:, [1, 0, 2]].astype(np.float64)) * h_f
    R = np.eye(3)
    t = np.array([8.0, 6.0, 9.0])
    K = cb.build_heart_laplacian(vox, len(vox), h_f)
    proj, valid = quiet(cb.build_projection_map, coords, R, t, 1.0, np.zeros(3), dx,
                        id_map, coarse.shape)
    rng = np.random.default_rng(5)
    xv = vox[:, 0].astype(np.float64)
    Vm = (-85.0 + 110.0 / (1.0 + np.exp(-(xv - 17.0) / 1.5)) + rng.normal(0, 0.5, len(vox)))
    Vm = Vm.astype(np.float32)
    psi_row = psi.ravel()[active_flat]
    solve, iters = quiet(cb.make_gpu_solver, A, pin_row, proj, valid, cb._scipy_csr_to_torch(
        K, torch.device("cpu"), torch.float32), 0.2625, h_f * 1e-3, dx, surf_rows,
        len(active_flat), torch.device("cpu"), cg_tol_mV=1e-7, cg_max=20000, cg_metric="linf",
        psi_row=psi_row)
    phi_s, n_it, res_mV, phi_full = quiet(solve, Vm, capture_full=True)
    A = A.tocsr()
    np.savez_compressed(
        HERE / "sbm.npz", fine=fine.astype(np.uint8), spacing=spacing, dx=dx, coarse=coarse,
        sigma_keys=np.array(list(sig_map)), sigma_vals=np.array(list(sig_map.values())),
        psi=psi, sigma_ext=sigma_ext, active_ids=active_flat, A_indptr=A.indptr,
        A_indices=A.indices, A_data=A.data, pin_row=pin_row, surf_flat=surf_flat,
        surf_rows=surf_rows, heart_vox=vox, h_fine=h_f, reg_t=t, proj=proj, valid=valid, Vm=Vm,
        phi_surf_ref=phi_s, phi_full_ref=phi_full, ref_iters=n_it)


def bspm_case():
    """Slab, stimulus and registration of bspm_loop (restated in the tests)."""
    nx, ny, nz = 24, 24, 8
    S = np.ones((nx, ny, nz), np.uint8)
    phi = np.ones(S.shape, np.float32)
    ect = np.zeros(S.shape, bool)
    ect[:4, :4, :] = True
    nodes, el, act = _stub(nx, ny, nz)
    kw = dict(voxel_size=0.5, dx_p=0.25, sigma_P=0.0, sigma_M=0.13, Cm=0.01, A_P=133.33,
              A_M=140.0, R_P=0.015, dt=0.02, T=12.0, theta=0.0,
              stim_protocol=[dict(name="corner", target="ectopic", amp=0.52, dur=1.0,
                                  onset=0.0)],
              ectopic_region=ect, stim_len_mm=1.0, c_pmj=0.0, n_pmj=1)
    reg = dict(R=np.eye(3), t=np.array([9.75, 7.5, 16.0]), scale=1.0, dice=0.9)
    return (nodes, el, act, S, phi), kw, reg


def bspm_loop():
    btg = ref.build_torso_grid
    cb = ref.compute_bspm
    (nodes, el, act, S, phi), kw, reg = bspm_case()
    lab = torso_case()
    dx = 1.5
    sig_map = {1: 0.2, 2: 0.05, 3: 0.7}
    sigma = np.zeros(lab.shape)
    for k, v in sig_map.items():
        sigma[lab == k] = v
    active = lab != 0
    active_flat = np.where(active.ravel())[0].astype(np.int32)
    id_map = np.full(lab.size, -1, np.int32)
    id_map[active_flat] = np.arange(len(active_flat), dtype=np.int32)
    A = btg._assemble_stiffness(sigma, dx * 1e-3, active, active_flat, id_map)
    surf_flat, surf_rows = btg._find_surface_ids(lab, active, id_map)
    interior = np.where(active.ravel())[0]
    pin_row = int(id_map[int(interior[len(interior) // 2])])
    origin = np.zeros(3)
    grid = dict(shape=lab.shape, dx_mm=dx, origin_mm=origin, sigma_vol=sigma,
                active_mask=active, tissue_mask=active, active_ids=active_flat,
                active_id_map=id_map, surface_flat=surf_flat, surface_rows=surf_rows,
                surface_xyz=btg.voxel_ids_to_xyz(surf_flat, lab.shape, dx, origin),
                pin_row=pin_row, A_scipy=A, use_sbm=False)
    out = {}
    sync = torch.cuda.synchronize
    torch.cuda.synchronize = lambda *a, **k: None     # the loop syncs CUDA after its warm-up
    try:
        with tempfile.TemporaryDirectory() as td:
            vm_path = Path(td) / "vm_snapshots.npz"
            out_path = Path(td) / "bspm.npz"
            quiet(ref.pipeline.run_coupled, nodes, el, act, S, S.copy(), phi, cg_tol=1e-12,
                  cg_max_iter=200, n_frames=10, device="cpu", dtype=torch.float64,
                  vm_save_dt=1.0, out_vm_npz=vm_path, **kw)
            quiet(cb.run_bspm_loop, vm_path, grid, reg, 0.2625, 0.5, out_path, cg_tol_mV=1e-6,
                  cg_max_iter=5000, cg_metric="rms", verbose=False)
            for tag, path in (("vm", vm_path), ("out", out_path)):
                z = np.load(path)
                out[f"{tag}_keys"] = np.array(sorted(z.files))
                out[f"{tag}_dtypes"] = np.array([str(z[k].dtype) for k in sorted(z.files)])
                for k in z.files:
                    out[f"{tag}_{k}"] = z[k]
    finally:
        torch.cuda.synchronize = sync
    np.savez_compressed(HERE / "bspm_loop.npz", labels=lab, dx=dx,
                        sigma_keys=np.array(list(sig_map)),
                        sigma_vals=np.array(list(sig_map.values())), **out)


def transmural_case():
    """Truncated ellipsoidal shell with its surface labels (restated in the
    tests): +1 on myocardial voxels touching the exterior, -1 on those
    touching the cavity, nothing on the cut base plane."""
    from scipy import ndimage as ndi
    n = (30, 26, 24)
    ii, jj, kk = np.indices(n).astype(np.float64)
    r = np.sqrt(((ii - 14.5) / 13.0) ** 2 + ((jj - 12.5) / 11.0) ** 2 + ((kk - 6.0) / 16.0) ** 2)
    outer, inner = r <= 1.0, r <= 0.62
    S = (outer & ~inner & (kk <= 19)).astype(np.uint8)
    cav = inner & (kk <= 19)
    ext = ~outer
    st = ndi.generate_binary_structure(3, 1)
    lab = np.zeros(n, np.int8)
    lab[(S == 1) & ndi.binary_dilation(ext, st)] = 1
    lab[(S == 1) & ndi.binary_dilation(cav, st)] = -1
    return S, lab


def transmural():
    hp = _refload.REF_ROOT / "hrdayapy"
    _refload._pkg("hrdayapy.coordinates", hp / "coordinates")
    _refload._pkg("hrdayapy.coordinates.functions", hp / "coordinates" / "functions")
    mod = _refload._load("hrdayapy.coordinates.functions.generate_transmural_coordinate",
                         hp / "coordinates" / "functions" / "generate_transmural_coordinate.py")
    S, lab = transmural_case()
    phi = quiet(mod.generate_transmural_coordinate, S, lab, device="cpu", tol=1e-8,
                maxiter=20000)
    np.savez_compressed(HERE / "transmural.npz", S=S, surface_label=lab, phi=phi)


def act_maps():
    """The upstream activation-map writer on upstream snapshots; keys are
    prefixed "slab_" (340 ms isotropic run, thresholds -20 / -60 mV) and
    "chatter_" (synthetic trace, debounce 3 ms, whose input is stored)."""
    nx, ny, nz = 16, 16, 4
    h, dt, T, vdt = 0.25, 0.02, 340.0, 0.5
    S = np.ones((nx, ny, nz), np.uint8)
    phi = np.ones(S.shape, np.float32)
    ect = np.zeros(S.shape, bool)
    ect[:4, :4, :] = True
    nodes, el, act = _stub(nx, ny, nz)
    prot = [dict(name="corner", target="ectopic", amp=0.52, dur=1.0, onset=0.0)]
    am = ref.activation_maps
    out = {}
    with tempfile.TemporaryDirectory() as td:
        vm_path = Path(td) / "vm.npz"
        quiet(ref.pipeline.run_coupled, nodes, el, act, S, S.copy(), phi,
              voxel_size=h, dx_p=0.25, sigma_P=0.0, sigma_M=0.13, Cm=0.01, A_P=133.33,
              A_M=140.0, R_P=0.015, dt=dt, T=T, theta=0.0, stim_protocol=prot,
              ectopic_region=ect, stim_len_mm=1.0, c_pmj=0.0, n_pmj=1,
              cg_tol=1e-12, cg_max_iter=200, n_frames=10, device="cpu",
              dtype=torch.float64, vm_save_dt=vdt, out_vm_npz=vm_path)
        snap = quiet(ref.load_vm_snapshots.load_vm_snapshots, vm_path)
        mp = Path(td) / "maps.npz"
        quiet(am.compute_activation_maps, snap, S, act_threshold=-20.0, deact_threshold=-60.0,
              save_path=mp)
        z = np.load(mp)
        out.update({"slab_" + k: z[k] for k in z.files if k != "source_vm_path"})
        # chattering synthetic trace: every crossing kept, then debounced
        rng = np.random.default_rng(11)
        t = np.arange(120, dtype=np.float32) * 0.5
        Vm = (-40.0 + 25.0 * np.sin(t[:, None] / 3.0 + rng.uniform(0, 6, 6)[None, :])
              + rng.normal(0, 6.0, (120, 6))).astype(np.float32)
        vs = ref.load_vm_snapshots.VmSnapshots(
            node_ids=np.arange(6, dtype=np.int32), coords_mm=rng.uniform(0, 5, (6, 3)).astype(np.float32),
            vox_idx=np.stack([np.arange(6), np.zeros(6, int), np.zeros(6, int)], 1).astype(np.int32),
            Vm=Vm, time_vm=t, dt_solver=0.5, vm_save_dt=0.5, path=Path("chatter.npz"))
        cp = Path(td) / "chatter.npz"
        quiet(am.compute_activation_maps, vs, None, act_threshold=-40.0, deact_threshold=-45.0,
              min_event_gap_ms=3.0, save_path=cp)
        z = np.load(cp)
        out.update({"chatter_" + k: z[k] for k in z.files if k != "source_vm_path"})
        out.update(chatter_in_Vm=Vm, chatter_in_t=t, chatter_in_coords=vs.coords_mm,
                   chatter_in_vox=vs.vox_idx)
    out.update(h=h, dt=dt, T=T, vm_save_dt=vdt)
    np.savez_compressed(HERE / "act_maps_iso.npz", **out)


PMJ_CASES = (  # (tag, direction, c_pmj, T)
    ("ortho", "orthodromic", 5.0, 80.0),
    ("ortho_block", "orthodromic", 1e-5, 40.0),
    ("anti", "antidromic", 5.0, 100.0))
PMJ_GRID = dict(dx_m=0.25, dx_p=0.25, dt=0.05, n_pmj=1)


def pmj_exp4():
    """Runs the upstream experiment core unchanged: its package imports are
    served by the upstream modules loaded by path."""
    import types
    hp = _refload.REF_ROOT / "hrdayapy"
    exp = _refload.REF_ROOT / "experiments" / "experiment_3"
    afn = sys.modules["hrdayapy.anisotropic_simulation.functions"]
    afn.purkinje_myocardium_anisotropic_solver = ref.aniso.purkinje_myocardium_anisotropic_solver
    afn.load_vm_snapshots = _refload._load(
        "hrdayapy.anisotropic_simulation.functions.load_vm_snapshots",
        hp / "anisotropic_simulation" / "functions" / "load_vm_snapshots.py").load_vm_snapshots
    afn.compute_activation_maps = _refload._load(
        "hrdayapy.anisotropic_simulation.functions.activation_maps",
        hp / "anisotropic_simulation" / "functions" / "activation_maps.py").compute_activation_maps
    _refload._load("hrdayapy._spacing_resolve", hp / "_spacing_resolve.py")
    coupled = _refload._load("hrdayapy.anisotropic_simulation.coupled",
                             hp / "anisotropic_simulation" / "coupled.py")
    sys.modules["hrdayapy.anisotropic_simulation"].compute_anisotropic_coupled = \
        coupled.compute_anisotropic_coupled
    sys.modules["hrdayapy.simulation.functions"].activation_maps = ref.activation_maps
    sys.path.insert(0, str(exp))
    ec = _refload._load("experiment_common", exp / "experiment_common.py")
    out = dict(PMJ_GRID)
    g = PMJ_GRID
    for tag, direction, c_pmj, T in PMJ_CASES:
        with tempfile.TemporaryDirectory() as td:
            r = quiet(ec.run_directional, ec.SIGMA_L, ec.SIGMA_T, ec.SIGMA_P, g["dt"], g["dx_p"],
                      g["dx_m"], T, tag, c_pmj, g["n_pmj"], direction, Path(td))
        for k in ("myo_act", "p_act", "p_arc_length", "pmj_junction_capture_fraction",
                  "pmj_propagating_capture", "pmj_n_myo_activated", "pmj_delay_ms",
                  "pmj_coupled_myo_idx"):
            out[f"{tag}_{k}"] = np.asarray(r[k])
        out[f"{tag}_T"] = T
        out[f"{tag}_c_pmj"] = c_pmj
    np.savez_compressed(HERE / "pmj_exp4.npz", **out)


if __name__ == "__main__":
    torch.set_num_threads(8)
    which = sys.argv[1:] or ["cells", "pacing", "iso", "aniso", "maps", "pmj", "torso", "bspm",
                             "transmural", "sbm"]
    for w in which:
        print("generating", w, flush=True)
        {"cells": ttp06_cells, "pacing": ttp06_pacing, "iso": mono_iso,
         "aniso": mono_aniso, "maps": act_maps, "pmj": pmj_exp4, "torso": torso,
         "bspm": bspm_loop, "transmural": transmural, "sbm": sbm}[w]()
