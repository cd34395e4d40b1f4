"""The ECG half of the drop-in, end to end through the public API:
compute_coupled writes vm_snapshots.npz, compute_bspm reads it, solves every
frame on the GPU and writes bspm.npz.  Both files are checked against the
ones the upstream code writes for the same inputs (tests/golden/bspm_loop.npz:
upstream run_coupled and run_bspm_loop, ecg/functions/compute_bspm.py:445-670,
schema :651-664) -- same keys, dtypes, shapes and metadata, potentials within
tolerance -- and the potentials against the oracle's FP64 direct solve of the
reference operator.

Tolerance: relative L2 <= 1e-3 of the body-surface potentials with each
frame's surface mean removed.  An FP32 right-hand side (the reference's and
ours) carries a rounding-size net source that the pinned Neumann system
turns into a near-uniform offset, different for each FP32 evaluation order;
the ECG (differences of potentials) does not see it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bspm_case():
    """The inputs of tests/golden/make_golden.py:bspm_case."""
    nx, ny, nz = 24, 24, 8
    S = np.ones((nx, ny, nz), np.uint8)
    phi = np.ones(S.shape, np.float32)
    ect = np.zeros(S.shape, bool)
    ect[:4, :4, :] = True
    nodes = np.array([[ny + 8.0, nx + 8.0, nz + 8.0], [ny + 8.0, nx + 8.0, nz + 12.0]])
    el, act = np.array([[0, 1]]), np.array([0.0, 1.0])
    kw = dict(voxel_size=0.5, dx_p=0.25, sigma_P=0.0, sigma_M=0.13, Cm=0.01, A_P=133.33,
              A_M=140.0, R_P=0.015, dt=0.02, T=12.0, theta=0.0,
              stim_protocol=[dict(name="corner", target="ectopic", amp=0.52, dur=1.0,
                                  onset=0.0)],
              ectopic_region=ect, stim_len_mm=1.0, c_pmj=0.0, n_pmj=1)
    reg = dict(R=np.eye(3), t=np.array([9.75, 7.5, 16.0]), scale=1.0, dice=0.9)
    return (nodes, el, act, S, phi), kw, reg


def _offset_free_rel(a, b):
    a = a - a.mean(axis=0, keepdims=True)
    b = b - b.mean(axis=0, keepdims=True)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _schema(z):
    return [(k, str(z[k].dtype), z[k].shape) for k in sorted(z.files)]


def test_compute_bspm_end_to_end_vs_upstream(golden, tmp_path):
    from hrdayapy_b200.ecg import compute_bspm, load_bspm
    from hrdayapy_b200.ecg.torso_grid import torso_grid_from_labels
    from hrdayapy_b200.simulation import compute_coupled
    from oracle import torso as O
    g = golden("bspm_loop.npz")
    (nodes, el, act, S, phi), kw, reg = bspm_case()
    vm_path = tmp_path / "vm_snapshots.npz"
    compute_coupled(nodes, el, act, S, S, phi, vm_save_dt=1.0, vm_save_path=vm_path, **kw)

    # the snapshot file: the upstream writer's schema, potentials within 0.5 mV RMS
    z = np.load(vm_path)
    assert sorted(z.files) == list(g["vm_keys"])
    assert [str(z[k].dtype) for k in sorted(z.files)] == list(g["vm_dtypes"])
    for k in ("node_ids", "vox_idx", "coords_mm", "time_vm", "dt_solver", "vm_save_dt"):
        np.testing.assert_array_equal(z[k], g[f"vm_{k}"])
    assert z["Vm"].shape == g["vm_Vm"].shape
    assert float(np.sqrt(np.mean((z["Vm"].astype(np.float64) - g["vm_Vm"]) ** 2))) <= 0.5

    sig_map = {int(k): float(v) for k, v in zip(g["sigma_keys"], g["sigma_vals"])}
    grid = torso_grid_from_labels(g["labels"], sig_map, float(g["dx"]))
    out_path = tmp_path / "bspm.npz"
    bspm = compute_bspm(vm_path, grid, reg, sigma_i=0.2625, h_fine_mm=0.5, cg_tol_mV=1e-6,
                        cg_max_iter=5000, cg_metric="rms", verbose=False, save_path=out_path)
    ours = load_bspm(out_path)
    up = {k: g[f"out_{k}"] for k in g["out_keys"]}
    # the bspm.npz schema of the reference writer: keys, dtypes, shapes
    zo = np.load(out_path)
    assert [(k, d) for k, d, _ in _schema(zo)] == list(zip(g["out_keys"], g["out_dtypes"]))
    for k in up:
        assert ours[k].shape == up[k].shape, k
    for k in ("surface_flat", "time_ms", "reg_R", "reg_t", "reg_scale", "reg_dice", "sigma_i",
              "h_fine_mm", "dx_mm"):
        np.testing.assert_array_equal(ours[k], up[k], err_msg=k)
    np.testing.assert_allclose(ours["surface_xyz"], up["surface_xyz"], rtol=0, atol=1e-5)
    np.testing.assert_array_equal(ours["bspm_signal"], bspm)

    # potentials: against the upstream FP32 loop and the FP64 direct solve
    rel_up = _offset_free_rel(bspm.astype(np.float64), up["bspm_signal"].astype(np.float64))
    A, _, _ = O.assemble_stiffness(grid["sigma_vol"], float(g["dx"]) * 1e-3, grid["active_mask"])
    K = O.heart_laplacian(z["vox_idx"], len(z["vox_idx"]))
    proj, valid = O.projection_map(z["coords_mm"].astype(np.float64), reg["R"], reg["t"], 1.0,
                                   grid["origin_mm"], float(g["dx"]), grid["active_id_map"],
                                   grid["shape"])
    solver = O.Solver(A, grid["pin_row"])
    phi = np.stack([solver.solve(O.frame_rhs(K, vm, proj, valid, A.shape[0], grid["pin_row"],
                                             0.2625, 0.5e-3, float(g["dx"])))
                    for vm in z["Vm"]], 1)
    ref64 = phi[grid["surface_rows"]] * 1e3
    rel64 = _offset_free_rel(bspm.astype(np.float64), ref64)
    rel_up64 = _offset_free_rel(up["bspm_signal"].astype(np.float64), ref64)
    print(f"bspm end to end: {bspm.shape}, offset-free rel. L2 vs upstream {rel_up:.2e}, "
          f"vs FP64 {rel64:.2e} (upstream vs FP64 {rel_up64:.2e})")
    assert rel_up <= 1e-3
    assert rel64 <= 1e-3
