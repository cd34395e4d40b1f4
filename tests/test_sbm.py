"""Smoothed boundary method (use_sbm=True) on the host: the domain function
psi, the band and its materials, rows, pin and surface nodes, and the
oracle's smoothed-boundary stiffness, against the upstream functions' own
outputs on a small fine segmentation (tests/golden/sbm.npz, made by
tests/golden/make_golden.py from build_torso_grid.py:130-206, :260-386 and
make_gpu_solver's psi-weighted solve, compute_bspm.py:280-440)."""
import numpy as np
import pytest
import scipy.sparse as sp


def _grid(g):
    from hrdayapy_b200.ecg.torso_grid import torso_grid_from_labels
    sig_map = dict(zip(g["sigma_keys"].tolist(), g["sigma_vals"].tolist()))
    return torso_grid_from_labels(g["coarse"], sig_map, float(g["dx"]), psi_vol=g["psi"]), sig_map


def test_domain_function_and_resampling_match_upstream(golden):
    from hrdayapy_b200.ecg.torso_grid import _resample_labels, smoothed_domain
    g = golden("sbm.npz")
    coarse = _resample_labels(g["fine"], g["spacing"], float(g["dx"]))
    np.testing.assert_array_equal(coarse, g["coarse"])
    psi = smoothed_domain(g["fine"], g["spacing"], float(g["dx"]), coarse.shape)
    np.testing.assert_allclose(psi, g["psi"], rtol=0, atol=1e-15)
    assert (psi[coarse != 0] > 0).all()


def test_band_rows_pin_surface_and_sigma_match_upstream(golden):
    g = golden("sbm.npz")
    grid, _ = _grid(g)
    assert grid["use_sbm"]
    np.testing.assert_array_equal(grid["active_ids"], g["active_ids"])
    assert grid["pin_row"] == int(g["pin_row"])
    np.testing.assert_array_equal(grid["surface_flat"], g["surf_flat"])
    np.testing.assert_array_equal(grid["surface_rows"], g["surf_rows"])
    act = grid["active_mask"]
    np.testing.assert_array_equal(grid["sigma_vol"][act], g["sigma_ext"][act])
    # every system cell has a material, nothing outside the system has one
    assert (grid["labels"][act] > 0).all() and (grid["labels"][~act] == 0).all()


def test_compute_torso_grid_from_fine_labels(golden):
    from hrdayapy_b200.ecg.torso_grid import compute_torso_grid
    g = golden("sbm.npz")
    sig_map = dict(zip(g["sigma_keys"].tolist(), g["sigma_vals"].tolist()))
    grid = compute_torso_grid(sigma_map=sig_map, labels=g["fine"], spacing_mm=g["spacing"],
                              dx_coarse_mm=float(g["dx"]), use_sbm=True, verbose=False)
    np.testing.assert_array_equal(grid["active_ids"], g["active_ids"])
    np.testing.assert_allclose(grid["psi_vol"], g["psi"], rtol=0, atol=1e-15)
    sharp = compute_torso_grid(sigma_map=sig_map, labels=g["fine"], spacing_mm=g["spacing"],
                               dx_coarse_mm=float(g["dx"]), verbose=False)
    assert not sharp["use_sbm"] and "psi_vol" not in sharp
    np.testing.assert_array_equal(sharp["active_mask"], g["coarse"] != 0)


def test_sbm_needs_the_fine_segmentation():
    from hrdayapy_b200.ecg.torso_grid import compute_torso_grid
    with pytest.raises(ValueError, match="fine segmentation"):
        compute_torso_grid(sigma_map={1: 0.2}, labels=np.ones((4, 4, 4), np.int32),
                           use_sbm=True, verbose=False)


def test_saved_grid_round_trip(golden, tmp_path):
    from hrdayapy_b200.ecg.torso_grid import load_torso_grid, torso_grid_from_labels
    g = golden("sbm.npz")
    sig_map = dict(zip(g["sigma_keys"].tolist(), g["sigma_vals"].tolist()))
    torso_grid_from_labels(g["coarse"], sig_map, float(g["dx"]), psi_vol=g["psi"],
                           save_path=tmp_path / "grid.npz")
    back = load_torso_grid(tmp_path / "grid.npz")
    assert back["use_sbm"]
    np.testing.assert_allclose(back["psi_vol"], g["psi"].astype(np.float32))


def test_oracle_sbm_stiffness_matches_upstream(golden):
    from oracle import torso as orc
    g = golden("sbm.npz")
    act = g["psi"] > 0
    A, flat, _ = orc.assemble_stiffness(g["sigma_ext"], float(g["dx"]) * 1e-3, act,
                                        psi_vol=g["psi"])
    np.testing.assert_array_equal(flat, g["active_ids"])
    ref = sp.csr_matrix((g["A_data"], g["A_indices"], g["A_indptr"]), shape=A.shape)
    d = (A - ref).tocsr()
    assert abs(d).max() <= 1e-12 * abs(ref).max()
    assert A.nnz == ref.nnz


def test_oracle_sbm_solution_matches_upstream(golden):
    """The oracle's FP64 direct solve of the pinned smoothed-boundary system
    with the psi-weighted right-hand side reproduces the upstream solver's
    surface potentials (upstream iterated to 1e-7 mV, linf)."""
    from oracle import torso as orc
    g = golden("sbm.npz")
    act = g["psi"] > 0
    dx = float(g["dx"])
    A, flat, id_map = orc.assemble_stiffness(g["sigma_ext"], dx * 1e-3, act, psi_vol=g["psi"])
    K = orc.heart_laplacian(g["heart_vox"], len(g["heart_vox"]))
    psi_row = g["psi"].ravel()[flat]
    b = orc.frame_rhs(K, g["Vm"], g["proj"], g["valid"], len(flat), int(g["pin_row"]), 0.2625,
                      float(g["h_fine"]) * 1e-3, dx, psi_row=psi_row)
    x = orc.Solver(A, int(g["pin_row"])).solve(b)
    ref = g["phi_surf_ref"].astype(np.float64)
    err = np.linalg.norm(x[g["surf_rows"]] - ref) / np.linalg.norm(ref)
    assert err <= 1e-5, err
