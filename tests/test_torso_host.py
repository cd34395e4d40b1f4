"""Host-side torso preparation against the oracle (CPU only)."""
import numpy as np

from hrdayapy_b200.ecg import torso as T
from hrdayapy_b200.ecg.torso_grid import torso_grid_from_labels
from oracle import torso as O
from tests import torso_cases


def test_heart_neighbours_match_graph_laplacian(golden):
    g = golden("torso.npz")
    vox = g["heart_vox"]
    nbr = T.heart_neighbours(vox)
    K = O.heart_laplacian(vox, len(vox))
    rng = np.random.default_rng(0)
    v = rng.normal(size=len(vox))
    lap = np.where(nbr >= 0, v[np.maximum(nbr, 0)] - v[:, None], 0.0).sum(1)
    np.testing.assert_allclose(lap, K @ v, atol=1e-12)


def test_grid_projection_surface_pin(golden):
    g = golden("torso.npz")
    lab, sigma_map, dx, vox, coords, reg, h, Vm = torso_cases.golden_case(g)
    grid = torso_grid_from_labels(lab, sigma_map, dx)
    assert grid["pin_row"] == int(g["pin_row"])
    np.testing.assert_array_equal(grid["surface_rows"], g["surf_rows"])
    proj, valid = T.projection_map(coords, reg["R"], reg["t"], 1.0, grid["origin_mm"], dx,
                                   grid["active_id_map"], grid["shape"])
    np.testing.assert_array_equal(proj, g["proj"])
    # labels -> operator: the label table reproduces the assembled stiffness
    labels, table = T.labels_from_grid(grid)
    sig = table[labels]
    A, flat, _ = O.assemble_stiffness(sig, dx * 1e-3, labels != 0)
    import scipy.sparse as sp
    Aref = sp.csr_matrix((g["A_data"], g["A_indices"], g["A_indptr"]), shape=A.shape)
    assert abs(A - Aref).max() <= 1e-12 * abs(Aref).max()


def test_labels_from_reference_grid():
    lab, sigma_map, *_ = torso_cases.random_case()
    grid = torso_grid_from_labels(lab, sigma_map, 1.5)
    ref_like = dict(sigma_vol=grid["sigma_vol"], active_mask=grid["active_mask"])
    l2, t2 = T.labels_from_grid(ref_like)
    np.testing.assert_allclose(t2[l2], grid["sigma_vol"])


def test_twelve_lead_definitions():
    e = np.arange(10.0)[:, None] * np.ones((1, 3))
    L = T.twelve_lead(e)
    RA, LA, LL = 0.0, 1.0, 3.0
    assert np.allclose(L[0], LA - RA) and np.allclose(L[1], LL - RA) and np.allclose(L[2], LL - LA)
    assert np.allclose(L[0] + L[2], L[1])                      # Einthoven
    assert np.allclose(L[3] + L[4] + L[5], 0.0)                # augmented leads sum to zero
    assert np.allclose(L[6], 4.0 - (RA + LA + LL) / 3)


def test_fp64_pcg_oracle_matches_direct_solve():
    """The threaded FP64 Jacobi-CG of the oracle (the reference's _pcg_gpu
    in FP64 with a relative true-residual stop) reaches the direct solve of
    the pinned system, from zero and from a perturbed warm start; the CSR
    pinning equals the reference's LIL pinning."""
    lab, sigma_map, dx, vox, coords, reg, h, frames = torso_cases.random_case(shape=(24, 20, 28))
    grid = torso_grid_from_labels(lab, sigma_map, dx)
    A, _, _ = O.assemble_stiffness(grid["sigma_vol"], dx * 1e-3, grid["active_mask"])
    pin = grid["pin_row"]
    Ap = O.pinned_csr(A, pin)
    assert abs(Ap - O.pinned(A, pin).tocsr()).max() == 0.0
    proj, valid = T.projection_map(coords, reg["R"], reg["t"], 1.0, grid["origin_mm"], dx,
                                   grid["active_id_map"], grid["shape"])
    K = O.heart_laplacian(vox, len(vox))
    b = O.frame_rhs(K, frames[1], proj.astype(np.int64), valid, A.shape[0], pin, 0.2625,
                    h * 1e-3, dx)
    xd = O.Solver(A, pin).solve(b)
    for x0 in (None, xd * (1.0 + 1e-3 * np.sin(np.arange(len(xd))))):
        x, it, rel, rst = O.pcg_fp64(Ap, b, x0, tol=1e-11)
        assert rel <= 1e-11 and it > 0
        assert np.linalg.norm(Ap @ x - b) <= 1e-11 * np.linalg.norm(b) * 1.0001
        assert np.linalg.norm(x - xd) <= 1e-7 * np.linalg.norm(xd)
