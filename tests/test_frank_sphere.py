"""Known-answer test of the ECG operator: a current dipole at the centre of a
homogeneous, insulated sphere, against Frank's closed-form potential (Frank,
J. Appl. Phys. 23, 1225, 1952), as the reference's validation experiment
does (experiments/experiment_4/sphere_dipole_validation.py:135-217,
:428-438): sphere radius 100 mm, grid 2 mm, sigma 0.2 S/m, dipole
separation 4 mm; surface potentials gauge-aligned at the equator; pass if
the relative difference measure (RDM) is below 0.05.

The dipole is driven through the solver's own source path: a "heart" of
two graph-neighbour voxels 4 mm apart at -V and +V mV has a source
Laplacian of +S and -S, which the projection puts on the two torso rows
on the dipole axis.  The dipole moment is read back from the solver's
right-hand side."""
import numpy as np
import pytest

R_MM, DX_MM, SIGMA, D_MM = 100.0, 2.0, 0.2, 4.0


def _sphere_grid():
    from hrdayapy_b200.ecg.torso_grid import torso_grid_from_labels
    n = int(np.ceil(2 * R_MM * 1.3 / DX_MM))
    n += n % 2 == 0
    c = (n - 1) / 2
    ii, jj, kk = np.indices((n, n, n)).astype(np.float64)
    r = DX_MM * np.sqrt((ii - c) ** 2 + (jj - c) ** 2 + (kk - c) ** 2)
    origin = -np.full(3, c * DX_MM)
    return torso_grid_from_labels((r <= R_MM).astype(np.int32), {1: SIGMA}, DX_MM,
                                  origin_mm=origin), (n - 1) // 2


def _frank(p_vec, xyz_mm):
    """Frank's potential of a dipole p (A m) at the centre of the sphere."""
    p = np.linalg.norm(p_vec)
    r_mm = np.linalg.norm(xyz_mm, axis=1)
    cos_t = (xyz_mm @ (p_vec / p)) / np.clip(r_mm, 1e-12, None)
    r_m, R_m = r_mm * 1e-3, R_MM * 1e-3
    return p / (4 * np.pi * SIGMA) * (cos_t / r_m ** 2 + 2 * r_m * cos_t / R_m ** 3)


def _rdm(grid, x, b):
    """Surface RDM against Frank for the solution x of the right-hand side b
    (per row), both gauge-aligned at the surface node nearest the equator."""
    h_m = DX_MM * 1e-3
    xyz_rows = np.asarray(grid["active_ids"])
    ijk = np.stack(np.unravel_index(xyz_rows, grid["shape"]), 1) * DX_MM + grid["origin_mm"]
    p_vec = (b[:, None] * h_m ** 3 * ijk * 1e-3).sum(0)      # sum of I_q r_q
    rows = np.asarray(grid["surface_rows"])
    sx = np.asarray(grid["surface_xyz"], np.float64)
    ref = int(np.argmin(np.linalg.norm(sx - np.array([R_MM, 0.0, 0.0]), axis=1)))
    num = x[rows] - x[rows[ref]]
    ana = _frank(p_vec, sx)
    ana = ana - ana[ref]
    return float(np.linalg.norm(num - ana) / np.linalg.norm(ana)), p_vec


def _dipole_rhs(grid, c):
    """+1 / -1 A point sources at the rows 2 mm above and below the centre."""
    n = grid["shape"][0]
    h_m = DX_MM * 1e-3
    b = np.zeros(len(grid["active_ids"]))
    idm = np.asarray(grid["active_id_map"])
    b[idm[(c * n + c) * n + c + 1]] = 1.0 / h_m ** 3
    b[idm[(c * n + c) * n + c - 1]] = -1.0 / h_m ** 3
    return b


def test_oracle_operator_matches_frank():
    from oracle import torso as O
    grid, c = _sphere_grid()
    A, flat, _ = O.assemble_stiffness(grid["sigma_vol"], DX_MM * 1e-3, grid["active_mask"])
    b = _dipole_rhs(grid, c)
    b[grid["pin_row"]] = 0.0
    x = O.pcg_fp64(O.pinned_csr(A, grid["pin_row"]), b, tol=1e-10)[0]
    rdm, p_vec = _rdm(grid, x, b)
    assert abs(np.linalg.norm(p_vec) - D_MM * 1e-3) < 1e-9     # p = I d = 1 A x 4 mm
    assert rdm < 0.05, rdm


@pytest.mark.gpu
def test_gpu_solver_matches_frank_and_fp64():
    from hrdayapy_b200.ecg import torso as T
    from oracle import torso as O
    grid, c = _sphere_grid()
    labels, table = T.labels_from_grid(grid)
    h_fine = 2 * DX_MM                       # the two heart voxels are 4 mm apart
    vox = np.array([[0, 0, 0], [0, 0, 1]], np.int32)
    coords = vox[:, [1, 0, 2]].astype(np.float64) * h_fine
    t = grid["origin_mm"] + DX_MM * np.array([c + 0.5, c + 0.5, c - 0.5])
    proj, valid = T.projection_map(coords, np.eye(3), t, 1.0, grid["origin_mm"], DX_MM,
                                   grid["active_id_map"], grid["shape"])
    assert valid.all()
    rows = np.arange(len(grid["active_ids"]))
    solver = T.TorsoSolver(labels, table, DX_MM, grid["pin_row"], T.heart_neighbours(vox),
                           proj, 0.2625, h_fine, rows)
    try:
        _, st = solver.solve_frame(np.array([-10.0, 10.0], np.float32), 1e-8, "rel", 20000)
        assert st.status == 0 and st.rel_residual <= 1e-8
        x = solver.solution()
        b = solver.rhs().astype(np.float64)
    finally:
        solver.close()
    nz = np.nonzero(b)[0]
    assert len(nz) == 2 and abs(b[nz].sum()) <= 1e-6 * abs(b[nz]).max()   # a pure dipole
    rdm, p_vec = _rdm(grid, x, b)
    assert abs(p_vec[0]) + abs(p_vec[1]) <= 1e-9 * np.linalg.norm(p_vec)   # along the k axis
    assert rdm < 0.05, rdm
    # and the same field as the FP64 solve of the same right-hand side
    A, flat, _ = O.assemble_stiffness(grid["sigma_vol"], DX_MM * 1e-3, grid["active_mask"])
    xo = O.pcg_fp64(O.pinned_csr(A, grid["pin_row"]), b, tol=1e-10)[0]
    s = np.asarray(grid["surface_rows"])
    assert np.linalg.norm(x[s] - xo[s]) <= 1e-5 * np.linalg.norm(xo[s])
