"""The allocation-free residual check, through the C ABI.

hp_torso_residual_noalloc serves callers that may not allocate device
memory (a host framework that owns all allocations, a real-time loop, a
fixed memory budget): it must return the same FP64 true residual that the
allocating solver reports for the same x and b.  Collected last on purpose
(file name), and run both alone in a fresh process and after the other
tests."""
import ctypes as C

import numpy as np
import pytest

from tests import torso_cases

pytestmark = pytest.mark.gpu


def _padded(grid, labels, x_rows, b_rows):
    ni, nj, nk = grid["shape"]
    lab = np.zeros((ni + 2, nj + 2, nk + 2), np.uint8)
    lab[1:-1, 1:-1, 1:-1] = labels
    flat = np.asarray(grid["active_ids"], np.int64)
    i, j, k = np.unravel_index(flat, (ni, nj, nk))
    cell = ((i + 1) * (nj + 2) + (j + 1)) * (nk + 2) + (k + 1)
    x = np.zeros(lab.size)
    b = np.zeros(lab.size, np.float32)
    x[cell] = x_rows
    b[cell] = b_rows
    return lab, x, b, int(cell[grid["pin_row"]])


def _noalloc(grid, table, lab, x, b, pin):
    import torch
    from hrdayapy_b200 import _lib
    dev = torch.device("cuda")
    lab_d = torch.from_numpy(lab.ravel()).to(dev)
    x_d = torch.from_numpy(x).to(dev)
    b_d = torch.from_numpy(b).to(dev)
    sig = np.ascontiguousarray(table, np.float64)
    out = np.zeros(2)
    ni, nj, nk = grid["shape"]
    st = _lib.lib().hp_torso_residual_noalloc(
        ni, nj, nk, C.c_void_p(lab_d.data_ptr()), _lib.ptr(sig), len(sig),
        float(grid["dx_mm"]) * 1e-3, pin, C.c_void_p(x_d.data_ptr()),
        C.c_void_p(b_d.data_ptr()), _lib.ptr(out), None)
    return st, out


def test_noalloc_residual_matches_solver():
    from hrdayapy_b200.ecg import torso as T
    from hrdayapy_b200.ecg.torso_grid import torso_grid_from_labels
    from hrdayapy_b200 import _lib
    lab0, sigma_map, dx, vox, coords, reg, h, frames = torso_cases.random_case(seed=5)
    grid = torso_grid_from_labels(lab0, sigma_map, dx)
    labels, table = T.labels_from_grid(grid)
    proj, _ = T.projection_map(coords, reg["R"], reg["t"], 1.0, grid["origin_mm"], dx,
                               grid["active_id_map"], grid["shape"])
    solver = T.TorsoSolver(labels, table, dx, grid["pin_row"], T.heart_neighbours(vox), proj,
                           0.2625, h, grid["surface_rows"])
    try:
        # two calls in a row, each after a fresh frame solve
        for f in (0, 1):
            _, stats = solver.solve_frame(frames[f], 1e-6, "rel", 5000)
            x, b = solver.solution(), solver.rhs()
            lab, xp, bp, pin = _padded(grid, labels, x, b)
            st, out = _noalloc(grid, table, lab, xp, bp, pin)
            _lib.check(st, "hp_torso_residual_noalloc")
            rel = out[0] / out[1]
            assert stats.rel_residual > 0.0
            assert abs(rel - stats.rel_residual) <= 1e-9 * stats.rel_residual, (rel, stats.rel_residual)
            assert abs(out[1] - np.linalg.norm(b.astype(np.float64))) <= 1e-12 * out[1]
    finally:
        solver.close()


def test_noalloc_rejects_oversized_grid():
    from hrdayapy_b200 import _lib
    L = _lib.lib()
    out = np.zeros(2)
    sig = np.array([0.0, 0.2])
    # 1024 x 1024 x 1024 padded cells is above the fixed scratch capacity
    st = L.hp_torso_residual_noalloc(1022, 1022, 1022, C.c_void_p(16), _lib.ptr(sig), 2, 1e-3,
                                     -1, C.c_void_p(16), C.c_void_p(16), _lib.ptr(out), None)
    assert st == 1
    assert b"exceeds the maximum" in L.hp_last_error()


def test_noalloc_rejects_tissue_on_the_border():
    """The padded grid's one-voxel border must be air: a conductive border
    cell would act as a neighbour the solver's operator does not have."""
    import torch
    from hrdayapy_b200 import _lib
    L = _lib.lib()
    ni, nj, nk = 6, 5, 4
    lab = np.zeros((ni + 2, nj + 2, nk + 2), np.uint8)
    lab[1:-1, 1:-1, 1:-1] = 1
    lab[0, 3, 2] = 1                       # tissue on the border
    dev = torch.device("cuda")
    lab_d = torch.from_numpy(lab.ravel()).to(dev)
    x_d = torch.zeros(lab.size, dtype=torch.float64, device=dev)
    b_d = torch.ones(lab.size, dtype=torch.float32, device=dev)
    sig = np.array([0.0, 0.2])
    out = np.zeros(2)
    st = L.hp_torso_residual_noalloc(ni, nj, nk, C.c_void_p(lab_d.data_ptr()), _lib.ptr(sig), 2,
                                     1e-3, -1, C.c_void_p(x_d.data_ptr()),
                                     C.c_void_p(b_d.data_ptr()), _lib.ptr(out), None)
    assert st == 1
    assert b"border" in L.hp_last_error()
