"""Learned preconditioner: the tcgen05 forward and the hand-written backward
against torch autograd on the CPU (the oracle for this part), then on-GPU
training and flexible CG on held-out frames."""
import ctypes as C

import numpy as np
import pytest

from tests import precond_ref as R
from tests import torso_cases

pytestmark = pytest.mark.gpu


def _small(seed=2, shape=(16, 16, 256)):
    from hrdayapy_b200.ecg import torso as T
    from hrdayapy_b200.ecg.torso_grid import torso_grid_from_labels
    lab0, sigma_map, dx, vox, coords, reg, h, frames = torso_cases.random_case(seed=seed, shape=shape)
    grid = torso_grid_from_labels(lab0, sigma_map, dx)
    labels, table = T.labels_from_grid(grid)
    proj, _ = T.projection_map(coords, reg["R"], reg["t"], 1.0, grid["origin_mm"], dx,
                               grid["active_id_map"], grid["shape"])
    solver = T.TorsoSolver(labels, table, dx, grid["pin_row"], T.heart_neighbours(vox), proj,
                           0.2625, h, grid["surface_rows"])
    return solver, grid, labels, table, dx, frames


def _cos(a, b):
    return float(np.dot(a, b) / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30))


def test_forward_and_gradients_vs_torch():
    import torch
    from hrdayapy_b200.ecg.precond import LearnedPreconditioner, param_offsets, LAYERS
    solver, grid, labels, table, dx, frames = _small()
    pc = LearnedPreconditioner(solver, labels, len(table), omega=0.6, seed=3)
    try:
        arr = pc.arrays
        ng = arr.n_cells
        rng = np.random.default_rng(0)
        act = np.zeros(ng, bool)
        lab_p = np.zeros((arr.ni + 2, arr.nj + 2, arr.nk + 2), np.uint8)
        lab_p[1:-1, 1:-1, 1:-1] = labels
        act[:] = lab_p.ravel() != 0
        act[arr.pin_cell] = False
        r = (rng.normal(size=ng) * act).astype(np.float32) * 1e3
        e = (rng.normal(size=ng) * act).astype(np.float32) * 1e-4
        rd = torch.from_numpy(r).cuda()
        ed = torch.from_numpy(e).cuda()
        loss_gpu = pc.train_step(rd.data_ptr(), ed.data_ptr(), lr=0.0)
        y_gpu, s_gpu, err = pc.output()
        assert err == 0
        params, grads = pc.params()
        invd = R.invd_from_labels(labels, table, dx * 1e-3, arr.pin_cell)
        feat, s_ref = R.features(r.astype(np.float64), invd, labels, arr.pin_cell, len(table))
        assert abs(s_gpu - s_ref) <= 1e-4 * s_ref
        y_ref, P = R.net(feat, params, requires_grad=True)
        L = R.loss(y_ref, s_ref, r, invd, e, labels, arr.pin_cell, 0.6)
        L.backward()
        g_ref = P.grad.numpy()
        yr = y_ref.detach().numpy()
        assert np.linalg.norm(y_gpu - yr) <= 3e-2 * np.linalg.norm(yr)
        assert abs(loss_gpu - float(L)) <= 3e-2 * float(L)
        offs, n = param_offsets()
        for (ow, ob), name, co in zip(offs, LAYERS, R.LCOUT):
            gw, gr = grads[ow:ob], g_ref[ow:ob]
            assert _cos(gw, gr) >= 0.99, (name, _cos(gw, gr))
            assert np.linalg.norm(gw - gr) <= 0.1 * np.linalg.norm(gr), name
            gb, gbr = grads[ob:ob + co], g_ref[ob:ob + co]
            assert np.linalg.norm(gb - gbr) <= 0.1 * np.linalg.norm(gbr) + 1e-12, name
    finally:
        pc.close()
        solver.close()


def test_training_and_fcg_on_held_out_frames():
    """Train on the plain solver's residual/error pairs of the first frames,
    then solve later frames with flexible CG: converged to the FP64 true
    residual <= 1e-6, and fewer iterations than plain Jacobi-PCG."""
    import torch
    from hrdayapy_b200.ecg.precond import LearnedPreconditioner
    solver, grid, labels, table, dx, frames = _small(seed=4, shape=(24, 24, 256))
    pc = LearnedPreconditioner(solver, labels, len(table), omega=0.6, seed=5)
    try:
        # more frames by interpolating the wavefront frames
        fr = np.concatenate([frames, frames[::-1]]).astype(np.float32)
        vm = torch.from_numpy(fr).cuda().contiguous()
        hist = pc.train(vm[:6], ks=(0, 4, 16, 48), repeats=4, lr=2e-3)
        assert np.all(np.isfinite(hist))
        assert hist[-8:].mean() < hist[:8].mean()       # training lowers the loss
        plain, learned = [], []
        for f in range(6, len(fr)):
            solver.reset()
            solver.solve_frame(fr[f - 1], 1e-6, "rel", 20000)
            _, sp = solver.solve_frame(fr[f], 1e-6, "rel", 20000)
            plain.append(sp.iterations)
            solver.reset()
            solver.solve_frame(fr[f - 1], 1e-6, "rel", 20000)
            _, sl = pc.solve_frame(fr[f], 1e-6, 20000, 400)
            assert sl.rel_residual <= 1e-6 and sl.status == 0
            learned.append(sl.iterations)
        assert np.mean(learned) < np.mean(plain), (learned, plain)
    finally:
        pc.close()
        solver.close()
