"""Learned preconditioner: the tcgen05 forward and the hand-written backward
against torch autograd on the CPU (the oracle for this part), then on-GPU
training and flexible CG on held-out frames."""
import ctypes as C

import numpy as np
import pytest

from tests import precond_ref as R
from tests import torso_cases

pytestmark = pytest.mark.gpu


def _small(seed=2, shape=(24, 24, 256)):
    from hrdayapy_b200.ecg import torso as T
    from hrdayapy_b200.ecg.torso_grid import torso_grid_from_labels
    lab0, sigma_map, dx, vox, coords, reg, h, frames = torso_cases.random_case(seed=seed, shape=shape)
    grid = torso_grid_from_labels(lab0, sigma_map, dx)
    labels, table = T.labels_from_grid(grid)
    proj, _ = T.projection_map(coords, reg["R"], reg["t"], 1.0, grid["origin_mm"], dx,
                               grid["active_id_map"], grid["shape"])
    solver = T.TorsoSolver(labels, table, dx, grid["pin_row"], T.heart_neighbours(vox), proj,
                           0.2625, h, grid["surface_rows"])
    return solver, grid, labels, table, dx, vox


def _wave_frames(vox, n, seed):
    """Seeded activation-front frames (mV) sweeping across the heart voxels."""
    rng = np.random.default_rng(seed)
    x = vox[:, 0].astype(np.float64) + 0.4 * vox[:, 2]
    lo, hi = x.min(), x.max()
    out = []
    for f in range(n):
        front = lo + (hi - lo) * (f + 0.5) / n
        out.append(-85.0 + 110.0 / (1.0 + np.exp(-(front - x) / 1.5)) + rng.normal(0, 0.3, len(x)))
    return np.array(out, np.float32)


def _cos(a, b):
    return float(np.dot(a, b) / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30))


def test_forward_and_gradients_vs_torch():
    import torch
    from hrdayapy_b200.ecg.precond import LearnedPreconditioner, param_offsets, LAYERS
    solver, grid, labels, table, dx, vox = _small(shape=(16, 16, 256))
    pc = LearnedPreconditioner(solver, labels, len(table), omega=0.6, seed=3, coarse_agg=-1,
                               zero_output=False)
    try:
        arr = pc.arrays
        ng = arr.n_cells
        rng = np.random.default_rng(0)
        act = np.zeros(ng, bool)
        lab_p = np.zeros((arr.ni + 2, arr.nj + 2, arr.nk + 2), np.uint8)
        lab_p[1:-1, 1:-1, 1:-1] = labels
        act[:] = lab_p.ravel() != 0
        act[arr.pin_cell] = False
        invd = R.invd_from_labels(labels, table, dx * 1e-3, arr.pin_cell)
        r = (rng.normal(size=ng) * act).astype(np.float32) * 1e3
        # an error field correlated with D^-1 r, so that r.e > 0 as for a true pair
        e = ((invd * r + 1e-4 * rng.normal(size=ng)) * act).astype(np.float32)
        rd = torch.from_numpy(r).cuda()
        ed = torch.from_numpy(e).cuda()
        loss_gpu = pc.train_step(rd.data_ptr(), ed.data_ptr(), lr=0.0)
        y_gpu, s_gpu, err = pc.output()
        assert err == 0
        params, grads = pc.params()
        feat, s_ref = R.features(r.astype(np.float64), invd, labels, arr.pin_cell, len(table))
        assert abs(s_gpu - s_ref) <= 1e-4 * s_ref
        y_ref, P = R.net(feat, params, requires_grad=True)
        L = R.loss(y_ref, s_ref, r, invd, e, labels, table, dx * 1e-3, arr.pin_cell, 0.6)
        L.backward()
        g_ref = P.grad.numpy()
        yr = y_ref.detach().numpy()
        assert np.linalg.norm(y_gpu - yr) <= 3e-2 * np.linalg.norm(yr)
        assert abs(loss_gpu - float(L)) <= 3e-2 * abs(float(L)) + 1e-6
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


def test_coarse_level_vs_numpy():
    """Without the network M(r) = omega D^-1 r + Q A_c^-1 Q^T r: the GPU
    application against an FP64 numpy Galerkin solve of the same aggregates."""
    import torch
    from hrdayapy_b200.ecg.precond import LearnedPreconditioner
    solver, grid, labels, table, dx, vox = _small(seed=3)
    pc = LearnedPreconditioner(solver, labels, len(table), omega=0.6, seed=1)
    try:
        ag, nc = pc.coarse_info()
        assert ag >= 4 and 0 < nc <= 2048
        arr = pc.arrays
        rng = np.random.default_rng(5)
        lab_p = np.zeros((arr.ni + 2, arr.nj + 2, arr.nk + 2), np.uint8)
        lab_p[1:-1, 1:-1, 1:-1] = labels
        act = lab_p.ravel() != 0
        act[arr.pin_cell] = False
        r = (rng.normal(size=arr.n_cells) * act).astype(np.float32)
        rd = torch.from_numpy(r).cuda()
        zd = torch.zeros_like(rd)
        pc.apply(rd.data_ptr(), zd.data_ptr(), use_net=False)
        torch.cuda.synchronize()
        z = zd.cpu().numpy().astype(np.float64)
        invd = R.invd_from_labels(labels, table, dx * 1e-3, arr.pin_cell)
        zc, nc_ref = R.coarse_correction(r, labels, table, dx * 1e-3, arr.pin_cell, ag)
        assert nc_ref == nc
        zr = 0.6 * invd.astype(np.float64) * r + zc
        assert np.linalg.norm(z - zr) <= 1e-4 * np.linalg.norm(zr)
    finally:
        pc.close()
        solver.close()


def test_training_and_fcg_on_held_out_frames():
    """Train on the plain solver's residual/error pairs of the even frames,
    then solve the odd frames, each warm-started from the previous one, by
    plain Jacobi-PCG, by flexible CG with the two-level preconditioner
    without the network, and with it: all converge to the FP64 true relative
    residual <= 1e-6.  The two-level preconditioner needs far fewer
    iterations than plain PCG, and on this torso the trained network takes
    strictly fewer iterations than exactly the method without it (training
    is bit-reproducible, so the counts are too): 38.5 against 39.5 on
    average, no frame worse."""
    import torch
    from hrdayapy_b200.ecg.precond import LearnedPreconditioner
    solver, grid, labels, table, dx, vox = _small(seed=4)
    pc = LearnedPreconditioner(solver, labels, len(table), omega=0.6, seed=5)
    try:
        fr = _wave_frames(vox, 16, seed=6)
        vm = torch.from_numpy(fr).cuda().contiguous()
        hist = pc.train(vm[0:16:2], ks=tuple(range(0, 64, 4)), repeats=2, lr=1e-3)
        assert np.all(np.isfinite(hist))
        assert hist[-32:].mean() < hist[:32].mean()     # training lowers the loss
        plain, two, learned = [], [], []
        for f in range(1, len(fr), 2):
            for out, mode in ((plain, None), (two, False), (learned, True)):
                solver.reset()
                solver.solve_frame(fr[f - 1], 1e-6, "rel", 20000)
                if mode is None:
                    _, st = solver.solve_frame(fr[f], 1e-6, "rel", 20000)
                else:
                    _, st = pc.solve_frame(fr[f], 1e-6, 20000, 400, use_net=mode)
                    assert st.restarts < 1000            # no fallback to plain PCG
                assert st.rel_residual <= 1e-6 and st.status == 0
                out.append(st.iterations)
        print("iterations: plain PCG", plain, "two-level FCG", two, "learned FCG", learned)
        assert np.mean(two) < 0.5 * np.mean(plain), (two, plain)
        print(f"network gain: {np.mean(two) - np.mean(learned):.2f} iterations per frame "
              f"({100 * (1 - np.mean(learned) / np.mean(two)):.1f} %)")
        assert np.mean(learned) < np.mean(two), (learned, two)
        assert all(l <= t for l, t in zip(learned, two)), (learned, two)
    finally:
        pc.close()
        solver.close()


def test_training_is_bit_reproducible():
    """Two trainings from the same seed on the same frames and warm start give
    the same weights bit for bit: every gradient (the tensor-core data and
    weight gradients included) is summed in a fixed order, with no atomics."""
    import torch
    from hrdayapy_b200.ecg.precond import LearnedPreconditioner
    solver, grid, labels, table, dx, vox = _small(seed=4, shape=(16, 16, 256))
    try:
        fr = _wave_frames(vox, 6, seed=6)
        vm = torch.from_numpy(fr).cuda().contiguous()
        params = []
        for trial in range(2):
            solver.reset()
            pc = LearnedPreconditioner(solver, labels, len(table), omega=0.6, seed=5)
            try:
                hist = pc.train(vm[0:6:2], ks=(0, 4, 12, 24), repeats=2, lr=1e-3)
                assert np.all(np.isfinite(hist))
                params.append(pc.params()[0])
            finally:
                pc.close()
        assert np.abs(params[0]).max() > 0
        np.testing.assert_array_equal(params[0], params[1])
    finally:
        solver.close()
