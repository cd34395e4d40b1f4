"""Host-side preparation (brick layout, tag bits, coefficients, Purkinje and
junction CSR, stimulus schedule) checked on the CPU against the oracle's
assembled global Laplacian and time loop."""
import numpy as np
import scipy.sparse as sp
import pytest

from hrdayapy_b200 import layout as L
from hrdayapy_b200 import monodomain as M
from oracle import mono as orc
from tests import cases
from tests.kernel_emulator import coefficient_matrix, emulate


@pytest.mark.parametrize("brick", [(4, 4, 8), (4, 8, 8), (2, 4, 16), (8, 8, 8)])
def test_layout_roundtrip(brick):
    rng = np.random.default_rng(0)
    S = (rng.uniform(size=(19, 13, 21)) < 0.3).astype(np.uint8)
    lay = L.build_layout(S, brick, anisotropic=True)
    vox = lay.vox_idx
    assert (vox == np.argwhere(S == 1)).all()
    assert len(np.unique(lay.slot_of_node)) == len(vox)
    bv = lay.bv
    b = lay.slot_of_node // bv
    loc = lay.slot_of_node % bv
    bi, bj, bk = brick
    li, lj, lk = loc // (bj * bk), (loc // bk) % bj, loc % bk
    rec = lay.brick_coords[b] * np.array(brick) + np.stack([li, lj, lk], 1)
    assert (rec == vox).all()
    # neighbour table: the brick itself sits at index 13, neighbours are adjacent
    assert (lay.brick_nbr[:, 13] == np.arange(lay.n_bricks)).all()
    for q, (di, dj, dk) in enumerate([(a, c, e) for a in (-1, 0, 1) for c in (-1, 0, 1)
                                      for e in (-1, 0, 1)]):
        ok = lay.brick_nbr[:, q] >= 0
        d = lay.brick_coords[lay.brick_nbr[ok, q]] - lay.brick_coords[ok]
        assert (d == np.array([di, dj, dk])).all()


def test_empty_mask():
    lay = L.build_layout(np.zeros((4, 4, 4), np.uint8), (4, 4, 8))
    assert lay.n_bricks == 0 and lay.n_slots == 0


def _coef_vs_oracle(args, kw, aniso, fibre=None):
    nodes, el, act, S, phi = args
    kw = dict(kw)
    if aniso:
        kwp = dict(kw, A_P=2.0 / kw["R_P"])
        prob, info = M.prepare(nodes, el, act, S, S, phi, fibre_dir=fibre, anisotropic=True,
                               **kwp)
        r = orc.run(nodes, el, act, S, phi, fibre_dir=fibre, anisotropic=True,
                    T=kw["dt"], **{k: v for k, v in kw.items() if k != "T"})
    else:
        prob, info = M.prepare(nodes, el, act, S, S, phi, **kw)
        r = orc.run(nodes, el, act, S, phi, T=kw["dt"], **{k: v for k, v in kw.items() if k != "T"})
    Lref = r["L"].tocsr() * (kw["dt"] / kw["Cm"])
    Lref.setdiag(0.0)
    Lref.eliminate_zeros()
    Cm = coefficient_matrix(prob)
    diff = abs(Cm - Lref)
    scale = abs(Lref).max()
    assert diff.max() <= 2e-6 * scale, diff.max() / scale
    return prob, info, r


def test_iso_coefficients_match_oracle_laplacian():
    args, kw = cases.iso_case()
    _coef_vs_oracle(args, kw, aniso=False)


def test_aniso_coefficients_match_oracle_laplacian():
    args, fibre, kw = cases.aniso_case()
    prob, info, r = _coef_vs_oracle(args, kw, aniso=True, fibre=fibre)
    assert info["Np"] == r["Np"]
    np.testing.assert_allclose(info["comp_nodes"], r["comp_nodes"])
    assert info["pmj_ids"] == r["pmj_ids"]
    assert info["pmj_patches"] == r["pmj_patches"]


def test_ragged_coefficients_match_oracle_laplacian():
    args, fibre, kw = cases.ragged_aniso_case(T=0.02)
    _coef_vs_oracle(args, kw, aniso=True, fibre=fibre)


def test_stimulus_schedule():
    assert M.stim_active(0.0, 0.0, 1.0, None, None)
    assert not M.stim_active(1.0, 0.0, 1.0, None, None)
    assert M.stim_active(10.5, 0.0, 1.0, 10.0, None)
    assert not M.stim_active(20.5, 0.0, 1.0, 10.0, 2)
    assert not M.stim_active(-0.1, 0.0, 1.0, 10.0, 2)
    for t in np.arange(0, 50, 0.37):
        for args in [(0.0, 1.0, None, None), (2.0, 2.0, 7.0, 3), (1.0, 0.5, 5.0, None)]:
            assert M.stim_active(t, *args) == orc.stim_active(t, *args)


def test_kernel_algorithm_emulation_matches_oracle():
    """The skewed single-pass step, stimulus bits and event recording give
    the oracle's trajectory (FP64 emulation, aniso + Purkinje + junctions)."""
    args, fibre, kw = cases.aniso_case()
    nodes, el, act, S, phi = args
    kw = dict(kw, T=6.0)
    prob, info = M.prepare(nodes, el, act, S, S, phi, fibre_dir=fibre, anisotropic=True,
                           vm_save_dt=0.02, act_threshold=-20.0, **dict(kw, A_P=2.0 / kw["R_P"]))
    snaps, psnaps, a_em = emulate(prob)
    r = orc.run(nodes, el, act, S, phi, fibre_dir=fibre, anisotropic=True, vm_save_dt=0.02, **kw)
    np.testing.assert_allclose(snaps, r["Vm"], atol=2e-3)
    np.testing.assert_allclose(psnaps, r["Vp"], atol=2e-3)
    a = orc.activation_maps(r["Vm"], r["time_vm"], -20.0, -20.0)["activation_times"]
    if a.shape[1]:
        np.testing.assert_allclose(a_em, a[:, 0], atol=1e-4, equal_nan=True)


@pytest.mark.parametrize("aniso", [False, True])
def test_theta_scheme_emulation_matches_oracle(aniso):
    """The GPU theta-scheme algorithm (weighted Jacobi-CG from the warm start
    x = W, reference stopping rule) against the oracle's restatement of the
    reference's BiCGSTAB at theta = 0.5.  The operator the kernels apply is
    self-adjoint in the Ai-weighted inner product the CG uses."""
    if aniso:
        args, fibre, kw = cases.aniso_case()
        extra = dict(fibre_dir=fibre, anisotropic=True)
        kw = dict(kw, A_P=2.0 / kw["R_P"])
    else:
        args, kw = cases.iso_case()
        extra = {}
    nodes, el, act, S, phi = args
    kw = dict(kw, T=6.0)
    prob, info = M.prepare(nodes, el, act, S, S, phi, vm_save_dt=0.02, act_threshold=-20.0,
                           theta=0.5, cg_tol=1e-7, cg_max_iter=100, **extra, **kw)
    C = coefficient_matrix(prob)
    Lh = C - sp.diags(np.asarray(C.sum(axis=1)).ravel())
    w = np.concatenate([np.full(prob.n_pk, prob.pk_weight), np.ones(C.shape[0] - prob.n_pk)])
    WL = sp.diags(w) @ Lh
    assert abs(WL - WL.T).max() <= 1e-6 * abs(WL).max()
    snaps, psnaps, a_em = emulate(prob)
    assert max(emulate.cn_iters) < 100
    kwo = {k: v for k, v in kw.items() if k != "A_P"} if aniso else kw
    r = orc.run(nodes, el, act, S, phi, vm_save_dt=0.02, theta=0.5, cg_tol=1e-10,
                cg_max_iter=200, **extra, **kwo)
    np.testing.assert_allclose(snaps, r["Vm"], atol=2e-3)
    if prob.n_pk and aniso:
        np.testing.assert_allclose(psnaps, r["Vp"], atol=2e-3)
    a = orc.activation_maps(r["Vm"], r["time_vm"], -20.0, -20.0)["activation_times"]
    if a.shape[1]:
        np.testing.assert_allclose(a_em, a[:, 0], atol=1e-4, equal_nan=True)


def test_bad_arguments():
    args, kw = cases.iso_case()
    nodes, el, act, S, phi = args
    with pytest.raises(ValueError):
        M.prepare(nodes, el, act, S, S, phi, **dict(kw, stim_protocol=[dict(target="bogus",
                                                                             amp=1, dur=1)]))
    with pytest.raises(ValueError):
        M.prepare(nodes, el, act, S, S, phi,
                  **dict(kw, stim_protocol=[dict(target="region", region="x", amp=1, dur=1)]))
    from hrdayapy_b200.anisotropic_simulation import purkinje_myocardium_anisotropic_solver
    with pytest.raises(TypeError):
        purkinje_myocardium_anisotropic_solver(nodes, el, act, S, S, phi,
                                               np.zeros(S.shape + (3,)), A_P=1.0)
    from hrdayapy_b200 import monodomain
    with pytest.raises(ValueError):
        monodomain.run(nodes, el, act, S, S, phi, theta=1.5, **kw)
    prob, _ = M.prepare(nodes, el, act, S, S, phi, theta=0.5, cg_tol=1e-6, cg_max_iter=50, **kw)
    assert (prob.theta, prob.cn_tol, prob.cn_max_iter) == (0.5, 1e-6, 50)
    S_P = np.pi * kw.get("R_P", 0.015) ** 2
    ai_p = kw.get("A_P", 133.33) * S_P * kw.get("dx_p", 0.2)
    ai_m = kw.get("A_M", 0.14) * kw["voxel_size"] ** 3
    assert prob.pk_weight == pytest.approx(ai_p / ai_m)
    with pytest.raises(ValueError):
        monodomain.run(nodes, el, act, S, S, phi, theta=0.0, device="cpu", **kw)
