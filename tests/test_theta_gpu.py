"""GPU parity of the theta-scheme diffusion half (the reference's default
theta = 0.5, Crank-Nicolson) against the upstream code's own activation maps
(golden ``act_cn``) and against the oracle's FP64 restatement of the
reference's BiCGSTAB step.

Tolerances as for the explicit step: Vm RMS <= 0.5 mV, activation <= 0.1 ms."""
import numpy as np
import pytest

from tests import cases
from tests.test_mono_gpu import ACT_TOL, VM_RMS_TOL, _rms

pytestmark = pytest.mark.gpu


def _run_theta(args, kw, fibre=None, theta=0.5, cg_tol=1e-6, **extra):
    from hrdayapy_b200 import monodomain as M
    nodes, el, act, S, phi = args
    aniso = fibre is not None
    kwx = dict(kw)
    if aniso:
        kwx["A_P"] = 2.0 / kwx["R_P"]
    prob, info = M.prepare(nodes, el, act, S, S, phi, fibre_dir=fibre, anisotropic=aniso,
                           vm_save_dt=kw["dt"], act_threshold=-20.0, deact_threshold=-20.0,
                           theta=theta, cg_tol=cg_tol, cg_max_iter=100, **{**kwx, **extra})
    sim = M.MonoHandle(prob)
    sim.run(prob.n_steps)
    vm = sim.vm_frames()
    a, na, d, nd = sim.events()
    stats = sim.cn_stats()
    sim.close()
    return prob, vm, a, na, stats


def _oracle_theta(args, kw, fibre=None, theta=0.5):
    from oracle import mono as orc
    nodes, el, act, S, phi = args
    extra = dict(fibre_dir=fibre, anisotropic=True) if fibre is not None else {}
    r = orc.run(nodes, el, act, S, phi, vm_save_dt=kw["dt"], theta=theta, cg_tol=1e-10,
                cg_max_iter=200, **extra, **kw)
    ra = orc.activation_maps(r["Vm"], r["time_vm"], -20.0, -20.0)["activation_times"]
    return r, ra


@pytest.mark.parametrize("name", ["iso", "aniso"])
def test_theta_vs_upstream_golden(golden, name):
    g = golden(f"mono_{name}.npz")
    if name == "iso":
        args, kw = cases.iso_case()
        fibre = None
    else:
        args, fibre, kw = cases.aniso_case()
    prob, vm, a, na, (iters, solves, unconv, brk) = _run_theta(args, kw, fibre=fibre)
    assert solves == prob.n_steps and unconv == 0 and brk == 0
    assert 0 < iters <= 20 * solves
    ref = g["act_cn"][:, 0]
    assert np.isfinite(ref).all() and (na >= 1).all()
    assert np.max(np.abs(a[0] - ref)) <= ACT_TOL
    r, _ = _oracle_theta(args, kw, fibre=fibre)
    assert vm.shape == r["Vm"].shape
    assert _rms(vm, r["Vm"]) <= VM_RMS_TOL


@pytest.mark.parametrize("brick", [(4, 4, 8), (8, 8, 8)])
@pytest.mark.parametrize("theta", [0.5, 1.0])
def test_theta_ragged_vs_oracle(brick, theta):
    """Ragged anisotropic heart with Purkinje tree and junctions, theta = 0.5
    (Crank-Nicolson) and 1 (backward Euler), at the reference's default
    tolerance."""
    args, fibre, kw = cases.ragged_aniso_case(T=25.0)
    prob, vm, a, na, (iters, solves, unconv, brk) = _run_theta(
        args, kw, fibre=fibre, theta=theta, cg_tol=1e-5, brick=brick)
    assert unconv == 0 and brk == 0
    r, ra = _oracle_theta(args, kw, fibre=fibre, theta=theta)
    assert vm.shape == r["Vm"].shape
    assert _rms(vm, r["Vm"]) <= VM_RMS_TOL
    ok = np.isfinite(ra[:, 0])
    assert ok.sum() > 0.5 * len(ok)
    assert (na[ok] >= 1).all() and (na[~ok] == 0).all()
    assert np.max(np.abs(a[0][ok] - ra[ok, 0])) <= ACT_TOL


def test_theta_public_api(tmp_path, golden):
    """The drop-in entry point with the reference's default theta = 0.5 (no
    theta argument): activation table against the upstream code's own."""
    from hrdayapy_b200.simulation import compute_coupled
    g = golden("mono_iso.npz")
    args, kw = cases.iso_case()
    nodes, el, act, S, phi = args
    kw = dict(kw)
    kw.pop("stim_len_mm")
    res = compute_coupled(nodes, el, act, S, S, phi, stim_len_mm=1.0, cg_tol=1e-6,
                          save_path=tmp_path / "c.npz", vm_save_dt=kw["dt"],
                          vm_save_path=tmp_path / "vm.npz", n_frames=10,
                          act_threshold=-20.0, deact_threshold=-20.0, **kw)
    assert (tmp_path / "c.npz").exists() and (tmp_path / "vm.npz").exists()
    assert np.isfinite(res["vm_snapshots"]).all()
    assert np.max(np.abs(res["activation_times"][:, 0] - g["act_cn"][:, 0])) <= ACT_TOL


def test_theta_graph_and_host_loop_agree():
    """Device-side solve loops (conditional graph nodes) and the host-tested
    chunks run the same kernels in the same order: bit-identical results,
    same iteration counts."""
    from hrdayapy_b200 import monodomain as M
    args, fibre, kw = cases.aniso_case()
    nodes, el, act, S, phi = args
    out = []
    for chunk in (0, 16):
        prob, _ = M.prepare(nodes, el, act, S, S, phi, fibre_dir=fibre, anisotropic=True,
                            vm_save_dt=kw["dt"], theta=0.5, cg_tol=1e-6,
                            **dict(kw, A_P=2.0 / kw["R_P"], T=4.0))
        sim = M.MonoHandle(prob)
        sim.run(prob.n_steps, graph_chunk=chunk)
        out.append((sim.vm_frames(), sim.voltage()[1], sim.cn_stats()))
        sim.close()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2]
