"""Parity at the benchmark configurations' own sizes (not toy grids).

Config 1: the 64 x 64 x 16 isotropic slab at 0.25 mm (sigma 0.13 S/m,
chi 1400 /cm, Cm 1 uF/cm^2, 52 uA/uF for 1 ms in the 4 x 4 x 16 corner, all
epicardial cells), dt = 0.02 ms for the full 300 ms, FP32 on the GPU
against the FP64 oracle of the reference method at the same scheme
(run_coupled, simulation/functions/purkinje_myocardium_pipeline.py:1030-1420).
Long runs accumulate FP32 drift through the whole action potential and its
repolarisation, which short toy runs cannot show.

Tolerances (FP32 vs an FP64 run of the reference method): Vm RMS <= 0.5 mV
over every 1 ms frame and node, max activation-time error <= 0.1 ms at the
-20 mV crossing.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VM_RMS_TOL = 0.5     # mV
ACT_TOL = 0.1        # ms


def _gpu_slab(theta=0.0, T=None, cg_tol=1e-7):
    from hrdayapy_b200 import monodomain as M, synthetic
    args, _, kw = synthetic.slab()
    if T is not None:
        kw = dict(kw, T=T)
    nodes, el, act, S, phi = args
    prob, _ = M.prepare(nodes, el, act, S, S, phi, vm_save_dt=1.0, act_threshold=-20.0,
                        deact_threshold=-20.0, theta=theta, cg_tol=cg_tol, **kw)
    sim = M.MonoHandle(prob)
    sim.run(prob.n_steps, graph_chunk=50)
    vm = sim.vm_frames()
    a, na, _, _ = sim.events()
    vnow, _ = sim.voltage()
    sim.close()
    return args, kw, vm, a[0], na, vnow


def _oracle_slab(args, kw, theta=0.0, cg_tol=1e-10):
    from oracle import mono as orc
    nodes, el, act, S, phi = args
    ctx = orc.setup(nodes, el, act, S, phi, vm_save_dt=None, theta=theta, cg_tol=cg_tol,
                    cg_max_iter=500, **kw)
    first, fr, ft = orc.advance_events(ctx, ctx["n_steps"], -20.0, frame_every=50, chunk=500)
    return first, fr, ft, ctx["V"][ctx["Np"]:]


def test_config1_slab_300ms_vs_fp64_oracle():
    args, kw, vm, act_gpu, na, vnow = _gpu_slab()
    first, fr, ft, v_end = _oracle_slab(args, kw)
    assert vm.shape == fr.shape == (300, 64 * 64 * 16)
    rms = float(np.sqrt(np.mean((vm.astype(np.float64) - fr) ** 2)))
    rms_end = float(np.sqrt(np.mean((vnow.astype(np.float64) - v_end) ** 2)))
    assert np.isfinite(first).all() and (na >= 1).all()
    err = float(np.max(np.abs(act_gpu.astype(np.float64) - first)))
    print(f"config 1 (64x64x16, 300 ms, theta 0): Vm RMS {rms:.3e} mV over 300 frames, "
          f"final-state RMS {rms_end:.3e} mV, max |dLAT| {err:.3e} ms")
    assert rms <= VM_RMS_TOL
    assert rms_end <= VM_RMS_TOL
    assert err <= ACT_TOL


def test_config1_slab_theta_half_vs_fp64_oracle():
    """The reference's default scheme (theta = 0.5, Crank-Nicolson with its
    BiCGSTAB, pipeline.py:662-754, 1383-1391) over the whole activation of
    the slab (60 ms): the GPU's matrix-free CG at its FP32 floor (1e-7)
    against the oracle's BiCGSTAB at 1e-10."""
    args, kw, vm, act_gpu, na, vnow = _gpu_slab(theta=0.5, T=60.0, cg_tol=1e-7)
    first, fr, ft, v_end = _oracle_slab(args, kw, theta=0.5, cg_tol=1e-10)
    assert vm.shape == fr.shape
    rms = float(np.sqrt(np.mean((vm.astype(np.float64) - fr) ** 2)))
    ok = np.isfinite(first)
    assert ok.all() and (na >= 1).all()
    err = float(np.max(np.abs(act_gpu.astype(np.float64) - first)))
    print(f"config 1 (64x64x16, 60 ms, theta 0.5): Vm RMS {rms:.3e} mV, max |dLAT| {err:.3e} ms")
    assert rms <= VM_RMS_TOL
    assert err <= ACT_TOL
