"""Pins the oracle (FP64 CPU restatement) to fixtures produced by running the
upstream HrdayaPy code itself (tests/golden/make_golden.py)."""
import numpy as np
import pytest

from oracle import mono
from tests import cases

PHENO = {"endo": 0, "mid": 1, "epi": 2}


@pytest.mark.parametrize("key", ["endo", "mid", "epi"])
def test_ttp06_cells(golden, key):
    g = golden("ttp06_cells.npz")
    st = g[f"{key}_state"].copy()
    I = mono.ttp06_step(g[f"{key}_V"], st, 0.02, np.full(len(st), PHENO[key], np.int8))
    np.testing.assert_allclose(I, g[f"{key}_Iion"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(st, g[f"{key}_state_out"], rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("key", ["endo", "mid", "epi"])
def test_ttp06_pacing_trace(golden, key):
    g = golden("ttp06_pacing.npz")
    st = np.tile(mono.TTP06_INIT, (1, 1))
    V = np.array([mono.V0])
    ph = np.array([PHENO[key]], np.int8)
    trace = np.empty(20000)
    for k in range(20000):
        Is = 52.0 if k < 50 else 0.0
        I = mono.ttp06_step(V, st, 0.02, ph)
        V = V + 0.02 * (Is - I)
        trace[k] = V[0]
    np.testing.assert_allclose(trace[:500], g[f"{key}_V_fine"], atol=1e-9)
    np.testing.assert_allclose(trace[::25], g[f"{key}_V"], atol=1e-7)


def test_mono_iso_bit_exact(golden):
    g = golden("mono_iso.npz")
    (nodes, el, act, S, phi), kw = cases.iso_case()
    r = mono.run(nodes, el, act, S, phi, vm_save_dt=0.02, **kw)
    assert r["Vm"].shape[0] == int(g["n_frames"])
    np.testing.assert_array_equal(r["vox_idx"], g["vox_idx"])
    # float32 snapshots of an FP64 run: identical to the upstream code
    np.testing.assert_allclose(r["Vm"][::25], g["Vm_sub"], atol=1e-4)
    np.testing.assert_allclose(r["Vm"][-1], g["Vm_last"], atol=1e-4)
    a = mono.activation_maps(r["Vm"], r["time_vm"], -20.0, -20.0)
    np.testing.assert_allclose(a["activation_times"], g["act"], atol=1e-5)


def test_mono_aniso(golden):
    g = golden("mono_aniso.npz")
    (nodes, el, act, S, phi), fibre, kw = cases.aniso_case()
    r = mono.run(nodes, el, act, S, phi, fibre_dir=fibre, anisotropic=True,
                 vm_save_dt=0.02, **kw)
    np.testing.assert_array_equal(r["vox_idx"], g["vox_idx"])
    assert r["Np"] == int(g["n_comp"])
    np.testing.assert_allclose(r["Vm"][::25], g["Vm_sub"], atol=1e-4)
    np.testing.assert_allclose(r["Vm"][-1], g["Vm_last"], atol=1e-4)
    np.testing.assert_allclose(r["Vp"][::25], g["Vp_sub"], atol=1e-4)
    a = mono.activation_maps(r["Vm"], r["time_vm"], -20.0, -20.0)
    assert a["activation_times"].shape == g["act"].shape
    np.testing.assert_allclose(a["activation_times"], g["act"], atol=1e-5)


def test_scheme_gap_is_reported(golden):
    """theta=0 (the method built here) vs the upstream default theta=0.5: the
    gap is a property of the scheme, recorded for the documentation."""
    for name in ("mono_iso.npz", "mono_aniso.npz"):
        g = golden(name)
        gap = np.nanmax(np.abs(g["act"][:, 0] - g["act_cn"][:, 0]))
        assert 0.0 < gap < 0.5
