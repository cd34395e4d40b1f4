"""PMJ capture / delay harness (the reference's Experiment 4 core) on the GPU
time step at theta = 0.5, against the upstream harness's own outputs
(tests/golden/pmj_exp4.npz), plus its host-side pieces on the CPU."""
import numpy as np
import pytest

from hrdayapy_b200.experiments import pmj

CASES = (("ortho", "orthodromic"), ("ortho_block", "orthodromic"), ("anti", "antidromic"))


def test_geometry_matches_fixture(golden):
    g = golden("pmj_exp4.npz")
    S, Z, phi, fibre = pmj.build_myocardium(float(g["dx_m"]))
    assert int(S.sum()) == g["ortho_myo_act"].shape[0]
    assert (fibre[S == 1] == pmj.FIBRE_DIRECTION).all()
    ect = pmj.build_ectopic_region(S.shape, float(g["dx_m"]))
    assert ect[S == 1].any()
    nodes, el, act = pmj.build_purkinje(float(g["dx_m"]))
    assert nodes.shape == (3, 3) and act.argmin() == 0


def test_host_pieces():
    t = np.arange(5, dtype=np.float32)
    Vm = np.array([[-80, -80, -80], [-50, -80, -80], [-30, -80, -30], [0, -80, -60],
                   [10, -80, -20]], np.float32)
    fc = pmj.first_crossing_times(Vm, t, -40.0)
    assert fc[0] == pytest.approx(1.5) and np.isnan(fc[1]) and fc[2] == pytest.approx(1.8)
    arc = np.linspace(0, 20, 41).astype(np.float32)
    cv = pmj.estimate_purkinje_cv(arc, arc / 2.0)
    assert cv["cv_mm_per_ms"] == pytest.approx(2.0) and cv["r2"] == pytest.approx(1.0)
    assert np.isnan(pmj.estimate_purkinje_cv(arc[:5], arc[:5])["cv_mm_per_ms"])
    rows = [dict(direction="orthodromic", n_pmj=1, c_pmj_scale=s, propagating_capture=c)
            for s, c in ((0.1, False), (0.3, True), (1.0, True))]
    assert pmj.find_transition(rows, "orthodromic", 1) == dict(status="bracketed", lo=0.1, hi=0.3)
    assert pmj.find_transition(rows, "antidromic", 1)["status"] == "no_data"
    with pytest.raises(ValueError):
        pmj.pmj_capture_delay(np.zeros((1, 3)), np.zeros(1), np.zeros(1), np.zeros(1), 0.1, 1,
                              "sideways")


@pytest.mark.gpu
@pytest.mark.parametrize("tag,direction", CASES)
def test_capture_and_delay_vs_upstream(golden, tag, direction):
    g = golden("pmj_exp4.npz")
    r = pmj.run_directional(pmj.SIGMA_L, pmj.SIGMA_T, pmj.SIGMA_P, float(g["dt"]),
                            float(g["dx_p"]), float(g["dx_m"]), float(g[f"{tag}_T"]),
                            float(g[f"{tag}_c_pmj"]), int(g["n_pmj"]), direction)
    np.testing.assert_array_equal(r["pmj_coupled_myo_idx"], g[f"{tag}_pmj_coupled_myo_idx"])
    np.testing.assert_allclose(r["p_arc_length"], g[f"{tag}_p_arc_length"], rtol=1e-6)
    assert r["pmj_junction_capture_fraction"] == float(g[f"{tag}_pmj_junction_capture_fraction"])
    assert r["pmj_propagating_capture"] == bool(g[f"{tag}_pmj_propagating_capture"])
    ref_delay = float(g[f"{tag}_pmj_delay_ms"])
    if np.isnan(ref_delay):
        assert np.isnan(r["pmj_delay_ms"])
    else:
        assert abs(r["pmj_delay_ms"] - ref_delay) <= 0.1
    for key in ("p_act", "myo_act"):
        a, b = r[key], g[f"{tag}_{key}"]
        both = np.isfinite(a) & np.isfinite(b)
        assert (np.isfinite(a) != np.isfinite(b)).sum() <= max(1, int(0.002 * len(b))), key
        if both.any():
            assert np.max(np.abs(a[both] - b[both])) <= 0.1, key
