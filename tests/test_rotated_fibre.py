"""Known-answer test of the anisotropic 18-connected stencil: the oblique-
fibre conduction ellipse of the reference's validation experiment
(experiments/experiment_5/rotated_fiber_values.py:11-58,
rotated_fiber_common.py:30-131,150-278).

A 20 x 10 x 10 mm slab of myocardium with a one-voxel insulating border is
stimulated over its x <= 1 mm face (0.36 uA/mm^2 for 2 ms), with the fibres
along x (longitudinal), along z (transverse) or along (1, 0, 1) / sqrt 2
(45 degrees, the case that needs the twelve edge-diagonal stencil terms).
sigma_l 0.133, sigma_t 0.0176 mS/mm, Cm 0.01 uF/mm^2, A_M 140 /mm,
theta 0.5, dt 0.5 ms.  Activation is the -40 mV upstroke crossing.  Inside
the region 3 mm from the stimulated and far faces, 0.5 mm from the y walls
and 0.6 mm from the z walls:

* the planar conduction velocity is the inverse slope of a least-squares
  line of activation time against x (rotated_fiber_common.py:150-175);
* the local normal speed is 1 / |grad t| with central differences
  (one-sided at the box edges), and its eikonal prediction is
  sqrt(v_l^2 (n.f)^2 + v_t^2 (1 - (n.f)^2)) for the local normal n and fibre
  f, v_l and v_t taken from the longitudinal and transverse runs
  (rotated_fiber_values.py:54-58; rotated_fiber_common.py:178-245); the
  reference passes the 45-degree run when its RMS relative error is below
  5 % (rotated_fiber_values.py:35).

The reference runs the experiment at dx 0.1 mm; the GPU test does too,
through compute_anisotropic_coupled, and applies the reference's pass rule.
The oracle runs the same experiment at dx 0.25 mm on the CPU, where the
axial fronts are checked for planarity (the oblique pointwise error is
about 11 % at that spacing, so the pass rule is not applied there), and on the
45-degree case the GPU run at that size is compared with it node by node."""
import numpy as np
import pytest

LX, LY, LZ, PAD = 20.0, 10.0, 10.0, 1
SIGMA_L, SIGMA_T, CM, A_M = 0.133, 0.0176, 0.01, 140.0
STIM = [dict(name="face_stimulus", target="ectopic", amp=0.36, dur=2.0, onset=0.0)]
DT, THETA, TOL = 0.5, 0.5, 0.05
FIBRES = {"longitudinal": np.array([1.0, 0.0, 0.0]),
          "transverse": np.array([0.0, 0.0, 1.0]),
          "rotated45": np.array([1.0, 0.0, 1.0]) / np.sqrt(2.0)}


def _slab(dx, fibre):
    """Padded slab, fibre field, stimulated face and a two-node Purkinje stub
    5 mm outside the slab (sigma_P = 0, c_pmj = 0: it carries no current)."""
    n = [max(2, int(round(L / dx))) + 2 * PAD for L in (LX, LY, LZ)]
    S = np.zeros(n, np.uint8)
    S[PAD:-PAD, PAD:-PAD, PAD:-PAD] = 1
    fd = np.zeros(tuple(n) + (3,), np.float32)
    fd[S == 1] = fibre
    x = (np.indices(n)[0] - PAD) * dx
    face = (x >= 0) & (x <= 1.0)
    stub = np.array([[LX + 5, LY + 5, LZ + 5], [LX + 5, LY + 5, LZ + 10]]) / dx + PAD
    return S, fd, face, stub


def _region(vox, act, dx):
    c = (np.asarray(vox) - PAD) * dx
    x, y, z = c[:, 0], c[:, 1], c[:, 2]
    return ((x >= 3.0) & (x <= LX - 3.0) & (y >= 0.5) & (y <= LY - 0.5)
            & (z >= 0.6) & (z <= LZ - 0.6) & np.isfinite(act))


def _planar_cv(vox, act, dx):
    m = _region(vox, act, dx)
    assert m.sum() >= 10
    x = (np.asarray(vox)[m, 0] - PAD) * dx
    A = np.stack([x, np.ones_like(x)], 1)
    slope = np.linalg.lstsq(A, act[m].astype(np.float64), rcond=None)[0][0]
    assert slope > 0
    return 1.0 / slope


def _normal_speed(vox, act, dx):
    """Local wavefront normal and normal speed 1 / |grad t| on the dense box
    of myocardial voxels: central differences where both neighbours
    activated, one-sided where only one did, NaN otherwise."""
    vox = np.asarray(vox)
    idx = vox - vox.min(0)
    shape = tuple(idx.max(0) + 1)
    assert len(idx) == np.prod(shape)                   # the slab is a full box
    t = np.full(shape, np.nan)
    t[tuple(idx.T)] = act
    g = np.empty(shape + (3,))
    for a in range(3):
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[a], hi[a] = slice(0, -1), slice(1, None)
        fwd = np.full(shape, np.nan)
        bwd = np.full(shape, np.nan)
        fwd[tuple(lo)] = t[tuple(hi)]
        bwd[tuple(hi)] = t[tuple(lo)]
        d = (fwd - bwd) / (2 * dx)
        d = np.where(np.isnan(d), (fwd - t) / dx, d)
        d = np.where(np.isnan(d), (t - bwd) / dx, d)
        g[..., a] = d
    g = g[tuple(idx.T)]
    mag = np.linalg.norm(g, axis=1)
    with np.errstate(invalid="ignore", divide="ignore"):
        return g / mag[:, None], 1.0 / mag


def _eikonal_rms(vox, act, dx, fibre, v_l, v_t):
    """RMS relative error of the local normal speed against the eikonal
    ellipse inside the fit region."""
    n, cn = _normal_speed(vox, act, dx)
    m = _region(vox, act, dx) & np.isfinite(cn) & np.isfinite(n).all(1)
    assert m.sum() >= 10
    nf = n[m] @ fibre
    pred = np.sqrt(v_l ** 2 * nf ** 2 + v_t ** 2 * (1.0 - nf ** 2))
    return float(np.sqrt(np.mean(((cn[m] - pred) / pred) ** 2)))


def _oracle_run(dx, name, T):
    from oracle import mono as O
    S, fd, face, stub = _slab(dx, FIBRES[name])
    ctx = O.setup(stub, np.array([[0, 1]]), np.array([0.0, 1.0]), S,
                  np.zeros(S.shape, np.float32), fibre_dir=fd, voxel_size=dx, dx_p=dx,
                  sigma_P=0.0, sigma_l=SIGMA_L, sigma_t=SIGMA_T, Cm=CM, A_M=A_M, R_P=0.01,
                  dt=DT, T=T, anisotropic=True, theta=THETA, cg_tol=1e-8, cg_max_iter=5000,
                  stim_protocol=STIM, ectopic_region=face, stim_len_mm=1.0, c_pmj=0.0,
                  n_pmj=1)
    act, _, _ = O.advance_events(ctx, int(round(T / DT)), act_threshold=-40.0)
    return ctx["vox_idx"], act


def _gpu_run(dx, name, T):
    from hrdayapy_b200.anisotropic_simulation.coupled import compute_anisotropic_coupled
    S, fd, face, stub = _slab(dx, FIBRES[name])
    r = compute_anisotropic_coupled(
        stub, np.array([[0, 1]]), np.array([0.0, 1.0]), S, S, np.zeros(S.shape, np.float32),
        fd, stim_protocol=STIM, ectopic_region=face, voxel_size=dx, dx_p=dx, sigma_P=0.0,
        sigma_l=SIGMA_L, sigma_t=SIGMA_T, Cm=CM, A_M=A_M, R_P=0.01, dt=DT, T=T, theta=THETA,
        stim_len_mm=1.0, c_pmj=0.0, n_pmj=1, cg_tol=1e-8, cg_max_iter=5000, n_frames=4)
    act = r["activation_times"]
    act = act[:, 0] if act.shape[1] else np.full(len(r["vox_idx"]), np.nan, np.float32)
    return r["vox_idx"], act


def _check_ellipse(runs, dx, pointwise_oblique):
    """Planar velocities and the pointwise eikonal errors.  The axial fronts
    must be planar (their own pointwise error below the tolerance); the
    pass rule on the oblique run is its pointwise error, as the reference's
    (run_experiment5_rotated_fiber.py:80-86).  The planar fit of the oblique
    run against sqrt((v_l^2 + v_t^2) / 2) is reported only: the z walls bend
    that front, so the fit's assumption of a normal along x fails
    (run_experiment5_rotated_fiber.py:103-106)."""
    v = {k: _planar_cv(*runs[k], dx) for k in FIBRES}
    v_l, v_t = v["longitudinal"], v["transverse"]
    pred45 = np.sqrt((v_l ** 2 + v_t ** 2) / 2.0)
    rms = {k: _eikonal_rms(*runs[k], dx, FIBRES[k], v_l, v_t) for k in FIBRES}
    stats = dict(v=v, naive_v45=pred45, rms=rms)
    print(stats)
    assert v_l > v["rotated45"] > v_t
    assert rms["longitudinal"] < TOL and rms["transverse"] < TOL, stats
    if pointwise_oblique:
        assert rms["rotated45"] < TOL, stats
    return stats


# simulated time per fibre configuration at dx 0.25 mm: each front has
# crossed the fit region by then
T_COARSE = {"longitudinal": 60.0, "transverse": 150.0, "rotated45": 80.0}


def test_oracle_conduction_ellipse():
    dx = 0.25
    runs = {k: _oracle_run(dx, k, T_COARSE[k]) for k in FIBRES}
    _check_ellipse(runs, dx, pointwise_oblique=False)


@pytest.mark.gpu
def test_gpu_conduction_ellipse_reference_size():
    dx = 0.1
    runs = {k: _gpu_run(dx, k, 150.0) for k in FIBRES}
    _check_ellipse(runs, dx, pointwise_oblique=True)


@pytest.mark.gpu
def test_gpu_oblique_activation_matches_oracle():
    dx, T = 0.25, T_COARSE["rotated45"]
    vg, ag = _gpu_run(dx, "rotated45", T)
    vo, ao = _oracle_run(dx, "rotated45", T)
    assert np.array_equal(np.asarray(vg), np.asarray(vo))
    fin = np.isfinite(ao)
    assert np.array_equal(np.isfinite(ag), fin)
    d = np.abs(ag[fin].astype(np.float64) - ao[fin])
    print("max |dt|", d.max(), "mean", d.mean())
    assert d.max() < 2e-3                       # ms; measured 1.4e-4 on a B200
