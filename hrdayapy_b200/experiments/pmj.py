"""PMJ capture / delay and conduction-velocity harness on the GPU time step.

Restates the reference's Experiment 2-4 core
(experiments/experiment_3/experiment_common.py, constants from
experiments/experiment_3/base_values.py, transition search from
run_experiment4.py:148-196): a Purkinje fibre (root -> graze -> PMJ
polyline) coupled at one junction to a 2.5 x 2.5 x 50 mm anisotropic slab
(fibres along z), driven either at the Purkinje root (orthodromic) or by a
far-field myocardial focus (antidromic), solved by this package's
``compute_anisotropic_coupled`` at the reference's theta = 0.5.

Differences from the reference's flow, none in the arithmetic of the
results: myocardial activation times come from the in-loop event tables of
the GPU step (every step; the reference saves snapshots every
max(dt, 0.05 ms) and interpolates between them, the same computation when
dt >= 0.05 ms) and no intermediate files are written.
"""
from __future__ import annotations

import numpy as np

# base_values.py:96-100 (geometry), material and stimulus constants
P_ROOT = np.array([1.25, 7.5, -45.0])
P_GRAZE = np.array([1.25, 5.5, -3.0])
P_PMJ = np.array([1.25, 1.25, 0.0])
MYO_PAD_VOX = 1
SIGMA_P = 0.6          # mS/mm
SIGMA_L = 0.133        # mS/mm along the fibre
SIGMA_T = 0.0176       # mS/mm across
FIBRE_DIRECTION = np.array([0.0, 0.0, 1.0])
CM = 0.01              # uF/mm^2
A_M = 140.0            # 1/mm
R_P = 0.1125           # mm
C_PMJ = 5.0            # mS
N_PMJ = 1
ACT_THRESHOLD = -40.0  # mV
REF_DT, REF_DX_P, REF_DX_M = 0.05, 0.10, 0.10
STIM_LEN_MM, STIM_AMP, STIM_DUR = 2.0, 12.0, 1.0

# experiment_common.py:147-191
THETA, CG_TOL, CG_MAX_ITER = 0.5, 1e-8, 500
VM_SAVE_DT = 0.05
SLAB_X_MM, SLAB_Y_MM, SLAB_Z_MM = 2.5, 2.5, 50.0
ANTI_STIM_OFFSET_FROM_FAR_MM = 4.0
ANTI_STIM_RADIUS_MM = 2.0
ANTI_STIM_TARGET_MM = np.array([1.25, 1.25, SLAB_Z_MM - ANTI_STIM_OFFSET_FROM_FAR_MM])

# CV-fit exclusion buffers (experiment_common.py:448-457)
MYO_LATERAL_BUFFER_MM, MYO_ENTRY_BUFFER_MM, MYO_EXIT_BUFFER_MM = 2.0, 8.0, 8.0
PMJ_RADIUS_EXCLUDE_MM = 6.0
PURKINJE_ROOT_BUFFER_MM, PURKINJE_PMJ_BUFFER_MM = 5.0, 5.0
MIN_FIT_POINTS_MYO, MIN_FIT_POINTS_PKJ = 20, 5

# capture (experiment_common.py:557-567)
DIRECTIONS = ("orthodromic", "antidromic")
PROPAGATION_CHECK_RADIUS_MM = 6.0
PURKINJE_PROPAGATION_CHECK_MM = 5.0


def _axis_cells(length_mm, dx_m):
    return max(2, int(round(length_mm / dx_m))) + 2 * MYO_PAD_VOX


def build_myocardium(dx_m: float):
    """Slab mask with a one-voxel zero border (S = Z), phi = 0 (endocardial
    cells throughout) and fibres along z (experiment_common.py:197-231)."""
    shape = tuple(_axis_cells(L, dx_m) for L in (SLAB_X_MM, SLAB_Y_MM, SLAB_Z_MM))
    S = np.zeros(shape, np.uint8)
    p = MYO_PAD_VOX
    S[p:-p, p:-p, p:-p] = 1
    fibre = np.zeros(shape + (3,), np.float32)
    fibre[S == 1] = FIBRE_DIRECTION
    return S, S.copy(), np.zeros(shape, np.float32), fibre


def physical_to_voxel_idx(points_mm, dx_m: float):
    """Slab-frame mm -> the voxel-index units the solver's ``nodes`` take."""
    return np.asarray(points_mm) / dx_m + MYO_PAD_VOX


def build_purkinje(dx_m: float):
    """Root -> graze -> PMJ polyline; node 0 (earliest) is the root."""
    nodes = physical_to_voxel_idx(np.stack([P_ROOT, P_GRAZE, P_PMJ]), dx_m).astype(np.float64)
    return nodes, np.array([[0, 1], [1, 2]], np.int64), np.array([0.0, 1.0, 2.0])


def build_ectopic_region(S_shape, dx_m: float, target_mm=None, radius_mm=None):
    """Voxels within radius_mm (slab frame) of target_mm (default: the
    antidromic far-field focus), experiment_common.py:570-596."""
    target = ANTI_STIM_TARGET_MM if target_mm is None else np.asarray(target_mm)
    r = ANTI_STIM_RADIUS_MM if radius_mm is None else radius_mm
    ii, jj, kk = np.indices(S_shape)
    d2 = (((ii - MYO_PAD_VOX) * dx_m - target[0]) ** 2 + ((jj - MYO_PAD_VOX) * dx_m - target[1]) ** 2
          + ((kk - MYO_PAD_VOX) * dx_m - target[2]) ** 2)
    return d2 <= r ** 2


def purkinje_ordered_trace(results):
    """Root -> PMJ ordered compartment trace from the two branches' frames
    (the shared graze node once): coords, arc length, Vm, t
    (experiment_common.py:272-303)."""
    bm0, bm1 = results["branch_map"]
    if bm0[-1] != bm1[0]:
        raise ValueError("expected branch 0 and 1 to share the graze node")
    ids = list(bm0) + list(bm1[1:])
    f0 = np.asarray(results["branch_frames_p"][0], np.float32)
    f1 = np.asarray(results["branch_frames_p"][1], np.float32)
    xyz = np.asarray(results["comp_nodes"])[ids].astype(np.float32)
    arc = np.concatenate([[0.0], np.cumsum(np.linalg.norm(np.diff(xyz, axis=0), axis=1))])
    return (xyz, arc.astype(np.float32), np.concatenate([f0, f1[:, 1:]], axis=1),
            np.asarray(results["times"], np.float32))


def first_crossing_times(Vm, t, threshold: float):
    """First upward crossing per column, linear interpolation in float32 as
    the activation maps (experiment_common.py:306-322); NaN if none."""
    Vm = np.asarray(Vm)
    hit = (Vm[:-1] < threshold) & (Vm[1:] >= threshold)
    out = np.full(Vm.shape[1], np.nan, np.float32)
    cols = np.nonzero(hit.any(axis=0))[0]
    f = hit[:, cols].argmax(axis=0)
    v0, v1 = Vm[f, cols], Vm[f + 1, cols]
    den = np.where(v1 - v0 == 0, 1e-9, v1 - v0)
    frac = np.clip((threshold - v0) / den, 0.0, 1.0)
    out[cols] = (t[f] + frac * (t[f + 1] - t[f])).astype(np.float32)
    return out


def _pmj_mm(dx_m):
    return P_PMJ + MYO_PAD_VOX * dx_m


def find_pmj_coupled_myo_nodes(myo_coords_mm, dx_m: float, n_pmj: int):
    """The n_pmj tissue nodes nearest the PMJ: the solver's own junction
    patch rule (experiment_common.py:598-612)."""
    d = np.linalg.norm(myo_coords_mm - _pmj_mm(dx_m)[None, :], axis=1)
    return np.argsort(d)[:min(n_pmj, len(myo_coords_mm))]


def pmj_capture_delay(myo_coords, myo_act, p_act, p_arc_length, dx_m: float, n_pmj: int,
                      direction: str) -> dict:
    """Junction capture fraction, propagating capture beyond the junction and
    transjunctional delay (experiment_common.py:615-703)."""
    if direction not in DIRECTIONS:
        raise ValueError(f"direction must be one of {DIRECTIONS}, got {direction!r}")
    p_term = float(p_act[-1]) if np.isfinite(p_act[-1]) else np.nan
    idx = find_pmj_coupled_myo_nodes(myo_coords, dx_m, n_pmj)
    coupled = myo_act[idx]
    fin = np.isfinite(coupled)
    both = fin.any() and np.isfinite(p_term)
    if direction == "orthodromic":
        frac = float(fin.mean()) if len(coupled) else np.nan
        delay = float(np.mean(coupled[fin]) - p_term) if both else np.nan
        dist = np.linalg.norm(myo_coords - _pmj_mm(dx_m)[None, :], axis=1)
        prop = bool((np.isfinite(myo_act) & (dist >= PROPAGATION_CHECK_RADIUS_MM)).any())
    else:
        frac = float(np.isfinite(p_term))
        delay = float(p_term - np.mean(coupled[fin])) if both else np.nan
        reach = p_arc_length <= float(p_arc_length[-1]) - PURKINJE_PROPAGATION_CHECK_MM
        prop = bool((reach & np.isfinite(p_act)).any())
    return dict(pmj_coupled_myo_idx=idx, pmj_junction_capture_fraction=frac,
                pmj_propagating_capture=prop,
                pmj_n_myo_activated=int(np.isfinite(myo_act).sum()), pmj_delay_ms=delay)


def _linear_cv(s, t, n_min):
    if len(s) < n_min:
        return dict(cv_mm_per_ms=np.nan, cv_cm_per_s=np.nan, n_points=len(s), r2=np.nan,
                    slope=np.nan)
    slope, icept = np.polyfit(s, t, 1)
    res = np.sum((t - (slope * s + icept)) ** 2)
    tot = np.sum((t - t.mean()) ** 2)
    return dict(cv_mm_per_ms=float(1.0 / slope), cv_cm_per_s=float(100.0 / slope),
                n_points=len(s), r2=float(1.0 - res / tot) if tot > 0 else np.nan,
                slope=float(slope))


def estimate_myocardial_cv(coords_mm, act_ms, dx_m: float) -> dict:
    """CV = 1 / slope of activation time vs z over the slab interior
    (experiment_common.py:461-492)."""
    off = MYO_PAD_VOX * dx_m
    x, y, z = coords_mm[:, 0], coords_mm[:, 1], coords_mm[:, 2]
    lat = ((x >= off + MYO_LATERAL_BUFFER_MM) & (x <= off + SLAB_X_MM - MYO_LATERAL_BUFFER_MM) &
           (y >= off + MYO_LATERAL_BUFFER_MM) & (y <= off + SLAB_Y_MM - MYO_LATERAL_BUFFER_MM))
    zin = (z >= off + MYO_ENTRY_BUFFER_MM) & (z <= off + SLAB_Z_MM - MYO_EXIT_BUFFER_MM)
    far = np.linalg.norm(coords_mm - _pmj_mm(dx_m)[None, :], axis=1) >= PMJ_RADIUS_EXCLUDE_MM
    m = np.isfinite(act_ms) & lat & zin & far
    return _linear_cv(z[m], act_ms[m], MIN_FIT_POINTS_MYO)


def estimate_purkinje_cv(arc_length_mm, act_ms) -> dict:
    """CV along the fibre away from the root and the PMJ
    (experiment_common.py:495-516)."""
    L = float(arc_length_mm[-1])
    m = (np.isfinite(act_ms) & (arc_length_mm >= PURKINJE_ROOT_BUFFER_MM) &
         (arc_length_mm <= L - PURKINJE_PMJ_BUFFER_MM))
    return _linear_cv(arc_length_mm[m], act_ms[m], MIN_FIT_POINTS_PKJ)


def run_directional(sigma_l: float, sigma_t: float, sigma_P: float, dt: float, dx_p: float,
                    dx_m: float, T: float, c_pmj: float, n_pmj: int, direction: str, *,
                    theta: float = THETA, cg_tol: float = CG_TOL,
                    cg_max_iter: int = CG_MAX_ITER) -> dict:
    """One cell of the capture / delay sweep (experiment_common.py:706-820):
    activation times of both domains and the PMJ summary."""
    from ..anisotropic_simulation import compute_anisotropic_coupled
    if direction not in DIRECTIONS:
        raise ValueError(f"direction must be one of {DIRECTIONS}, got {direction!r}")
    S, Z, phi, fibre = build_myocardium(dx_m)
    nodes, elements, act_times = build_purkinje(dx_m)
    ect = None
    if direction == "orthodromic":
        prot = [dict(name="purkinje_root", target="root", amp=STIM_AMP, dur=STIM_DUR, onset=0.0)]
    else:
        ect = build_ectopic_region(S.shape, dx_m)
        if not ect.any():
            raise RuntimeError("antidromic ectopic_region is empty at this dx_m")
        prot = [dict(name="myo_far_field", target="ectopic", amp=STIM_AMP, dur=STIM_DUR,
                     onset=0.0)]
    n_steps = int(round(T / dt))
    res = compute_anisotropic_coupled(
        nodes, elements, act_times, S, Z, phi, fibre, stim_protocol=prot, ectopic_region=ect,
        voxel_size=dx_m, dx_p=dx_p, sigma_P=sigma_P, sigma_l=sigma_l, sigma_t=sigma_t, Cm=CM,
        A_M=A_M, R_P=R_P, dt=dt, T=T, theta=theta, stim_len_mm=STIM_LEN_MM, c_pmj=c_pmj,
        n_pmj=n_pmj, cg_tol=cg_tol, cg_max_iter=cg_max_iter, n_frames=n_steps,
        act_threshold=ACT_THRESHOLD, deact_threshold=ACT_THRESHOLD)
    # (x, y, z) of the tree frame: the solver's node coordinates with the
    # row / column swap undone (experiment_common.py:791-795)
    myo_coords = np.asarray(res["coords_mm"])[:, [1, 0, 2]]
    at = np.asarray(res["activation_times"])
    myo_act = at[:, 0].astype(np.float32) if at.shape[1] else np.full(len(myo_coords), np.nan,
                                                                       np.float32)
    _, arc, p_vm, p_t = purkinje_ordered_trace(res)
    p_act = first_crossing_times(p_vm, p_t, ACT_THRESHOLD)
    out = dict(myo_coords=myo_coords, myo_act=myo_act, p_arc_length=arc, p_act=p_act,
               direction=direction, c_pmj=c_pmj, n_pmj=n_pmj)
    out.update(pmj_capture_delay(myo_coords, myo_act, p_act, arc, dx_m, n_pmj, direction))
    return out


def find_transition(results, direction: str, n_pmj: int) -> dict:
    """Capture / block transition over a c_pmj sweep, assuming capture is
    monotone in c_pmj: the smallest scale from which every larger one
    captures (run_experiment4.py:148-180).  Rows carry ``direction``,
    ``n_pmj``, ``c_pmj_scale`` and ``propagating_capture``."""
    rows = sorted((r for r in results if r["direction"] == direction and r["n_pmj"] == n_pmj),
                  key=lambda r: r["c_pmj_scale"])
    if not rows:
        return dict(status="no_data")
    caps = [bool(r["propagating_capture"]) for r in rows]
    sc = [r["c_pmj_scale"] for r in rows]
    i = next((k for k in range(len(caps)) if all(caps[k:])), None)
    if i == 0:
        return dict(status="always_capture", hi=sc[0])
    if i is None:
        return dict(status="never_capture", lo=sc[-1])
    return dict(status="bracketed", lo=sc[i - 1], hi=sc[i])
