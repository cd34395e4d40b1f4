"""ORACLE -- test infrastructure, not product code.

FP64 CPU restatement of HrdayaPy's monodomain path, used only by
tests/, by ``__graft_entry__.smoke()`` as the checker and by ``bench.py``'s
CPU-baseline leg.  The product package never imports this module.

Each function restates one upstream function (paths relative to the
upstream project root):

* :func:`discretise_tree`   -- simulation/functions/purkinje_myocardium_pipeline.py:88-114
* :func:`build_myo_mesh`    -- purkinje_myocardium_pipeline.py:761-833
* :func:`build_myo_mesh_anisotropic` -- anisotropic_simulation/functions/
  purkinje_myocardium_anisotropic_solver.py:856-1074
* :func:`global_laplacian`  -- purkinje_myocardium_pipeline.py:578-651 and
  purkinje_myocardium_anisotropic_solver.py:606-746
* :func:`map_pmj`, :func:`find_terminals` -- pipeline.py:888-920
* :func:`stim_active`, :func:`resolve_stim_sites` -- pipeline.py:947-1023,
  purkinje_myocardium_anisotropic_solver.py:1204-1300
* :func:`phenotypes`        -- ionic_models/hetero_solver.py:74-128
* :func:`run`               -- run_coupled (pipeline.py:1030-1420) and the
  anisotropic solver (..._anisotropic_solver.py:1308-1820); the time loop
  itself runs in C (ttp06_oracle.c): orc_mono_run at theta = 0,
  orc_mono_run_cn (the reference's BiCGSTAB, pipeline.py:662-754) at
  theta > 0
* :func:`activation_maps`   -- simulation/functions/activation_maps.py:63-116,295-350

Parity is pinned by tests/test_oracle_golden.py against fixtures produced by
running the upstream code itself (tests/golden/make_golden.py).
"""
from __future__ import annotations

import ctypes
import math
from pathlib import Path

import numpy as np
import scipy.sparse as sp
from scipy.spatial import cKDTree

_HERE = Path(__file__).resolve().parent
_LIB = None


def lib():
    """The compiled C half of the oracle (built by ``make -C oracle``)."""
    global _LIB
    if _LIB is None:
        so = _HERE / "liboracle.so"
        if not so.exists():
            raise RuntimeError(f"oracle library missing: build it with make -C {_HERE}")
        L = ctypes.CDLL(str(so))
        P = ctypes.c_void_p
        L.orc_ttp06_step.argtypes = [ctypes.c_int64, P, P, ctypes.c_double, P, P, P, P]
        L.orc_ttp06_step.restype = None
        L.orc_ttp06_cell.argtypes = [ctypes.c_double, P, ctypes.c_double, ctypes.c_int,
                                     ctypes.c_double, ctypes.c_double]
        L.orc_ttp06_cell.restype = ctypes.c_double
        L.orc_mono_run.argtypes = [ctypes.c_int64, ctypes.c_int64, P, P, P, P, P, P,
                                   ctypes.c_double, ctypes.c_double, ctypes.c_int64,
                                   ctypes.c_int, P, P, P, P, P, P, ctypes.c_int64, P, P]
        L.orc_mono_run.restype = ctypes.c_int
        L.orc_mono_run_cn.argtypes = L.orc_mono_run.argtypes + [
            ctypes.c_double, ctypes.c_double, ctypes.c_int64, P]
        L.orc_mono_run_cn.restype = ctypes.c_int
        L.orc_num_threads.restype = ctypes.c_int
        _LIB = L
    return _LIB


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


TTP06_INIT = np.array([138.4, 10.355, 0.00013, 0.00448, 0.476, 0.0087, 0.00155,
                       0.7573, 0.7225, 3.164e-5, 0.8009, 0.9778, 0.9953, 0.3212,
                       2.235e-8, 3.715, 0.9068, 0.00036])
V0 = -86.709


def ttp06_step(V, state, dt, pheno, gks_scale=None, gkr_scale=None):
    """One TTP06 step for n cells (FP64).  state (n,18) updated in place."""
    V = np.ascontiguousarray(V, np.float64)
    assert state.dtype == np.float64 and state.flags.c_contiguous
    pheno = np.ascontiguousarray(pheno, np.int8)
    n = V.shape[0]
    Iion = np.empty(n)
    gs = None if gks_scale is None else np.ascontiguousarray(gks_scale, np.float64)
    gr = None if gkr_scale is None else np.ascontiguousarray(gkr_scale, np.float64)
    lib().orc_ttp06_step(n, _p(V), _p(state), float(dt), _p(pheno), _p(gs), _p(gr), _p(Iion))
    return Iion


# --------------------------------------------------------------------------
# Geometry
# --------------------------------------------------------------------------

def discretise_tree(nodes_mm, elements, dx):
    """pipeline.py:88-114: subdivide every element into round(len/dx) segments."""
    nodes_mm = np.asarray(nodes_mm, np.float32)
    n0 = len(nodes_mm)
    extra, edges, bmaps = [], [], []
    counter = n0
    for e in elements:
        p0, p1 = nodes_mm[e[0]], nodes_mm[e[1]]
        n_seg = max(1, int(np.round(float(np.linalg.norm(p1 - p0)) / dx)))
        bm = [int(e[0])]
        for k in range(1, n_seg):
            t = k / n_seg
            extra.append(((1 - t) * p0 + t * p1).tolist())
            bm.append(counter)
            counter += 1
        bm.append(int(e[1]))
        bmaps.append(bm)
        edges += [[bm[i], bm[i + 1]] for i in range(len(bm) - 1)]
    comp = np.array(nodes_mm.tolist() + extra, dtype=np.float32)
    return comp, np.array(edges, dtype=np.int32).reshape(-1, 2), bmaps


def _edges_for_offset(vox, flat_to_node, shape, off):
    Nx, Ny, Nz = shape
    ni, nj, nk = vox[:, 0] + off[0], vox[:, 1] + off[1], vox[:, 2] + off[2]
    inb = (ni >= 0) & (ni < Nx) & (nj >= 0) & (nj < Ny) & (nk >= 0) & (nk < Nz)
    nf = np.where(inb, ni * Ny * Nz + nj * Nz + nk, 0).astype(np.int64)
    nb = flat_to_node[nf]
    valid = inb & (nb >= 0)
    return np.where(valid)[0].astype(np.int64), nb[valid].astype(np.int64)


def _mesh_common(S):
    shape = S.shape
    Nx, Ny, Nz = shape
    vox = np.argwhere(S == 1).astype(np.int64)
    N = len(vox)
    f2n = -np.ones(Nx * Ny * Nz, dtype=np.int64)
    f2n[vox[:, 0] * Ny * Nz + vox[:, 1] * Nz + vox[:, 2]] = np.arange(N)
    return vox, f2n, shape


def build_myo_mesh(S, h, sigma_M):
    """pipeline.py:761-833 (6-connected, uniform w = sigma_M * h)."""
    vox, f2n, shape = _mesh_common(S)
    a_l, b_l = [], []
    for off in [(1, 0, 0), (0, 1, 0), (0, 0, 1)]:
        a, b = _edges_for_offset(vox, f2n, shape, off)
        a_l.append(a); b_l.append(b)
    a = np.concatenate(a_l); b = np.concatenate(b_l)
    return dict(vox_idx=vox, edges=np.stack([a, b], 1),
                edge_w=np.full(len(a), sigma_M * h), shape=shape)


def conductivity_tensor(fibre_dir, vox, sl, st):
    """..._anisotropic_solver.py:856-883: D = st I + (sl - st) f f^T."""
    f = fibre_dir[vox[:, 0], vox[:, 1], vox[:, 2], :].astype(np.float64)
    ds = sl - st
    return (st + ds * f[:, 0] ** 2, st + ds * f[:, 1] ** 2, st + ds * f[:, 2] ** 2,
            ds * f[:, 0] * f[:, 1], ds * f[:, 0] * f[:, 2], ds * f[:, 1] * f[:, 2])


def build_myo_mesh_anisotropic(S, h, fibre_dir, sigma_l, sigma_t):
    """..._anisotropic_solver.py:886-1074 (18-connected signed weights).

    Face edges: harmonic mean of D_kk times h.  Edge-diagonal pairs:
    +/- arithmetic mean of D_ij times h/2 (co-signed / counter-signed)."""
    vox, f2n, shape = _mesh_common(S)
    D00, D11, D22, D01, D02, D12 = conductivity_tensor(fibre_dir, vox, sigma_l, sigma_t)
    a_l, b_l, w_l = [], [], []
    for Dkk, off in ((D00, (1, 0, 0)), (D11, (0, 1, 0)), (D22, (0, 0, 1))):
        a, b = _edges_for_offset(vox, f2n, shape, off)
        Da, Db = Dkk[a], Dkk[b]
        w_l.append(2.0 * Da * Db / np.maximum(Da + Db, 1e-30) * h)
        a_l.append(a); b_l.append(b)
    for Dij, o_same, o_diff in ((D01, (1, 1, 0), (1, -1, 0)),
                                (D02, (1, 0, 1), (1, 0, -1)),
                                (D12, (0, 1, 1), (0, 1, -1))):
        for off, sgn in ((o_same, 1.0), (o_diff, -1.0)):
            a, b = _edges_for_offset(vox, f2n, shape, off)
            w_l.append(sgn * 0.5 * (Dij[a] + Dij[b]) * h / 2.0)
            a_l.append(a); b_l.append(b)
    a = np.concatenate(a_l); b = np.concatenate(b_l)
    return dict(vox_idx=vox, edges=np.stack([a, b], 1),
                edge_w=np.concatenate(w_l), shape=shape)


def find_terminals(elements, n_nodes):
    """pipeline.py:915-920."""
    deg = np.zeros(n_nodes, np.int64)
    np.add.at(deg, elements[:, 0], 1)
    np.add.at(deg, elements[:, 1], 1)
    t = [i for i in range(1, n_nodes) if deg[i] == 1]
    return t if t else [n_nodes - 1]


def map_pmj(comp_nodes, pmj_ids, vox, h, n_pmj):
    """pipeline.py:888-909: n_pmj nearest myocardial nodes (xyz = col,row,depth)."""
    nodes_mm = vox[:, [1, 0, 2]].astype(np.float32) * h
    k = min(n_pmj, len(nodes_mm))
    _, nn = cKDTree(nodes_mm).query(comp_nodes[pmj_ids], k=k)
    if k == 1:
        nn = nn[:, None]
    return [row.tolist() for row in nn]


def global_laplacian(Np, N_myo, comp_edges, w_pp, Ai_P, myo_edges, myo_w, Ai_M,
                     pmj_ids, pmj_patches, c_pmj):
    """pipeline.py:578-651 / aniso :606-746.  L = D^-1 K (CSR, FP64)."""
    N = Np + N_myo
    rows, cols, vals = [], [], []
    ce = np.asarray(comp_edges, np.int64).reshape(-1, 2)
    rows += [ce[:, 0], ce[:, 1]]; cols += [ce[:, 1], ce[:, 0]]
    vals += [np.full(len(ce), w_pp)] * 2
    pr, pc, pv = [], [], []
    for p, patch in zip(pmj_ids, pmj_patches):
        w = c_pmj / len(patch)
        for m in patch:
            pr += [p, Np + m]; pc += [Np + m, p]; pv += [w, w]
    rows.append(np.array(pr, np.int64)); cols.append(np.array(pc, np.int64))
    vals.append(np.array(pv, np.float64))
    me = np.asarray(myo_edges, np.int64) + Np
    mw = np.asarray(myo_w, np.float64)
    rows += [me[:, 0], me[:, 1]]; cols += [me[:, 1], me[:, 0]]; vals += [mw, mw]
    r = np.concatenate(rows); c = np.concatenate(cols); v = np.concatenate(vals)
    deg = np.bincount(r, weights=v, minlength=N)
    r = np.concatenate([r, np.arange(N)]); c = np.concatenate([c, np.arange(N)])
    v = np.concatenate([v, -deg])
    Ai = np.empty(N); Ai[:Np] = Ai_P; Ai[Np:] = Ai_M
    v = v / Ai[r]
    return sp.csr_matrix((v, (r, c)), shape=(N, N))


def stim_active(t, onset, dur, period, n_pulses):
    """pipeline.py:1012-1023."""
    if t < onset:
        return False
    if not period:
        return t < onset + dur
    k = int((t - onset) // period)
    if n_pulses is not None and k >= n_pulses:
        return False
    return (t - onset) - k * period < dur


def resolve_stim_sites(stim_protocol, root_mask_p, ectopic_region, vox, Np,
                       stim_regions=None):
    """pipeline.py:947-1009 / aniso :1204-1288 -> list of (node_ids, site dict)."""
    root_ids = np.where(root_mask_p)[0]
    if ectopic_region is not None:
        ect = Np + np.where(ectopic_region[vox[:, 0], vox[:, 1], vox[:, 2]].astype(bool))[0]
    else:
        ect = np.array([], np.int64)
    regions = {}
    for name, m in (stim_regions or {}).items():
        regions[name] = Np + np.where(np.asarray(m)[vox[:, 0], vox[:, 1], vox[:, 2]].astype(bool))[0]
    out = []
    for ev in stim_protocol:
        tgt = ev.get("target", "root")
        if tgt == "root":
            ids = root_ids
        elif tgt == "ectopic":
            ids = ect
        elif tgt == "region":
            ids = regions[ev.get("region")]
        elif tgt == "custom":
            ids = np.asarray(ev["node_ids"], np.int64)
        else:
            raise ValueError(tgt)
        out.append((np.unique(np.asarray(ids, np.int64)),
                    dict(amp=float(ev["amp"]), dur=float(ev["dur"]),
                         onset=float(ev.get("onset", 0.0)),
                         period=ev.get("period", None) or None,
                         n_pulses=ev.get("n_pulses", None))))
    return out


def phenotypes(Np, phi_myo, phi_endo_max, phi_epi_min):
    """hetero_solver.py:74-128: 0 endo (all Purkinje), 1 mid, 2 epi."""
    phi = np.asarray(phi_myo).astype(np.float32)
    lo, hi = np.float32(phi_endo_max), np.float32(phi_epi_min)
    ph = np.ones(len(phi), np.int8)
    ph[phi < lo] = 0
    ph[phi >= hi] = 2
    return np.concatenate([np.zeros(Np, np.int8), ph])


# --------------------------------------------------------------------------
# Full run
# --------------------------------------------------------------------------

def setup(nodes, elements, act_times, S, phi, *, fibre_dir=None, voxel_size=0.4,
          dx_p=0.2, sigma_P=0.225, sigma_M=6.5625e-5, sigma_l=None, sigma_t=None,
          Cm=0.01, A_P=133.33, A_M=140.0, R_P=0.015, dt=0.02, T=10.0,
          stim_protocol=None, ectopic_region=None, stim_regions=None,
          stim_len_mm=2.0, c_pmj=0.05, n_pmj=1, phi_endo_max=0.35, phi_epi_min=0.65,
          vm_save_dt=None, gks_scale=1.0, gkr_scale=1.0, anisotropic=False,
          theta=0.0, cg_tol=1e-5, cg_max_iter=100):
    """Set-up of the reference method (theta = 0 the explicit update, theta >
    0 the theta-scheme): assembled L, phenotypes, stimulus schedule, resting
    state.  ``anisotropic=True`` follows the
    anisotropic solver (A_P = 2/R_P, fibre tensor, 18-connected mesh);
    otherwise run_coupled (A_P argument, uniform sigma_M)."""
    h = float(voxel_size)
    nodes_mm = np.asarray(nodes, np.float32) * h
    elements = np.asarray(elements, np.int64)
    comp, cedges, bmaps = discretise_tree(nodes_mm, elements, dx_p)
    Np = len(comp)
    act = np.array(act_times, np.float32)
    fin = np.isfinite(act)
    act[~fin] = T
    mn = float(act[fin].min())
    root = np.where(np.isclose(act, mn, atol=1e-6))[0]
    rpos = nodes_mm[root].mean(axis=0)
    d = np.linalg.norm(comp - rpos[None, :], axis=1)
    root_mask = d <= stim_len_mm
    if not root_mask.any():
        root_mask[int(d.argmin())] = True
    S_P = math.pi * R_P ** 2
    if anisotropic:
        A_P = 2.0 / R_P
    w_pp = sigma_P * S_P / dx_p
    Ai_P = A_P * S_P * dx_p
    Ai_M = A_M * h ** 3
    if anisotropic:
        myo = build_myo_mesh_anisotropic(S, h, fibre_dir, sigma_l, sigma_t)
    else:
        myo = build_myo_mesh(S, h, sigma_M)
    vox = myo["vox_idx"]
    N_myo = len(vox)
    phi_myo = phi[vox[:, 0], vox[:, 1], vox[:, 2]].astype(np.float32)
    phi_myo = np.where(np.isfinite(phi_myo), phi_myo, 0.5)
    terms = set(find_terminals(elements, len(nodes_mm)))
    pmj_ids = sorted({bm[-1] for i, bm in enumerate(bmaps) if elements[i][1] in terms})
    if not pmj_ids:
        pmj_ids = [Np - 1]
    patches = map_pmj(comp, pmj_ids, vox, h, n_pmj)
    L = global_laplacian(Np, N_myo, cedges, w_pp, Ai_P, myo["edges"], myo["edge_w"],
                         Ai_M, pmj_ids, patches, c_pmj)
    N = Np + N_myo
    pheno = phenotypes(Np, phi_myo, phi_endo_max, phi_epi_min)
    n_steps = int(T / dt)
    if stim_protocol is None:
        stim_protocol = [dict(name="av_node", target="root", amp=12.0, dur=2.0, onset=0.0)]
    sites = resolve_stim_sites(stim_protocol, root_mask, ectopic_region, vox, Np, stim_regions)
    snap_every = max(1, int(round(vm_save_dt / dt))) if vm_save_dt else 1
    Lc = L.tocsr()
    Lc.sort_indices()
    return dict(L=L, ptr=Lc.indptr.astype(np.int64), idx=Lc.indices.astype(np.int32),
                val=Lc.data.astype(np.float64), N=N, Np=Np, pheno=pheno, sites=sites,
                dt=float(dt), Cm=float(Cm), n_steps=n_steps, snap_every=snap_every,
                V=np.full(N, V0), state=np.tile(TTP06_INIT, (N, 1)),
                gks=np.full(N, float(gks_scale)), gkr=np.full(N, float(gkr_scale)),
                step=0, theta=float(theta), cg_tol=float(cg_tol), cg_max_iter=int(cg_max_iter),
                cg_iters=0, Ai_P=Ai_P, Ai_M=Ai_M,
                vox_idx=vox, comp_nodes=comp, comp_edges=cedges, branch_map=bmaps,
                pmj_ids=pmj_ids, pmj_patches=patches)


def advance(ctx, n_steps, snapshots=True):
    """Runs n_steps more time steps (C time loop); returns (Vm, Vp, times)
    snapshots taken in this call (float32), labelled t = step * dt."""
    sites = ctx["sites"]
    nS = len(sites)
    dt, k0 = ctx["dt"], ctx["step"]
    site_ptr = np.zeros(nS + 1, np.int64)
    site_ptr[1:] = np.cumsum([len(s[0]) for s in sites])
    site_nodes = (np.concatenate([s[0] for s in sites]).astype(np.int32)
                  if nS else np.zeros(0, np.int32))
    site_amp = np.array([s[1]["amp"] for s in sites], np.float64)
    on = np.zeros((max(n_steps, 1), max(nS, 1)), np.uint8)
    for k in range(n_steps):
        t = (k0 + k) * dt
        for s, (_, st) in enumerate(sites):
            on[k, s] = stim_active(t, st["onset"], st["dur"], st["period"], st["n_pulses"])
    se = ctx["snap_every"]
    N, Np = ctx["N"], ctx["Np"]
    # snapshot steps of this call, in global step numbering
    first = (-k0) % se
    n_snap = len(range(first, n_steps, se)) if snapshots else 0
    snaps = np.zeros((max(n_snap, 1), N - Np), np.float32)
    psnaps = np.zeros((max(n_snap, 1), Np), np.float32)
    if snapshots and k0 % se != 0 and n_snap:
        raise ValueError("advance() must start on a snapshot boundary when snapshots are on")
    args = (N, Np, _p(ctx["ptr"]), _p(ctx["idx"]), _p(ctx["val"]),
            _p(ctx["pheno"]), _p(ctx["gks"]), _p(ctx["gkr"]), dt, ctx["Cm"],
            n_steps, nS, _p(site_ptr), _p(site_nodes), _p(site_amp), _p(on),
            _p(ctx["V"]), _p(ctx["state"]), se if snapshots else 0,
            _p(snaps), _p(psnaps))
    if ctx.get("theta", 0.0) == 0.0:
        rc = lib().orc_mono_run(*args)
    else:
        it = np.zeros(1, np.int64)
        rc = lib().orc_mono_run_cn(*args, ctx["theta"], ctx["cg_tol"], ctx["cg_max_iter"],
                                   _p(it))
        ctx["cg_iters"] += int(it[0])
    if rc != 0:
        raise RuntimeError(f"orc_mono_run failed ({rc})")
    ctx["step"] = k0 + n_steps
    times = np.array([(k0 + k) * dt for k in range(first, n_steps, se)], np.float32)
    return snaps[:n_snap], psnaps[:n_snap], times


def advance_events(ctx, n_steps, act_threshold=-20.0, frame_every=0, chunk=250):
    """Runs n_steps more time steps and records, in the loop, the first
    upward crossing of ``act_threshold`` of every myocardial node between
    consecutive post-step states, interpolated as activation_maps.py:63-89
    does (float32, den == 0 -> 1e-9, frac clipped to [0, 1]); the same as
    compute_activation_maps on snapshots saved every step
    (activation_maps.py:295-350), without holding them all: the steps run in
    chunks of ``chunk`` with every-step snapshots.  Returns (first
    activation time per myocardial node, NaN where none; Vm frames at the
    global steps that are multiples of ``frame_every`` (None if 0); their
    times).  The crossing state carries over between calls through ctx;
    ctx["_adv_seconds"] accumulates the wall time of the time loop alone
    (the C calls, without the crossing bookkeeping)."""
    import time
    N_myo = ctx["N"] - ctx["Np"]
    first = ctx.setdefault("_act_first", np.full(N_myo, np.nan, np.float32))
    thr = np.float32(act_threshold)
    se0 = ctx["snap_every"]
    ctx["snap_every"] = 1
    frames, ftimes = [], []
    try:
        done = 0
        while done < n_steps:
            n = min(chunk, n_steps - done)
            t0 = time.perf_counter()
            Vm, _, t = advance(ctx, n, snapshots=True)
            ctx["_adv_seconds"] = ctx.get("_adv_seconds", 0.0) + time.perf_counter() - t0
            prev = ctx.get("_act_prev")
            if prev is not None:
                Vm2 = np.concatenate([prev[0][None], Vm])
                t2 = np.concatenate([np.array([prev[1]], np.float32), t])
            else:
                Vm2, t2 = Vm, t
            above = Vm2 >= thr
            rising = np.diff(above.astype(np.int8), axis=0) == 1
            fi, ni = np.nonzero(rising)
            if fi.size:
                Vi, Vj = Vm2[fi, ni], Vm2[fi + 1, ni]
                den = Vj - Vi
                den = np.where(den == 0, np.float32(1e-9), den)
                frac = np.clip((thr - Vi) / den, 0.0, 1.0)
                tc = (t2[fi] + frac * (t2[fi + 1] - t2[fi])).astype(np.float32)
                # first crossing per node: fi ascends within the chunk
                order = np.lexsort((fi, ni))
                ni_o, tc_o = ni[order], tc[order]
                uniq, pos = np.unique(ni_o, return_index=True)
                new = np.isnan(first[uniq])
                first[uniq[new]] = tc_o[pos][new]
            ctx["_act_prev"] = (Vm[-1].copy(), np.float32(t[-1]))
            if frame_every:
                k0 = ctx["step"] - n
                sel = [r for r in range(n) if (k0 + r) % frame_every == 0]
                if sel:
                    frames.append(Vm[sel])
                    ftimes.append(t[sel])
            done += n
    finally:
        ctx["snap_every"] = se0
    fr = np.concatenate(frames) if frames else None
    ft = np.concatenate(ftimes) if ftimes else None
    return first.copy(), fr, ft


def run(nodes, elements, act_times, S, phi, **kw):
    """Full FP64 run of the reference method from rest.  Returns
    ``Vm`` (n_snap, N_myo) float32, ``time_vm``, ``Vp`` Purkinje snapshots,
    final ``V``/``state`` and the set-up bookkeeping."""
    ctx = setup(nodes, elements, act_times, S, phi, **kw)
    Vm, Vp, t = advance(ctx, ctx["n_steps"])
    out = dict(ctx)
    out.update(Vm=Vm, Vp=Vp, time_vm=t)
    return out


def activation_maps(Vm, t, act_threshold=-40.0, deact_threshold=-40.0):
    """activation_maps.py:63-116,295-350: every threshold crossing, linearly
    interpolated between consecutive snapshots (float32), NaN-padded."""
    Vm = np.asarray(Vm, np.float32)
    t = np.asarray(t, np.float32)
    N = Vm.shape[1]

    def crossings(mask, thr):
        fi, ni = np.nonzero(mask)
        if fi.size == 0:
            return np.zeros((N, 0), np.float32), np.zeros(N, np.int32)
        Vi, Vj = Vm[fi, ni], Vm[fi + 1, ni]
        den = Vj - Vi
        den = np.where(den == 0, np.float32(1e-9), den)
        frac = np.clip((np.float32(thr) - Vi) / den, 0.0, 1.0)
        tc = (t[fi] + frac * (t[fi + 1] - t[fi])).astype(np.float32)
        order = np.argsort(ni, kind="stable")
        ni, tc = ni[order], tc[order]
        cnt = np.bincount(ni, minlength=N)
        starts = np.cumsum(cnt) - cnt
        pos = np.arange(len(ni)) - np.repeat(starts, cnt)
        out = np.full((N, int(cnt.max())), np.nan, np.float32)
        out[ni, pos] = tc
        return out, cnt.astype(np.int32)

    above = Vm >= np.float32(act_threshold)
    rising = np.diff(above.astype(np.int8), axis=0) == 1
    act, n_act = crossings(rising, act_threshold)
    above_d = Vm >= np.float32(deact_threshold)
    falling = np.diff(above_d.astype(np.int8), axis=0) == -1
    deact, n_deact = crossings(falling, deact_threshold)
    return dict(activation_times=act, n_activations=n_act,
                deactivation_times=deact, n_deactivations=n_deact)
