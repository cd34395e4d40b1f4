"""Monodomain driver: the reference's run_coupled / anisotropic solver set-up
restated on the host, the time loop on the GPU through libhrdaya_b200.

Set-up follows simulation/functions/purkinje_myocardium_pipeline.py:1030-1345
and anisotropic_simulation/functions/purkinje_myocardium_anisotropic_solver.py
:1308-1745 (tree discretisation, root stimulus zone, membrane loading, PMJ
mapping, phenotype assignment, stimulus sites); the time loop (:1347-1420 /
:1746-1820) is hp_mono_run.  theta = 0 is the explicit update of the
fused step kernels; 0 < theta <= 1 (the reference's default is 0.5) solves
the theta-scheme diffusion half on the GPU each step by preconditioned CG
(stopping rule and iteration cap as the reference's BiCGSTAB: cg_tol,
cg_max_iter).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import tempfile
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _lib
from .layout import (TAG_PMJ, TAG_STIM_SHIFT, TAG_SURF, BrickLayout, aniso_coefficients,
                     build_layout, surface_nodes)

V0_REST = -86.709          # hetero_solver.py:82 (HeteroIonicSolver V0)
DEFAULT_BRICK = (4, 4, 8)


# --------------------------------------------------------------------------
# Purkinje tree helpers (same arithmetic as the reference, so node ids and
# coordinates match it exactly)
# --------------------------------------------------------------------------

def discretise_tree(nodes_mm: np.ndarray, elements: np.ndarray, dx: float):
    """Subdivide each element into max(1, round(len / dx)) segments.
    Original nodes keep their ids; new nodes are appended element by element
    (pipeline.py:88-114)."""
    nodes_mm = np.asarray(nodes_mm, np.float32)
    extra = []
    edges = []
    bmaps = []
    counter = len(nodes_mm)
    for e in np.asarray(elements):
        a, b = int(e[0]), int(e[1])
        p0, p1 = nodes_mm[a], nodes_mm[b]
        n_seg = max(1, int(np.round(float(np.linalg.norm(p1 - p0)) / dx)))
        bm = [a]
        for k in range(1, n_seg):
            t = k / n_seg
            extra.append((1 - t) * p0 + t * p1)
            bm.append(counter)
            counter += 1
        bm.append(b)
        bmaps.append(bm)
        edges.extend(zip(bm[:-1], bm[1:]))
    comp = np.concatenate([nodes_mm, np.asarray(extra, np.float32).reshape(-1, 3)])
    return comp.astype(np.float32), np.asarray(edges, np.int32).reshape(-1, 2), bmaps


def find_terminals(elements: np.ndarray, n_nodes: int):
    deg = np.bincount(np.asarray(elements).ravel(), minlength=n_nodes)
    t = np.where(deg[1:] == 1)[0] + 1
    return t.tolist() if len(t) else [n_nodes - 1]


def clip_purkinje_outside_Z(comp_nodes, comp_edges, Z, h):
    """Edges drawn outside the cut mask only (animation output,
    ..._anisotropic_solver.py:1107-1137, with its axis-bound fix)."""
    Nx, Ny, Nz = Z.shape
    v = np.clip(np.round(comp_nodes / h).astype(np.int32), [0, 0, 0], [Ny - 1, Nx - 1, Nz - 1])
    v = v[:, [1, 0, 2]]
    outside = ~np.asarray(Z)[v[:, 0], v[:, 1], v[:, 2]].astype(bool)
    keep = outside[comp_edges[:, 0]] & outside[comp_edges[:, 1]]
    return comp_edges[keep]


def stim_active(t, onset, dur, period, n_pulses) -> bool:
    """pipeline.py:1012-1023."""
    if t < onset:
        return False
    if not period:
        return t < onset + dur
    k = int((t - onset) // period)
    if n_pulses is not None and k >= n_pulses:
        return False
    return (t - onset) - k * period < dur


# --------------------------------------------------------------------------
# Problem description
# --------------------------------------------------------------------------

@dataclass
class MonoProblem:
    """Everything hp_mono_create needs, as host numpy arrays."""
    layout: BrickLayout
    tag: np.ndarray
    wface: np.ndarray | None
    doff: np.ndarray | None
    iso_coef: float
    anisotropic: bool
    pk_ptr: np.ndarray
    pk_idx: np.ndarray
    pk_coef: np.ndarray
    pk_stim: np.ndarray
    pmj_row: np.ndarray
    pmj_ptr: np.ndarray
    pmj_pk: np.ndarray
    pmj_coef: np.ndarray
    dt: float
    Cm: float
    n_steps: int
    site_amp: np.ndarray
    site_on: np.ndarray
    vm_every: int
    frame_every: int
    surf_nodes: np.ndarray
    surf_of_slot: np.ndarray
    act_threshold: float = -40.0
    deact_threshold: float = -40.0
    max_events: int = 4
    v0: float = V0_REST
    brick_variant: np.ndarray | None = None
    pk_variant: np.ndarray | None = None
    variant_gks: np.ndarray | None = None
    variant_gkr: np.ndarray | None = None
    kernel: int = 0          # HP_MONO_KERNEL_AUTO / _BRICK (1) / _PIPELINED (2) / _SPLIT (3)
    theta: float = 0.0       # 0 explicit diffusion half, (0, 1] theta-scheme (CG)
    cn_tol: float = 1e-5     # relative residual of the theta-scheme solve
    cn_max_iter: int = 100
    pk_weight: float = 1.0   # Ai_P / Ai_M

    @property
    def n_pk(self):
        return len(self.pk_ptr) - 1

    @property
    def n_myo(self):
        return len(self.layout.slot_of_node)


class MonoHandle:
    """Owns one hp_mono handle (device state of one problem)."""

    def __init__(self, prob: MonoProblem, stream=None):
        torch = _lib.require_cuda()
        L = _lib.lib()
        self.prob = prob
        lay = prob.layout
        self._keep = []

        def k(a, dtype):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=dtype)
            self._keep.append(a)
            return _lib.ptr(a)

        d = _lib.HpMonoDesc()
        d.n_bricks = lay.n_bricks
        d.bi, d.bj, d.bk = lay.brick
        d.anisotropic = int(prob.anisotropic)
        d.brick_nbr = k(lay.brick_nbr, np.int32)
        d.tag = k(prob.tag, np.uint32)
        d.wface = k(prob.wface, np.float32)
        d.doff = k(prob.doff, np.float32)
        d.iso_coef = float(prob.iso_coef)
        nvar = 1 if prob.variant_gks is None else len(prob.variant_gks)
        d.brick_variant = k(prob.brick_variant, np.uint8)
        d.n_variants = nvar
        d.variant_gks = k(np.ones(1) if prob.variant_gks is None else prob.variant_gks, np.float32)
        d.variant_gkr = k(np.ones(1) if prob.variant_gkr is None else prob.variant_gkr, np.float32)
        d.n_pk = prob.n_pk
        d.pk_ptr = k(prob.pk_ptr, np.int32)
        d.pk_idx = k(prob.pk_idx, np.int32)
        d.pk_coef = k(prob.pk_coef, np.float32)
        d.pk_stim = k(prob.pk_stim, np.uint8)
        d.pk_variant = k(prob.pk_variant, np.uint8)
        d.n_pmj_rows = len(prob.pmj_ptr) - 1
        d.pmj_row = k(prob.pmj_row, np.int32)
        d.pmj_ptr = k(prob.pmj_ptr, np.int32)
        d.pmj_pk = k(prob.pmj_pk, np.int32)
        d.pmj_coef = k(prob.pmj_coef, np.float32)
        d.dt = float(prob.dt)
        d.Cm = float(prob.Cm)
        d.v0 = float(prob.v0)
        d.n_steps = int(prob.n_steps)
        # site tables: (n_sites,) / (n_steps + 1,) for one heart, one row per
        # variant for an ensemble
        amp = np.atleast_2d(np.asarray(prob.site_amp, np.float32))
        on = np.atleast_2d(np.asarray(prob.site_on, np.uint8))
        if amp.shape[0] != nvar or on.shape != (nvar, prob.n_steps + 1):
            raise ValueError(f"site tables {amp.shape} / {on.shape} do not match {nvar} variants "
                             f"and {prob.n_steps} steps")
        d.n_sites = amp.shape[1]
        d.site_amp = k(amp if amp.size else np.zeros((nvar, 1)), np.float32)
        d.site_on = k(on, np.uint8)
        d.n_myo = prob.n_myo
        d.slot_of_node = k(lay.slot_of_node, np.int32)
        d.vm_every = int(prob.vm_every)
        d.n_surf = len(prob.surf_nodes)
        d.surf_of_slot = k(prob.surf_of_slot, np.int32)
        d.frame_every = int(prob.frame_every)
        d.act_threshold = float(prob.act_threshold)
        d.deact_threshold = float(prob.deact_threshold)
        d.max_events = int(prob.max_events)
        d.kernel = int(prob.kernel)
        d.theta = float(prob.theta)
        d.cn_tol = float(prob.cn_tol)
        d.cn_max_iter = int(prob.cn_max_iter)
        d.pk_weight = float(prob.pk_weight)
        self._desc = d
        if stream is None:
            # a dedicated stream: CUDA graphs cannot capture the legacy stream
            self._torch_stream = torch.cuda.Stream()
            stream = C.c_void_p(self._torch_stream.cuda_stream)
        self.stream = stream
        h = C.c_void_p()
        _lib.check(L.hp_mono_create(C.byref(d), C.byref(h), self.stream), "hp_mono_create")
        self.h = h
        self._keep = []   # create() synchronised: host arrays no longer needed
        self.n_vm_frames = ((prob.n_steps + prob.vm_every - 1) // prob.vm_every
                            if prob.vm_every > 0 else 0)
        self.n_anim_frames = ((prob.n_steps + prob.frame_every - 1) // prob.frame_every
                              if prob.frame_every > 0 else 0)

    # ---------------------------------------------------------------
    def run(self, n: int, graph_chunk: int = 50):
        _lib.check(_lib.lib().hp_mono_run(self.h, int(n), int(graph_chunk), self.stream),
                   "hp_mono_run")

    def cn_stats(self):
        """Theta-scheme counters: (CG iterations, solves, solves stopped by
        the iteration cap, breakdowns); zeros at theta = 0."""
        v = [C.c_int64() for _ in range(4)]
        _lib.check(_lib.lib().hp_mono_cn_stats(self.h, *[C.byref(x) for x in v]),
                   "hp_mono_cn_stats")
        return tuple(int(x.value) for x in v)

    def kernel_info(self):
        """(kernel id, grid CTAs, dynamic shared memory bytes) of the step."""
        k, g, sm = C.c_int32(), C.c_int32(), C.c_int64()
        _lib.check(_lib.lib().hp_mono_kernel_info(self.h, C.byref(k), C.byref(g), C.byref(sm)),
                   "hp_mono_kernel_info")
        return int(k.value), int(g.value), int(sm.value)

    @property
    def steps_done(self) -> int:
        return int(_lib.lib().hp_mono_steps_done(self.h))

    def vm_frames(self, f0=0, nf=None, out=None):
        nf = self.n_vm_frames - f0 if nf is None else nf
        if out is None:
            out = np.empty((nf, self.prob.n_myo), np.float32)
        _lib.check(_lib.lib().hp_mono_copy_vm(self.h, f0, nf, _lib.ptr(out), 0, self.stream),
                   "hp_mono_copy_vm")
        self.sync()
        return out

    def vm_frames_async(self, f0, nf, out):
        """Starts the device-to-host copy of snapshots [f0, f0 + nf) into out
        ((nf, n_myo) float32 in pinned host memory: a torch tensor made with
        pin_memory=True, or a numpy view of one) and returns at once.  The
        copy runs on a copy stream of this handle, ordered after every step
        enqueued so far, so the steps enqueued next overlap it; each frame
        has its own device slot, which later steps never overwrite.  out
        holds the frames once wait_copies() returns.  A handle made on a
        caller's stream queues the copy on that stream instead (no overlap)."""
        import torch
        nf = int(nf)
        ptr = C.c_void_p(out.data_ptr()) if hasattr(out, "data_ptr") else _lib.ptr(out)
        if tuple(out.shape) != (nf, self.prob.n_myo) and not (nf == 1 and tuple(out.shape) ==
                                                              (self.prob.n_myo,)):
            raise ValueError(f"out has shape {tuple(out.shape)}, expected ({nf}, "
                             f"{self.prob.n_myo})")
        stream = self.stream
        own = getattr(self, "_torch_stream", None)
        if own is not None:
            if getattr(self, "_copy_stream", None) is None:
                self._copy_stream = torch.cuda.Stream()
            ev = torch.cuda.Event()
            ev.record(own)
            self._copy_stream.wait_event(ev)
            stream = C.c_void_p(self._copy_stream.cuda_stream)
        _lib.check(_lib.lib().hp_mono_copy_vm(self.h, int(f0), nf, ptr, 0, stream),
                   "hp_mono_copy_vm")

    def wait_copies(self):
        """Blocks until every copy started by vm_frames_async has landed."""
        cs = getattr(self, "_copy_stream", None)
        if cs is not None:
            cs.synchronize()
        elif getattr(self, "_torch_stream", None) is None:
            self.sync()

    def vm_frames_device(self, dst_ptr: int, f0: int, nf: int):
        _lib.check(_lib.lib().hp_mono_copy_vm(self.h, f0, nf, C.c_void_p(dst_ptr), 1, self.stream),
                   "hp_mono_copy_vm")

    def anim_frames(self):
        nf = self.n_anim_frames
        surf = np.empty((nf, len(self.prob.surf_nodes)), np.float32)
        pk = np.empty((nf, self.prob.n_pk), np.float32)
        _lib.check(_lib.lib().hp_mono_copy_frames(self.h, 0, nf, _lib.ptr(surf), _lib.ptr(pk), 0,
                                                  self.stream), "hp_mono_copy_frames")
        self.sync()
        return surf, pk

    def events(self):
        me, nm = self.prob.max_events, self.prob.n_myo
        act = np.empty((me, nm), np.float32)
        nact = np.empty(nm, np.int32)
        dea = np.empty((me, nm), np.float32)
        ndea = np.empty(nm, np.int32)
        _lib.check(_lib.lib().hp_mono_copy_events(self.h, _lib.ptr(act), _lib.ptr(nact),
                                                  _lib.ptr(dea), _lib.ptr(ndea), self.stream),
                   "hp_mono_copy_events")
        return act, nact, dea, ndea

    def voltage(self):
        vm = np.empty(self.prob.n_myo, np.float32)
        vp = np.empty(max(self.prob.n_pk, 1), np.float32)
        _lib.check(_lib.lib().hp_mono_copy_v(self.h, _lib.ptr(vm), _lib.ptr(vp), self.stream),
                   "hp_mono_copy_v")
        return vm, vp[: self.prob.n_pk]

    def state(self):
        lay = self.prob.layout
        st = np.empty((18, lay.n_slots), np.float32)
        sp = np.empty((18, max(self.prob.n_pk, 1)), np.float32)
        _lib.check(_lib.lib().hp_mono_copy_state(self.h, _lib.ptr(st), _lib.ptr(sp), self.stream),
                   "hp_mono_copy_state")
        return st[:, lay.slot_of_node], sp[:, : self.prob.n_pk]

    def sync(self):
        import torch
        torch.cuda.synchronize()

    def close(self):
        if getattr(self, "h", None):
            self.wait_copies()   # no copy may read the snapshots once they are freed
            _lib.lib().hp_mono_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------------
# Set-up shared by the isotropic and anisotropic drop-ins
# --------------------------------------------------------------------------

def prepare(nodes, elements, activation_times, S, Z, phi, *, fibre_dir=None,
            anisotropic=False, voxel_size=0.4, dx_p=0.2, sigma_P=0.225,
            sigma_M=6.5625e-5, sigma_l=None, sigma_t=None, Cm=0.01, A_P=133.33,
            A_M=0.14, R_P=0.015, dt=0.1, T=400.0, stim_protocol=None,
            ectopic_region=None, stim_regions=None, stim_len_mm=2.0, c_pmj=0.05,
            n_pmj=1, phi_endo_max=0.35, phi_epi_min=0.65, vm_save_dt=None,
            save_every=None, act_threshold=-40.0, deact_threshold=-40.0,
            max_events=4, brick=None, theta=0.0, cg_tol=1e-5, cg_max_iter=100,
            verbose=False):
    """Builds the MonoProblem and the bookkeeping the result dict needs."""
    if not 0.0 <= float(theta) <= 1.0:
        raise ValueError(f"theta={theta} must lie in [0, 1]")
    h = float(voxel_size)
    S = np.asarray(S)
    Z = np.asarray(Z) if Z is not None else S
    brick = tuple(brick or DEFAULT_BRICK)
    nodes_mm = np.asarray(nodes, np.float32) * np.float32(h)
    elements = np.asarray(elements, np.int64).reshape(-1, 2)
    comp, cedges, bmaps = discretise_tree(nodes_mm, elements, dx_p)
    Np = len(comp)

    # AV-node stimulus zone (pipeline.py:1147-1158)
    act = np.array(activation_times, dtype=np.float32)
    fin = np.isfinite(act)
    act[~fin] = T
    mn = float(act[fin].min())
    root = np.where(np.isclose(act, mn, atol=1e-6))[0]
    rpos = nodes_mm[root].mean(axis=0)
    dists = np.linalg.norm(comp - rpos[None, :], axis=1)
    root_mask = dists <= stim_len_mm
    if not root_mask.any():
        root_mask[int(dists.argmin())] = True

    S_P = math.pi * R_P ** 2
    w_pp = sigma_P * S_P / dx_p
    Ai_P = A_P * S_P * dx_p
    Ai_M = A_M * h ** 3
    dtc = dt / Cm

    lay = build_layout(S, brick, anisotropic)
    vox = lay.vox_idx
    N_myo = len(vox)
    if anisotropic:
        scale = dtc / Ai_M * h  # dt/(Cm A_M h^2)
        wface, doff = aniso_coefficients(lay, S, fibre_dir, sigma_l, sigma_t, scale)
        iso_coef = 0.0
    else:
        wface = doff = None
        iso_coef = dtc * (sigma_M * h) / Ai_M

    # phenotypes (hetero_solver.py:97-101 on float32 phi, NaN -> 0.5)
    phi_myo = np.asarray(phi)[vox[:, 0], vox[:, 1], vox[:, 2]].astype(np.float32)
    phi_myo = np.where(np.isfinite(phi_myo), phi_myo, np.float32(0.5))
    ph = np.full(N_myo, 2, np.uint32)
    ph[phi_myo < np.float32(phi_endo_max)] = 1
    ph[phi_myo >= np.float32(phi_epi_min)] = 3
    tag_node = ph | lay.nbr_bits

    # junctions (pipeline.py:1182-1209, map_pmj :888-909)
    terms = set(find_terminals(elements, len(nodes_mm)))
    pmj_ids = sorted({bm[-1] for i, bm in enumerate(bmaps) if int(elements[i][1]) in terms})
    if not pmj_ids:
        pmj_ids = [Np - 1]
    from scipy.spatial import cKDTree
    myo_xyz = vox[:, [1, 0, 2]].astype(np.float32) * np.float32(h)
    kq = min(int(n_pmj), N_myo)
    _, nn = cKDTree(myo_xyz).query(comp[pmj_ids], k=kq)
    nn = np.asarray(nn).reshape(len(pmj_ids), kq)

    # Purkinje CSR: cable edges then junction edges, coefficient dt/(Cm Ai_P) w
    rows = [cedges[:, 0], cedges[:, 1]]
    cols = [cedges[:, 1], cedges[:, 0]]
    vals = [np.full(len(cedges), dtc * w_pp / Ai_P)] * 2
    jp = np.repeat(np.asarray(pmj_ids, np.int64), kq)
    jm = nn.reshape(-1).astype(np.int64)
    w_pmj = c_pmj / kq
    rows.append(jp)
    cols.append(-(lay.slot_of_node[jm].astype(np.int64)) - 1)
    vals.append(np.full(len(jp), dtc * w_pmj / Ai_P))
    r = np.concatenate(rows).astype(np.int64)
    c = np.concatenate(cols).astype(np.int64)
    v = np.concatenate(vals)
    o = np.argsort(r, kind="stable")
    pk_ptr = np.zeros(Np + 1, np.int64)
    pk_ptr[1:] = np.cumsum(np.bincount(r, minlength=Np))
    pk_idx, pk_coef = c[o], v[o]
    # myocardial side: rows per junction voxel
    pm_nodes, pm_inv = np.unique(jm, return_inverse=True)
    o2 = np.argsort(pm_inv, kind="stable")
    pmj_ptr = np.zeros(len(pm_nodes) + 1, np.int64)
    pmj_ptr[1:] = np.cumsum(np.bincount(pm_inv, minlength=len(pm_nodes)))
    pmj_pk = jp[o2]
    pmj_coef = np.full(len(jp), dtc * w_pmj / Ai_M)
    pmj_row_node = np.full(N_myo, -1, np.int64)
    if c_pmj != 0.0:
        pmj_row_node[pm_nodes] = np.arange(len(pm_nodes))
        tag_node[pm_nodes] |= np.uint32(TAG_PMJ)
    else:   # zero conductance: junction terms vanish, skip them entirely
        pmj_ptr = np.zeros(1, np.int64)
        pmj_pk = np.zeros(0, np.int64)
        pmj_coef = np.zeros(0)
        keep = pk_idx >= 0
        cnt = np.bincount(r[o][keep], minlength=Np)
        pk_ptr = np.zeros(Np + 1, np.int64)
        pk_ptr[1:] = np.cumsum(cnt)
        pk_idx, pk_coef = pk_idx[keep], pk_coef[keep]

    # stimulus sites (pipeline.py:947-1009, aniso :1204-1288)
    if stim_protocol is None:
        stim_protocol = [dict(name="av_node", target="root", amp=12.0, dur=2.0, onset=0.0)]
    if len(stim_protocol) > _lib.HP_MAX_SITES:
        raise ValueError(f"at most {_lib.HP_MAX_SITES} stimulus sites are supported")
    pk_stim = np.zeros(Np, np.uint8)
    root_ids = np.where(root_mask)[0]
    ect = (np.where(np.asarray(ectopic_region)[vox[:, 0], vox[:, 1], vox[:, 2]].astype(bool))[0]
           if ectopic_region is not None else np.zeros(0, np.int64))
    regions = {}
    for name, m in (stim_regions or {}).items():
        regions[name] = np.where(np.asarray(m)[vox[:, 0], vox[:, 1], vox[:, 2]].astype(bool))[0]
    sites = []
    for s_i, ev in enumerate(stim_protocol):
        tgt = ev.get("target", "root")
        bit = np.uint32(1 << (TAG_STIM_SHIFT + s_i))
        if tgt == "root":
            pk_stim[root_ids] |= np.uint8(1 << s_i)
        elif tgt == "ectopic":
            tag_node[ect] |= bit
        elif tgt == "region":
            rn = ev.get("region")
            if rn not in regions:
                raise ValueError(f"Stimulus '{ev.get('name', tgt)}' has target='region' with "
                                 f"region={rn!r}, but stim_regions only defines {sorted(regions)}.")
            tag_node[regions[rn]] |= bit
        elif tgt == "custom":
            ids = np.asarray(ev["node_ids"], np.int64)
            pk_stim[ids[ids < Np]] |= np.uint8(1 << s_i)
            tag_node[ids[ids >= Np] - Np] |= bit
        else:
            raise ValueError(f"Unknown stimulus target '{tgt}' (expected 'root', 'ectopic', "
                             "'region', or 'custom').")
        sites.append(dict(amp=float(ev["amp"]), dur=float(ev["dur"]),
                          onset=float(ev.get("onset", 0.0)),
                          period=ev.get("period", None) or None,
                          n_pulses=ev.get("n_pulses", None)))
    n_steps = int(T / dt)
    site_on = np.zeros(n_steps + 1, np.uint8)
    for kk in range(n_steps + 1):
        t = kk * dt
        m = 0
        for s_i, st in enumerate(sites):
            if stim_active(t, st["onset"], st["dur"], st["period"], st["n_pulses"]):
                m |= 1 << s_i
        site_on[kk] = m

    # outputs
    vm_every = max(1, int(round(vm_save_dt / dt))) if vm_save_dt else 0
    frame_every = int(save_every) if save_every else 0
    surf = surface_nodes(S, Z, vox)
    surf_of_node = np.full(N_myo, -1, np.int32)
    surf_of_node[surf] = np.arange(len(surf), dtype=np.int32)
    if frame_every:
        tag_node[surf] |= np.uint32(TAG_SURF)

    prob = MonoProblem(
        layout=lay, tag=lay.to_slots(tag_node, 0, np.uint32), wface=wface, doff=doff,
        iso_coef=iso_coef, anisotropic=anisotropic,
        pk_ptr=pk_ptr.astype(np.int32), pk_idx=pk_idx.astype(np.int32),
        pk_coef=pk_coef.astype(np.float32), pk_stim=pk_stim,
        pmj_row=lay.to_slots(pmj_row_node, -1, np.int32), pmj_ptr=pmj_ptr.astype(np.int32),
        pmj_pk=pmj_pk.astype(np.int32), pmj_coef=pmj_coef.astype(np.float32),
        dt=dt, Cm=Cm, n_steps=n_steps, site_amp=np.array([s["amp"] for s in sites], np.float32),
        site_on=site_on, vm_every=vm_every, frame_every=frame_every, surf_nodes=surf,
        surf_of_slot=lay.to_slots(surf_of_node, -1, np.int32), act_threshold=act_threshold,
        deact_threshold=deact_threshold, max_events=max_events, theta=float(theta),
        cn_tol=float(cg_tol), cn_max_iter=int(cg_max_iter), pk_weight=float(Ai_P / Ai_M))
    info = dict(comp_nodes=comp, comp_edges_full=cedges,
                comp_edges=clip_purkinje_outside_Z(comp, cedges, Z, h), branch_map=bmaps,
                vox_idx=vox, nodes_mm=myo_xyz, Np=Np, pmj_ids=pmj_ids,
                pmj_patches=nn.tolist(), surface_node_ids=surf, root_mask=root_mask)
    return prob, info


def save_vm_snapshots(path, node_ids, coords_mm, vox_idx, Vm, times, dt_solver, vm_save_dt):
    """Same schema as the reference's _save_vm_snapshots (pipeline.py:1500-1570)."""
    path = Path(path).with_suffix(".npz")
    path.parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(str(path), node_ids=node_ids.astype(np.int32),
                        coords_mm=coords_mm.astype(np.float32), vox_idx=vox_idx.astype(np.int32),
                        Vm=np.asarray(Vm, dtype=np.float32, order="C"),
                        time_vm=times.astype(np.float32), dt_solver=np.float32(dt_solver),
                        vm_save_dt=np.float32(vm_save_dt))


def save_npz(results, path):
    """Same schema as the reference's _save_npz (pipeline.py:1427-1450)."""
    path = Path(path).with_suffix(".npz")
    d = {"time": np.array(results["times"], np.float32), "comp_nodes": results["comp_nodes"],
         "comp_edges": results["comp_edges"], "surf_verts": results["surf_verts"],
         "surf_faces": results["surf_faces"], "vert_to_surf_node": results["vert_to_surf_node"],
         "surf_frames": np.asarray(results["frames_surf"], np.float32)}
    for b, bm in enumerate(results["branch_map"]):
        d[f"bmap_{b}"] = np.array(bm, np.int32)
        d[f"branch_{b}"] = np.asarray(results["branch_frames_p"][b], np.float32)
    np.savez_compressed(str(path), **d)


def _surface_mesh(Z, surf_nodes_mm, h):
    """Marching-cubes surface for the animation output.  Needs scikit-image
    (as the reference does); empty arrays when it is not installed."""
    try:
        from skimage.measure import marching_cubes
    except ImportError:
        return (np.zeros((0, 3), np.float32), np.zeros((0, 3), np.int32),
                np.zeros(0, np.int32))
    from scipy.spatial import cKDTree
    verts, faces, _, _ = marching_cubes(np.asarray(Z).astype(np.float32), level=0.5,
                                        spacing=(h, h, h))
    sv = verts[:, [1, 0, 2]].astype(np.float32)
    _, nn = cKDTree(surf_nodes_mm).query(sv, k=1)
    return sv, faces.astype(np.int32), nn.astype(np.int32)


def run(nodes, elements, activation_times, S, Z, phi, *, fibre_dir=None, anisotropic=False,
        theta=0.0, dtype=None, device=None, n_frames=100, frame_save_dt=None,
        out_npz=None, out_vm_npz=None, vm_save_dt=None, vm_tmp_dir=None, anim_tmp_dir=None,
        cg_tol=None, cg_max_iter=None, graph_chunk=50, verbose=False, **kw):
    """Full run with the reference's return dict, plus activation events.
    theta = 0 runs the fused explicit step; 0 < theta <= 1 the theta-scheme
    with its CG solve (cg_tol, cg_max_iter as the reference's defaults)."""
    if device is not None and not str(device).startswith("cuda"):
        raise ValueError(f"device={device!r}: this implementation runs on CUDA only")
    T = kw.get("T", 400.0)
    dt = kw.get("dt", 0.1)
    n_steps = int(T / dt)
    if frame_save_dt is not None:
        save_every = max(1, int(round(frame_save_dt / dt)))
    else:
        save_every = max(1, n_steps // max(1, int(n_frames)))
    run_vm = vm_save_dt is not None and out_vm_npz is not None
    cn = {} if float(theta) == 0.0 else dict(
        theta=float(theta), cg_tol=1e-5 if cg_tol is None else float(cg_tol),
        cg_max_iter=100 if cg_max_iter is None else int(cg_max_iter))
    prob, info = prepare(nodes, elements, activation_times, S, Z, phi, fibre_dir=fibre_dir,
                         anisotropic=anisotropic, vm_save_dt=vm_save_dt if run_vm else None,
                         save_every=save_every, **cn, **kw)
    sim = MonoHandle(prob)
    try:
        vm = None
        if run_vm and sim.n_vm_frames > 0:
            # the snapshots stream into pinned host memory chunk by chunk,
            # each chunk's copy overlapping the next chunk's steps
            import torch
            ve = prob.vm_every
            nvf = sim.n_vm_frames
            buf = torch.empty((nvf, prob.n_myo), dtype=torch.float32, pin_memory=True)
            per = max(1, min(nvf, 64))
            f0 = 0
            while f0 < nvf:
                nf_ = min(per, nvf - f0)
                end = n_steps if f0 + nf_ == nvf else (f0 + nf_) * ve
                sim.run(end - sim.steps_done, graph_chunk)
                sim.vm_frames_async(f0, nf_, buf[f0:f0 + nf_])
                f0 += nf_
            if sim.steps_done < n_steps:
                sim.run(n_steps - sim.steps_done, graph_chunk)
            sim.wait_copies()
            vm = buf.numpy()
        else:
            sim.run(n_steps, graph_chunk)
        surf, pk = sim.anim_frames()
        act, nact, dea, ndea = sim.events()
    finally:
        sim.close()
    Np = info["Np"]
    times = [k * dt for k in range(0, n_steps, save_every)]
    branch_frames = [pk[:, np.asarray(bm)] for bm in info["branch_map"]]
    sv, sf, vs = _surface_mesh(Z if Z is not None else S,
                               info["nodes_mm"][info["surface_node_ids"]], float(kw["voxel_size"]))
    results = dict(comp_nodes=info["comp_nodes"], comp_edges=info["comp_edges"],
                   branch_map=info["branch_map"], branch_frames_p=branch_frames,
                   surf_verts=sv, surf_faces=sf, vert_to_surf_node=vs, frames_surf=surf,
                   times=times)
    # node bookkeeping of the snapshot / activation-map files
    results["node_ids"] = np.arange(len(info["vox_idx"]), dtype=np.int32) + Np
    results["coords_mm"] = info["nodes_mm"]
    results["vox_idx"] = info["vox_idx"]
    me = prob.max_events
    results["activation_times"] = _events_table(act, nact, me)
    results["n_activations"] = nact
    results["deactivation_times"] = _events_table(dea, ndea, me)
    results["n_deactivations"] = ndea
    if run_vm:
        ve = prob.vm_every
        tv = np.array([k * dt for k in range(0, n_steps, ve)], np.float32)
        save_vm_snapshots(out_vm_npz, np.arange(len(info["vox_idx"]), dtype=np.int32) + Np,
                          info["nodes_mm"], info["vox_idx"], vm, tv, dt, ve * dt)
        results["vm_snapshots"] = vm
        results["time_vm"] = tv
        results["vm_snapshots_path"] = str(Path(out_vm_npz).with_suffix(".npz"))
    if out_npz is not None:
        save_npz(results, out_npz)
    return results


def _events_table(t, n, max_events):
    """(max_events, N) slot tables -> (N, n_cols) NaN-padded event table
    with as many columns as the most events any node saw (capped)."""
    ncol = int(min(max_events, n.max())) if n.size else 0
    return np.ascontiguousarray(t[:ncol].T)
