"""FP64 numpy emulation of the fused monodomain kernel's algorithm, run on
the product's MonoProblem (brick slots, tag bits, coefficient arrays, the
half-step skew and in-loop event recording, the theta-scheme's weighted
CG solve).  Used by CPU tests to check the
host-side preparation and the kernel's step logic against the oracle without
a GPU.  The ionic half uses the oracle's TTP06 (FP64)."""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from hrdayapy_b200.layout import DIAG_OFFSETS, FACE_OFFSETS, TAG_DIAG_SHIFT, TAG_FACE_SHIFT, TAG_PMJ
from oracle import mono as orc


def coefficient_matrix(prob):
    """Sparse (Np + N) x (Np + N) matrix of the per-edge coefficients the
    kernel applies (reference node order [Purkinje | myocardium])."""
    lay = prob.layout
    N = len(lay.vox_idx)
    Np = prob.n_pk
    vox = lay.vox_idx
    shape = lay.shape
    f2n = -np.ones(shape, np.int64)
    f2n[vox[:, 0], vox[:, 1], vox[:, 2]] = np.arange(N)
    tag = prob.tag[lay.slot_of_node].astype(np.int64)
    rows, cols, vals = [], [], []
    for q, off in enumerate(FACE_OFFSETS):
        has = (tag >> (TAG_FACE_SHIFT + q)) & 1 == 1
        i = np.where(has)[0]
        nb = vox[i] + off
        j = f2n[nb[:, 0], nb[:, 1], nb[:, 2]]
        assert (j >= 0).all()
        if prob.anisotropic:
            ax = q // 2
            src = i if q % 2 == 0 else j
            w = prob.wface[ax][lay.slot_of_node[src]].astype(np.float64)
        else:
            w = np.full(len(i), prob.iso_coef)
        rows.append(i + Np); cols.append(j + Np); vals.append(w)
    if prob.anisotropic:
        for q, off in enumerate(DIAG_OFFSETS):
            has = (tag >> (TAG_DIAG_SHIFT + q)) & 1 == 1
            i = np.where(has)[0]
            nb = vox[i] + off
            j = f2n[nb[:, 0], nb[:, 1], nb[:, 2]]
            assert (j >= 0).all()
            comp = q // 4
            sgn = 1.0 if q % 4 < 2 else -1.0
            d = prob.doff[comp].astype(np.float64)
            w = sgn * 0.25 * (d[lay.slot_of_node[i]] + d[lay.slot_of_node[j]])
            rows.append(i + Np); cols.append(j + Np); vals.append(w)
    node_of_slot = np.full(lay.n_slots, -1, np.int64)
    node_of_slot[lay.slot_of_node] = np.arange(N)
    # Purkinje rows
    for p in range(Np):
        for q in range(prob.pk_ptr[p], prob.pk_ptr[p + 1]):
            j = int(prob.pk_idx[q])
            col = j if j >= 0 else Np + node_of_slot[-j - 1]
            rows.append(np.array([p])); cols.append(np.array([col]))
            vals.append(np.array([float(prob.pk_coef[q])]))
    # junction rows on the myocardial side
    pm = np.where(tag & TAG_PMJ)[0]
    for i in pm:
        r = prob.pmj_row[lay.slot_of_node[i]]
        for q in range(prob.pmj_ptr[r], prob.pmj_ptr[r + 1]):
            rows.append(np.array([Np + i])); cols.append(np.array([prob.pmj_pk[q]]))
            vals.append(np.array([float(prob.pmj_coef[q])]))
    r = np.concatenate(rows); c = np.concatenate(cols); v = np.concatenate(vals)
    return sp.csr_matrix((v, (r, c)), shape=(Np + N, Np + N))


def emulate(prob, n_steps=None):
    """Runs the kernel algorithm; returns Vm snapshots (node order), Purkinje
    snapshots and the per-node first activation time."""
    lay = prob.layout
    N = len(lay.vox_idx)
    Np = prob.n_pk
    n_steps = prob.n_steps if n_steps is None else n_steps
    Cmat = coefficient_matrix(prob)
    deg = np.asarray(Cmat.sum(axis=1)).ravel()
    tag = prob.tag[lay.slot_of_node].astype(np.int64)
    pheno = np.concatenate([np.zeros(Np, np.int8), (tag & 3).astype(np.int8) - 1])
    stim_bits = np.concatenate([prob.pk_stim.astype(np.int64), (tag >> 20) & 0xFF])
    amp = prob.site_amp.astype(np.float64)
    dt, Cm = prob.dt, prob.Cm
    state = np.tile(orc.TTP06_INIT, (Np + N, 1))
    Vpost = np.full(Np + N, prob.v0)

    def ionic(V, istep):
        I = orc.ttp06_step(V, state, dt, pheno)
        on = stim_bits & int(prob.site_on[istep])
        Is = np.zeros(Np + N)
        for s in range(len(amp)):
            Is += np.where((on >> s) & 1, amp[s], 0.0)
        return V + (dt / Cm) * (-(I * Cm) + Is)

    Lh = (Cmat - sp.diags(deg)).tocsr()
    wgt = np.concatenate([np.full(Np, prob.pk_weight), np.ones(N)])
    dinv = 1.0 / (1.0 + prob.theta * deg)

    def cn_solve(W):
        """The GPU theta-scheme solve: Jacobi-preconditioned CG in the
        inner product weighted by wgt, from x = W (rhs - M W = Lh W)."""
        th = prob.theta
        tol2 = max(prob.cn_tol, 1e-7) ** 2
        LW = Lh @ W
        x, r = W.copy(), LW.copy()
        p = dinv * r
        bb = float(np.sum((W + (1.0 - th) * LW) ** 2))
        rz = float(np.sum(wgt * r * p))
        if float(r @ r) <= tol2 * bb or bb == 0.0:
            return x, 0
        for it in range(1, prob.cn_max_iter + 1):
            q = p - th * (Lh @ p)
            pq = float(np.sum(wgt * p * q))
            if not pq > 0.0:
                return x, it
            alpha = rz / pq
            x += alpha * p
            r -= alpha * q
            z = dinv * r
            rz_new = float(np.sum(wgt * r * z))
            if float(r @ r) <= tol2 * bb:
                return x, it
            p = z + (rz_new / rz) * p
            rz = rz_new
        return x, prob.cn_max_iter

    W = ionic(Vpost, 0)
    snaps, psnaps = [], []
    act = np.full(N, np.nan)
    iters = []
    for step in range(n_steps):
        if prob.theta == 0.0:
            Vn = np.clip(W + (Cmat @ W - deg * W), -150.0, 80.0)
        else:
            x, it = cn_solve(W)
            iters.append(it)
            Vn = np.clip(x, -150.0, 80.0)
        if step >= 1:
            Vp = Vpost[Np:]
            thr = prob.act_threshold
            cross = (Vp < thr) & (Vn[Np:] >= thr) & np.isnan(act)
            t0, t1 = (step - 1) * dt, step * dt
            frac = np.clip((thr - Vp) / np.where(Vn[Np:] - Vp == 0, 1e-9, Vn[Np:] - Vp), 0, 1)
            act = np.where(cross, t0 + frac * (t1 - t0), act)
        Vpost = Vn
        if prob.vm_every and step % prob.vm_every == 0:
            snaps.append(Vn[Np:].astype(np.float32))
            psnaps.append(Vn[:Np].astype(np.float32))
        W = ionic(Vn, step + 1)
    emulate.cn_iters = iters
    return np.array(snaps), np.array(psnaps), act
