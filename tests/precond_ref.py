"""torch (CPU, FP32 autograd) restatement of the learned preconditioner's
network, features, output and loss -- the oracle for csrc/precond.cu."""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F

from hrdayapy_b200.ecg.precond import LCIN, LCOUT, param_offsets


def bf16(x):
    return torch.as_tensor(x).to(torch.bfloat16).to(torch.float32)


def invd_from_labels(labels, table, h_m, pin_cell):
    """Padded Jacobi inverse diagonal, FP64 sums rounded to FP32 (torso.cu)."""
    ni, nj, nk = labels.shape
    lab = np.zeros((ni + 2, nj + 2, nk + 2), np.int64)
    lab[1:-1, 1:-1, 1:-1] = labels
    T = np.zeros((16, 16))
    for u in range(1, len(table)):
        for v in range(1, len(table)):
            su, sv = table[u], table[v]
            if su + sv >= 1e-30:
                T[u, v] = (2 * su * sv) / (su + sv) / h_m ** 2
    diag = np.zeros(lab.shape)
    for ax in range(3):
        for sh in (1, -1):
            nb = np.roll(lab, -sh, axis=ax)
            diag += T[lab, nb]
    invd = np.where(lab != 0, np.where(diag > 1e-30, 1.0 / np.maximum(diag, 1e-300), 1.0), 0.0)
    invd = invd.astype(np.float32).ravel()
    if pin_cell >= 0:
        invd[pin_cell] = 0.0
    return invd


def features(r_pad, invd_pad, labels, pin_cell, n_materials):
    ni, nj, nk = labels.shape
    lab = np.zeros((ni + 2, nj + 2, nk + 2), np.int64)
    lab[1:-1, 1:-1, 1:-1] = labels
    act = (lab != 0).ravel()
    if pin_cell >= 0:
        act[pin_cell] = False
    z = np.where(act, invd_pad.astype(np.float64) * r_pad, 0.0).reshape(lab.shape)[1:-1, 1:-1, 1:-1]
    raw = z.reshape(ni // 2, 2, nj // 2, 2, nk // 2, 2).sum((1, 3, 5)) / 8.0
    s = float(np.sqrt(np.mean(raw ** 2)))
    feat = np.zeros((ni // 2, nj // 2, nk // 2, 16))
    feat[..., 0] = raw / s
    L = labels.reshape(ni // 2, 2, nj // 2, 2, nk // 2, 2)
    frac = [(L == m).mean(axis=(1, 3, 5)) for m in range(n_materials)]
    feat[..., 1] = 1.0 - frac[0]
    for m in range(1, min(n_materials, 14)):
        feat[..., 1 + m] = frac[m]
    return bf16(feat), s


def net(feat, params, requires_grad=False):
    """feat (D, H, W, 16) -> y (D, H, W); params flat FP32 (BF16-rounded here)."""
    offs, n = param_offsets()
    P = torch.tensor(params, dtype=torch.float32, requires_grad=requires_grad)
    ws, bs = [], []
    for (ow, ob), ci, co in zip(offs, LCIN, LCOUT):
        w = P[ow:ob].view(co, ci, 3, 3, 3)
        ws.append(w)
        bs.append(P[ob:ob + co])

    def conv(x, l, relu=True):
        wq = ws[l] + (bf16(ws[l].detach()) - ws[l].detach())   # BF16 value, FP32 gradient
        y = F.conv3d(x, wq, bs[l], padding=1)
        return torch.relu(y) if relu else y

    x = feat.permute(3, 0, 1, 2)[None]
    e1a = conv(x, 0); e1b = conv(e1a, 1)
    p1 = F.avg_pool3d(e1b, (2, 2, 1))
    e2a = conv(p1, 2); e2b = conv(e2a, 3)
    p2 = F.avg_pool3d(e2b, (2, 2, 1))
    e3a = conv(p2, 4); e3b = conv(e3a, 5)
    u2 = torch.cat([F.interpolate(e3b, scale_factor=(2, 2, 1), mode="nearest"), e2b], 1)
    d2a = conv(u2, 6); d2b = conv(d2a, 7)
    u1 = torch.cat([F.interpolate(d2b, scale_factor=(2, 2, 1), mode="nearest"), e1b], 1)
    d1a = conv(u1, 8); d1b = conv(d1a, 9)
    y = conv(d1b, 10, relu=False)[0, 0]
    return y, P


def loss(y, s, r_pad, invd_pad, e_pad, labels, table, h_m, pin_cell, omega):
    """L = 1 - (r.z)^2 / ((z.A z)(r.e)), z = omega D^-1 r + s y[parent] on the
    unknown cells (no coarse level), A the torso stiffness (FP64)."""
    ni, nj, nk = labels.shape
    lab = np.zeros((ni + 2, nj + 2, nk + 2), np.int64)
    lab[1:-1, 1:-1, 1:-1] = labels
    act = (lab != 0).ravel().copy()
    if pin_cell >= 0:
        act[pin_cell] = False
    act = torch.tensor(act.reshape(lab.shape))
    T = np.zeros((16, 16))
    for u in range(1, len(table)):
        for v in range(1, len(table)):
            su, sv = table[u], table[v]
            if su + sv >= 1e-30:
                T[u, v] = (2 * su * sv) / (su + sv) / h_m ** 2
    r = torch.tensor(r_pad.astype(np.float64).reshape(lab.shape))
    e = torch.tensor(e_pad.astype(np.float64).reshape(lab.shape))
    zj = torch.tensor(omega * invd_pad.astype(np.float64).reshape(lab.shape)) * r
    yf = (s * y.double()).repeat_interleave(2, 0).repeat_interleave(2, 1).repeat_interleave(2, 2)
    yp = torch.zeros(lab.shape, dtype=torch.float64)
    yp[1:-1, 1:-1, 1:-1] = yf
    z = (zj + yp) * act
    az = torch.zeros_like(z)
    for ax in range(3):
        for sh in (1, -1):
            nb_lab = np.roll(lab, -sh, axis=ax)
            t = torch.tensor(T[lab, nb_lab])
            az = az + t * (z - torch.roll(z, -sh, dims=ax))
    az = az * act
    rz = (r * z * act).sum()
    zaz = (z * az).sum()
    re = (r * e * act).sum()
    return 1.0 - rz ** 2 / (zaz * re)


def coarse_correction(r_pad, labels, table, h_m, pin_cell, ag):
    """Q A_c^-1 Q^T r on the padded grid (FP64): aggregation over ag^3 cubes,
    Galerkin operator of the torso stiffness with the pinned voxel removed."""
    ni, nj, nk = labels.shape
    lab = np.zeros((ni + 2, nj + 2, nk + 2), np.int64)
    lab[1:-1, 1:-1, 1:-1] = labels
    T = np.zeros((16, 16))
    for u in range(1, len(table)):
        for v in range(1, len(table)):
            su, sv = table[u], table[v]
            if su + sv >= 1e-30:
                T[u, v] = (2 * su * sv) / (su + sv) / h_m ** 2
    unk = (lab != 0).ravel().copy()
    unk[pin_cell] = False
    ii, jj, kk = np.indices(lab.shape)
    box = ((np.maximum(ii - 1, 0) // ag) * ((nj + ag - 1) // ag) + np.maximum(jj - 1, 0) // ag) * \
        ((nk + ag - 1) // ag) + np.maximum(kk - 1, 0) // ag
    box = box.ravel()
    ub, cid = np.unique(box[unk], return_inverse=True)
    nc = len(ub)
    g = np.where(unk)[0]
    Ac = np.zeros((nc, nc))
    SI, SJ = (nj + 2) * (nk + 2), nk + 2
    labf = lab.ravel()
    cidf = np.full(lab.size, -1)
    cidf[g] = cid
    for off in (SI, -SI, SJ, -SJ, 1, -1):
        nb = g + off
        t = T[labf[g], labf[nb]]
        np.add.at(Ac, (cid, cid), t)
        m = unk[nb] & (t > 0)
        np.add.at(Ac, (cid[m], cidf[nb[m]]), -t[m])
    rc = np.bincount(cid, weights=r_pad[g].astype(np.float64), minlength=nc)
    zc = np.linalg.solve(Ac, rc)
    z = np.zeros(lab.size)
    z[g] = zc[cid]
    return z, nc
