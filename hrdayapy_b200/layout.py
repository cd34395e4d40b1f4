"""Host-side geometry preparation: voxel mask -> brick layout for the fused
monodomain kernel.

The reference numbers myocardial nodes in ``np.argwhere(S == 1)`` order
(C order over (i, j, k)) and assembles a global sparse Laplacian
(simulation/functions/purkinje_myocardium_pipeline.py:761-833 for the
6-connected isotropic mesh, anisotropic_simulation/functions/
purkinje_myocardium_anisotropic_solver.py:856-1074 for the 18-connected
fibre-tensor mesh).  Here the same voxels are stored in dense bricks of
``bi x bj x bk`` (k fastest) covering only the bricks that touch the mask,
and the Laplacian is never assembled: the kernel evaluates the stencil from
per-voxel neighbour bits and coefficients.  Node order is kept through
``slot_of_node`` so every output is reported in the reference's order.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# neighbour offsets in tag-bit order (include/hrdaya_b200.h)
FACE_OFFSETS = np.array([(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)])
DIAG_OFFSETS = np.array([(1, 1, 0), (-1, -1, 0), (1, -1, 0), (-1, 1, 0),
                         (1, 0, 1), (-1, 0, -1), (1, 0, -1), (-1, 0, 1),
                         (0, 1, 1), (0, -1, -1), (0, 1, -1), (0, -1, 1)])
TAG_FACE_SHIFT = 2
TAG_DIAG_SHIFT = 8
TAG_STIM_SHIFT = 20
TAG_PMJ = 1 << 28
TAG_SURF = 1 << 29


@dataclass
class BrickLayout:
    shape: tuple
    brick: tuple                      # (bi, bj, bk)
    vox_idx: np.ndarray               # (N, 3) int64, reference node order
    n_bricks: int
    brick_coords: np.ndarray          # (n_bricks, 3)
    brick_nbr: np.ndarray             # (n_bricks, 27) int32
    slot_of_node: np.ndarray          # (N,) int32
    nbr_bits: np.ndarray              # (N,) uint32 face+diag neighbour bits (node order)
    extras: dict = field(default_factory=dict)

    @property
    def bv(self) -> int:
        return int(np.prod(self.brick))

    @property
    def n_slots(self) -> int:
        return self.n_bricks * self.bv

    def to_slots(self, values, fill=0, dtype=None):
        """Scatter a per-node array (N, ...) into slot order (n_slots, ...)."""
        values = np.asarray(values)
        dtype = dtype or values.dtype
        out = np.full((self.n_slots,) + values.shape[1:], fill, dtype=dtype)
        out[self.slot_of_node] = values
        return out


def build_layout(S: np.ndarray, brick=(4, 4, 8), anisotropic: bool = False) -> BrickLayout:
    """Brick layout of the voxels with S == 1 (argwhere order preserved)."""
    S = np.asarray(S)
    shape = S.shape
    bi, bj, bk = brick
    vox = np.argwhere(S == 1).astype(np.int64)
    N = len(vox)
    bshape = ((shape[0] + bi - 1) // bi, (shape[1] + bj - 1) // bj, (shape[2] + bk - 1) // bk)
    bc = vox // np.array(brick)
    bflat = (bc[:, 0] * bshape[1] + bc[:, 1]) * bshape[2] + bc[:, 2]
    ub, binv = np.unique(bflat, return_inverse=True)
    n_bricks = len(ub)
    bcoords = np.stack(np.unravel_index(ub, bshape), 1).astype(np.int64)
    # dense brick-id grid with a one-brick border
    bgrid = -np.ones((bshape[0] + 2, bshape[1] + 2, bshape[2] + 2), np.int32)
    bgrid[bcoords[:, 0] + 1, bcoords[:, 1] + 1, bcoords[:, 2] + 1] = np.arange(n_bricks, dtype=np.int32)
    nbr = np.empty((n_bricks, 27), np.int32)
    q = 0
    for di in (-1, 0, 1):
        for dj in (-1, 0, 1):
            for dk in (-1, 0, 1):
                nbr[:, q] = bgrid[bcoords[:, 0] + 1 + di, bcoords[:, 1] + 1 + dj, bcoords[:, 2] + 1 + dk]
                q += 1
    loc = vox - bc * np.array(brick)
    slot = binv.astype(np.int64) * (bi * bj * bk) + (loc[:, 0] * bj + loc[:, 1]) * bk + loc[:, 2]
    # neighbour-in-mask bits
    P = np.zeros((shape[0] + 2, shape[1] + 2, shape[2] + 2), bool)
    P[1:-1, 1:-1, 1:-1] = S == 1
    bits = np.zeros(N, np.uint32)
    offs = [(FACE_OFFSETS, TAG_FACE_SHIFT)]
    if anisotropic:
        offs.append((DIAG_OFFSETS, TAG_DIAG_SHIFT))
    for table, shift in offs:
        for q, (di, dj, dk) in enumerate(table):
            has = P[vox[:, 0] + 1 + di, vox[:, 1] + 1 + dj, vox[:, 2] + 1 + dk]
            bits |= has.astype(np.uint32) << np.uint32(shift + q)
    return BrickLayout(shape=shape, brick=tuple(brick), vox_idx=vox, n_bricks=n_bricks,
                       brick_coords=bcoords, brick_nbr=nbr, slot_of_node=slot.astype(np.int32),
                       nbr_bits=bits)


def conductivity_tensor(fibre_dir, vox, sigma_l, sigma_t):
    """D = sigma_t I + (sigma_l - sigma_t) f f^T per node, FP64, fibre in raw
    array-axis order (purkinje_myocardium_anisotropic_solver.py:856-883)."""
    f = np.asarray(fibre_dir)[vox[:, 0], vox[:, 1], vox[:, 2], :].astype(np.float64)
    ds = float(sigma_l) - float(sigma_t)
    st = float(sigma_t)
    return (st + ds * f[:, 0] * f[:, 0], st + ds * f[:, 1] * f[:, 1], st + ds * f[:, 2] * f[:, 2],
            ds * f[:, 0] * f[:, 1], ds * f[:, 0] * f[:, 2], ds * f[:, 1] * f[:, 2])


def aniso_coefficients(lay: BrickLayout, S, fibre_dir, sigma_l, sigma_t, scale):
    """Per-slot face coefficients to +i/+j/+k (harmonic mean of D_kk, times
    `scale`) and scaled off-diagonal components D01, D02, D12.

    With scale = dt / (Cm A_M h^2) the kernel's explicit update reproduces
    the reference's edge weights (..._anisotropic_solver.py:997-1029):
    face w = harm(D_kk) h, diagonal w = +/- mean(D_ij) h / 2, divided by
    the membrane loading A_M h^3 and multiplied by dt / Cm.
    """
    vox = lay.vox_idx
    shape = lay.shape
    N = len(vox)
    D = conductivity_tensor(fibre_dir, vox, sigma_l, sigma_t)
    # node lookup for the +face neighbours
    f2n = -np.ones(shape, np.int64)
    f2n[vox[:, 0], vox[:, 1], vox[:, 2]] = np.arange(N)
    wf = np.zeros((3, N))
    for ax in range(3):
        nb = vox.copy()
        nb[:, ax] += 1
        ok = nb[:, ax] < shape[ax]
        m = np.full(N, -1, np.int64)
        m[ok] = f2n[nb[ok, 0], nb[ok, 1], nb[ok, 2]]
        has = m >= 0
        Da = D[ax][has]
        Db = D[ax][m[has]]
        wf[ax, has] = 2.0 * Da * Db / np.maximum(Da + Db, 1e-30) * scale
    doff = np.stack([D[3], D[4], D[5]]) * scale
    wface_s = np.zeros((3, lay.n_slots), np.float32)
    doff_s = np.zeros((3, lay.n_slots), np.float32)
    wface_s[:, lay.slot_of_node] = wf.astype(np.float32)
    doff_s[:, lay.slot_of_node] = doff.astype(np.float32)
    return wface_s, doff_s


def surface_nodes(S, Z, vox):
    """Z-surface myocardial nodes (pipeline.py:811-827): a node is on the
    surface if any face neighbour is outside the grid or outside Z."""
    shape = np.asarray(S).shape
    Z = np.asarray(Z)
    is_surf = np.zeros(len(vox), bool)
    for d in FACE_OFFSETS:
        n = vox + d
        inb = np.all((n >= 0) & (n < np.array(shape)), axis=1)
        c = np.clip(n, 0, np.array(shape) - 1)
        nb_in_Z = inb & (Z[c[:, 0], c[:, 1], c[:, 2]] == 1)
        is_surf |= ~nb_in_Z
    return np.where(is_surf)[0].astype(np.int32)
