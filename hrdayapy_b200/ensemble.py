"""Batched ensembles: independent heart variants of uneven size advanced by
one launch per step.

There is no ensemble in the reference: each run of run_coupled /
purkinje_myocardium_anisotropic_solver advances one heart
(simulation/functions/purkinje_myocardium_pipeline.py:1030-1463).  Here the
prepared problems of several variants (``monodomain.prepare``, same brick
shape, time step and run length) are concatenated brick by brick into one
problem: brick, slot, Purkinje-node and junction indices are offset, every
brick and Purkinje node carries its variant id, and each variant keeps its
own ionic scaling (g_Ks, g_Kr multipliers), stimulus sites and pulse
schedule.  The step kernels never mix variants: a brick's neighbour table
only names bricks of its own variant, so every variant evolves exactly as it
would alone (bit for bit).  Outputs are in concatenated node order;
``Ensemble.split`` cuts a per-node array back into per-variant pieces.
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass

import numpy as np

from .layout import BrickLayout
from .monodomain import MonoProblem

MAX_VARIANTS = 64   # HP_MAX_VARIANTS


@dataclass
class Ensemble:
    problem: MonoProblem
    node_offsets: np.ndarray      # (n_variants + 1,) myocardial node ranges
    pk_offsets: np.ndarray        # (n_variants + 1,) Purkinje node ranges

    @property
    def n_variants(self) -> int:
        return len(self.node_offsets) - 1

    def split(self, per_node, axis=-1):
        """Per-variant pieces of an array over the concatenated nodes."""
        a = np.asarray(per_node)
        return [np.take(a, np.arange(self.node_offsets[v], self.node_offsets[v + 1]), axis=axis)
                for v in range(self.n_variants)]


def build_ensemble(problems, gks=None, gkr=None) -> Ensemble:
    """Concatenate prepared single-heart problems into one ensemble problem.
    gks / gkr: per-variant multipliers of the phenotype g_Ks / g_Kr
    (default 1)."""
    probs = list(problems)
    nv = len(probs)
    if not 1 <= nv <= MAX_VARIANTS:
        raise ValueError(f"an ensemble holds 1..{MAX_VARIANTS} variants, got {nv}")
    p0 = probs[0]
    for p in probs[1:]:
        for name in ("dt", "Cm", "n_steps", "vm_every", "frame_every", "anisotropic", "v0",
                     "act_threshold", "deact_threshold", "max_events"):
            if getattr(p, name) != getattr(p0, name):
                raise ValueError(f"ensemble variants differ in {name}")
        if tuple(p.layout.brick) != tuple(p0.layout.brick):
            raise ValueError("ensemble variants must use one brick shape")
        if not p0.anisotropic and p.iso_coef != p0.iso_coef:
            raise ValueError("isotropic ensemble variants must share the conductivity")
        if p.variant_gks is not None and len(p.variant_gks) > 1:
            raise ValueError("variants must be single-heart problems")
    gks = np.ones(nv) if gks is None else np.asarray(gks, np.float64)
    gkr = np.ones(nv) if gkr is None else np.asarray(gkr, np.float64)
    if gks.shape != (nv,) or gkr.shape != (nv,):
        raise ValueError("gks / gkr need one value per variant")
    bv = p0.layout.bv
    n_sites = max(len(np.atleast_1d(p.site_amp)) for p in probs)

    nbr, tags, wface, doff, slot_of_node = [], [], [], [], []
    pk_ptr, pk_idx, pk_coef, pk_stim = [np.zeros(1, np.int64)], [], [], []
    pmj_row, pmj_ptr, pmj_pk, pmj_coef = [], [np.zeros(1, np.int64)], [], []
    surf_nodes, surf_of_slot = [], []
    brick_variant, pk_variant = [], []
    site_amp = np.zeros((nv, n_sites), np.float32)
    site_on = np.zeros((nv, p0.n_steps + 1), np.uint8)
    b_off = s_off = n_off = pk_off = pmj_off = nnz_off = pmj_nnz_off = surf_off = 0
    node_offsets, pk_offsets = [0], [0]
    for v, p in enumerate(probs):
        lay = p.layout
        nb = np.asarray(lay.brick_nbr, np.int64)
        nbr.append(np.where(nb >= 0, nb + b_off, -1))
        tags.append(np.asarray(p.tag, np.uint32))
        if p0.anisotropic:
            wface.append(np.asarray(p.wface, np.float32).reshape(3, -1))
            doff.append(np.asarray(p.doff, np.float32).reshape(3, -1))
        slot_of_node.append(np.asarray(lay.slot_of_node, np.int64) + s_off)
        # Purkinje CSR: j >= 0 a Purkinje node, j < 0 myocardial slot -j - 1
        ptr = np.asarray(p.pk_ptr, np.int64)
        idx = np.asarray(p.pk_idx, np.int64)
        pk_ptr.append(ptr[1:] + nnz_off)
        pk_idx.append(np.where(idx >= 0, idx + pk_off, -((-idx - 1) + s_off) - 1))
        pk_coef.append(np.asarray(p.pk_coef, np.float32))
        pk_stim.append(np.asarray(p.pk_stim, np.uint8))
        nnz_off += len(idx)
        # myocardial side of the junctions
        row = np.asarray(p.pmj_row, np.int64)
        pmj_row.append(np.where(row >= 0, row + pmj_off, row))
        pptr = np.asarray(p.pmj_ptr, np.int64)
        pmj_ptr.append(pptr[1:] + pmj_nnz_off)
        pmj_pk.append(np.asarray(p.pmj_pk, np.int64) + pk_off)
        pmj_coef.append(np.asarray(p.pmj_coef, np.float32))
        pmj_off += len(pptr) - 1
        pmj_nnz_off += int(pptr[-1])
        # animation surface
        sn = np.asarray(p.surf_nodes, np.int64)
        surf_nodes.append(sn + n_off)
        sos = np.asarray(p.surf_of_slot, np.int64)
        surf_of_slot.append(np.where(sos >= 0, sos + surf_off, sos))
        surf_off += len(sn)
        # variant ids and stimulus tables
        brick_variant.append(np.full(lay.n_bricks, v, np.uint8))
        pk_variant.append(np.full(p.n_pk, v, np.uint8))
        amp = np.atleast_1d(np.asarray(p.site_amp, np.float32))
        site_amp[v, :len(amp)] = amp
        site_on[v] = np.asarray(p.site_on, np.uint8).reshape(-1)
        b_off += lay.n_bricks
        s_off += lay.n_slots
        n_off += p.n_myo
        pk_off += p.n_pk
        node_offsets.append(n_off)
        pk_offsets.append(pk_off)

    cat = np.concatenate
    lay = BrickLayout(shape=None, brick=tuple(p0.layout.brick),
                      vox_idx=np.zeros((n_off, 3), np.int64), n_bricks=b_off,
                      brick_coords=np.zeros((b_off, 3), np.int64),
                      brick_nbr=cat(nbr).astype(np.int32),
                      slot_of_node=cat(slot_of_node).astype(np.int32),
                      nbr_bits=np.zeros(n_off, np.uint32),
                      extras={"variant_layouts": [p.layout for p in probs]})
    prob = dataclasses.replace(
        p0, layout=lay, tag=cat(tags),
        wface=cat(wface, axis=1).reshape(-1) if p0.anisotropic else None,
        doff=cat(doff, axis=1).reshape(-1) if p0.anisotropic else None,
        pk_ptr=cat(pk_ptr).astype(np.int32), pk_idx=cat(pk_idx).astype(np.int32),
        pk_coef=cat(pk_coef), pk_stim=cat(pk_stim),
        pmj_row=cat(pmj_row).astype(np.int32), pmj_ptr=cat(pmj_ptr).astype(np.int32),
        pmj_pk=cat(pmj_pk).astype(np.int32), pmj_coef=cat(pmj_coef),
        site_amp=site_amp, site_on=site_on,
        surf_nodes=cat(surf_nodes), surf_of_slot=cat(surf_of_slot).astype(np.int32),
        brick_variant=cat(brick_variant), pk_variant=cat(pk_variant),
        variant_gks=gks, variant_gkr=gkr)
    return Ensemble(prob, np.asarray(node_offsets), np.asarray(pk_offsets))
