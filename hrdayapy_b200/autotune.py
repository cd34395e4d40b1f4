"""Autotuner for the monodomain step: picks the brick shape and step kernel
(per-brick, pipelined or split) by timing each candidate on the problem
itself.

Brick shape decides how many padding slots partially filled bricks carry,
how large the halo of a tile is and how many CTAs fit an SM; which wins
depends on the geometry (a thin shell prefers thin bricks) and on the
device, so it is measured, not guessed.  ``relayout`` re-bricks a prepared
problem without repeating its set-up: every per-slot array goes back to node
order through ``slot_of_node`` and is scattered into the new bricks, and the
Purkinje CSR's myocardial-slot references are remapped.  Results are cached
(JSON) per device and problem signature.
"""
from __future__ import annotations

import dataclasses
import json
import os
import time
from pathlib import Path

import numpy as np

from .layout import build_layout
from .monodomain import MonoProblem

SHAPES = [(4, 4, 8), (4, 8, 8), (2, 4, 16), (8, 8, 8)]
KERNELS = {1: "brick", 2: "pipelined", 3: "split"}


def relayout(prob: MonoProblem, brick) -> MonoProblem:
    """The same problem stored in bricks of shape `brick`."""
    old = prob.layout
    if tuple(brick) == tuple(old.brick):
        return prob
    if old.shape is None:
        raise ValueError("relayout needs a single-heart problem (ensembles keep their bricks)")
    S = np.zeros(old.shape, np.uint8)
    v = old.vox_idx
    S[v[:, 0], v[:, 1], v[:, 2]] = 1
    new = build_layout(S, brick, prob.anisotropic)
    if not np.array_equal(new.vox_idx, old.vox_idx):
        raise RuntimeError("relayout: node order changed")
    sos_old = np.asarray(old.slot_of_node, np.int64)
    ns_old = old.n_slots

    def per_slot(a, fill=0):
        a = np.asarray(a)
        return new.to_slots(a[sos_old], fill=fill, dtype=a.dtype)

    def comp3(a):
        a = np.asarray(a).reshape(3, ns_old)
        return np.stack([per_slot(a[c]) for c in range(3)]).reshape(-1)

    node_of_old_slot = np.full(ns_old, -1, np.int64)
    node_of_old_slot[sos_old] = np.arange(len(sos_old))
    idx = np.asarray(prob.pk_idx, np.int64)
    myo = idx < 0
    nodes = node_of_old_slot[-idx[myo] - 1]
    if (nodes < 0).any():
        raise RuntimeError("relayout: a Purkinje edge points at a padding slot")
    idx = idx.copy()
    idx[myo] = -np.asarray(new.slot_of_node, np.int64)[nodes] - 1
    return dataclasses.replace(
        prob, layout=new, tag=per_slot(prob.tag),
        wface=comp3(prob.wface) if prob.anisotropic else None,
        doff=comp3(prob.doff) if prob.anisotropic else None,
        pk_idx=idx.astype(np.int32), pmj_row=per_slot(prob.pmj_row, fill=-1),
        surf_of_slot=per_slot(prob.surf_of_slot, fill=-1))


def _site_on(site_on, n):
    """Pulse table(s) resized to n steps (one row per variant kept apart)."""
    a = np.asarray(site_on, np.uint8)
    if a.ndim == 1:
        return np.ascontiguousarray(np.resize(a, n + 1))
    return np.ascontiguousarray(np.stack([np.resize(r, n + 1) for r in a]))


def _signature(prob, device_name):
    return (f"{device_name}|n={prob.n_myo}|pk={prob.n_pk}|aniso={int(prob.anisotropic)}|"
            f"bricks448={prob.layout.n_bricks if tuple(prob.layout.brick) == (4, 4, 8) else -1}")


def tune(prob: MonoProblem, shapes=SHAPES, kernels=(3, 2), steps=100, warmup=20,
         cache_path=None, verbose=False):
    """Time every (brick shape, kernel) candidate for `steps` steps after
    `warmup` and return (best_problem, table).  table: list of dicts with
    brick, kernel, voxel_steps_per_s (or error), best first.  With a cache
    hit the timing is skipped and the cached winner is re-bricked."""
    import torch
    from . import monodomain as M
    dev = torch.cuda.get_device_name()
    key = _signature(prob, dev)
    cache = {}
    if cache_path and Path(cache_path).exists():
        try:
            cache = json.loads(Path(cache_path).read_text())
        except (OSError, ValueError):
            cache = {}
    if key in cache:
        table = cache[key]
        best = table[0]
        return dataclasses.replace(relayout(prob, best["brick"]), kernel=best["kernel"]), table
    n = warmup + steps
    table = []
    layouts = {}
    for brick in shapes:
        brick = tuple(brick)
        try:
            layouts[brick] = relayout(prob, brick)
        except Exception as e:  # noqa: BLE001 -- recorded in the table
            table.append({"brick": list(brick), "kernel": None, "error": str(e)})
            continue
        for kern in kernels:
            p = dataclasses.replace(layouts[brick], kernel=kern, n_steps=n, vm_every=0,
                                    frame_every=0, site_on=_site_on(prob.site_on, n))
            try:
                # the handle launches on its own stream: time the steps by the
                # wall clock between two full synchronisations
                chunk = min(steps, 50)
                sim = M.MonoHandle(p)
                sim.run(warmup, graph_chunk=min(warmup, chunk))
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                sim.run(steps, graph_chunk=chunk)
                torch.cuda.synchronize()
                dt = time.perf_counter() - t0
                sim.close()
                rate = p.n_myo * steps / dt
                table.append({"brick": list(brick), "kernel": kern, "voxel_steps_per_s": rate})
                if verbose:
                    print(f"autotune {brick} {KERNELS[kern]}: {rate / 1e9:.2f} G voxel-steps/s",
                          flush=True)
            except Exception as e:  # noqa: BLE001
                table.append({"brick": list(brick), "kernel": kern, "error": str(e)})
    ok = [t for t in table if "voxel_steps_per_s" in t]
    if not ok:
        raise RuntimeError(f"autotune: no candidate ran: {table}")
    ok.sort(key=lambda t: -t["voxel_steps_per_s"])
    table = ok + [t for t in table if "voxel_steps_per_s" not in t]
    if cache_path:
        cache[key] = table
        try:
            Path(cache_path).parent.mkdir(parents=True, exist_ok=True)
            Path(cache_path).write_text(json.dumps(cache, indent=1))
        except OSError:
            pass
    best = table[0]
    p = layouts[tuple(best["brick"])]
    p = dataclasses.replace(p, kernel=best["kernel"])
    return p, table


def default_cache_path():
    return os.environ.get("HP_AUTOTUNE_CACHE",
                          str(Path.home() / ".cache" / "hrdayapy_b200" / "autotune.json"))
