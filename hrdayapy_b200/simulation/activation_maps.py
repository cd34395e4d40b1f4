"""Activation / deactivation maps with the reference's container and npz
schema (simulation/functions/activation_maps.py:156-470).

Two producers of the same ``ActivationMaps``:

* ``activation_maps_from_run`` -- from the event tables the GPU time step
  records in the loop (every threshold crossing of every voxel, interpolated
  linearly between consecutive post-step states, up to ``max_events`` per
  voxel); no snapshot file is needed.  With ``vm_save_dt = dt`` these are
  the crossings the reference finds in its snapshots.
* ``compute_activation_maps`` -- from a loaded Vm snapshot file, the
  reference's rule (activation_maps.py:63-152, 295-413): rising / falling
  crossings between consecutive frames, linear interpolation in float32 with
  the fraction clipped to [0, 1], every event kept, optional debounce.

``save_activation_maps`` / ``load_activation_maps`` write and read the
reference's npz (activation_maps.py:416-470): node_ids, coords_mm, vox_idx,
activation_times, deactivation_times (float32, NaN = none), n_activations,
n_deactivations (int32), act_threshold, deact_threshold (float32),
source_vm_path (str) and grid_shape (int32) when known.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from .vm_snapshots import _npz_path

REQUIRED = ("node_ids", "coords_mm", "vox_idx", "activation_times", "deactivation_times",
            "n_activations", "n_deactivations", "act_threshold", "deact_threshold")


@dataclass
class ActivationMaps:
    node_ids: np.ndarray
    coords_mm: np.ndarray
    vox_idx: np.ndarray
    activation_times: np.ndarray
    deactivation_times: np.ndarray
    n_activations: np.ndarray
    n_deactivations: np.ndarray
    act_threshold: float
    deact_threshold: float
    grid_shape: np.ndarray | None = None
    source_vm_path: str = ""
    path: Path = field(default_factory=lambda: Path("."))

    @property
    def N_myo(self) -> int:
        return int(self.activation_times.shape[0])

    @property
    def n_beats_activated(self) -> int:
        return int(self.activation_times.shape[1])

    @property
    def n_beats_deactivated(self) -> int:
        return int(self.deactivation_times.shape[1])

    @property
    def n_events(self) -> int:
        return max(self.n_beats_activated, self.n_beats_deactivated)

    def __repr__(self) -> str:
        return (f"ActivationMaps(N_myo={self.N_myo:,}, "
                f"activation_events={self.n_beats_activated}, "
                f"deactivation_events={self.n_beats_deactivated}, "
                f"act_threshold={self.act_threshold:g} mV, "
                f"deact_threshold={self.deact_threshold:g} mV, "
                f"never_activated={int((self.n_activations == 0).sum()):,})")

    @staticmethod
    def _column(table, event, n):
        k = event - 1
        if k < 0 or k >= table.shape[1]:
            return np.full(n, np.nan, dtype=np.float32)
        return table[:, k].copy()

    def activation_map(self, event: int = 1) -> np.ndarray:
        """Activation time of the ``event``-th beat (1-based), NaN if none."""
        return self._column(self.activation_times, event, self.N_myo)

    def deactivation_map(self, event: int = 1) -> np.ndarray:
        return self._column(self.deactivation_times, event, self.N_myo)

    def duration_map(self, event: int = 1) -> np.ndarray:
        return self.deactivation_map(event) - self.activation_map(event)

    def apd_map(self, event: int = 1) -> np.ndarray:
        return self.duration_map(event)

    def field_on_grid(self, values: np.ndarray) -> np.ndarray:
        """Per-node values scattered onto the mask grid (NaN background)."""
        if self.grid_shape is None:
            raise ValueError("grid_shape is not set on this ActivationMaps object -- "
                             "pass S to compute_activation_maps() to enable this.")
        g = np.full(tuple(int(x) for x in self.grid_shape), np.nan, dtype=np.float32)
        v = self.vox_idx
        g[v[:, 0], v[:, 1], v[:, 2]] = values
        return g

    def activation_grid(self, event: int = 1) -> np.ndarray:
        return self.field_on_grid(self.activation_map(event))

    def deactivation_grid(self, event: int = 1) -> np.ndarray:
        return self.field_on_grid(self.deactivation_map(event))

    def apd_grid(self, event: int = 1) -> np.ndarray:
        return self.field_on_grid(self.apd_map(event))


def _crossings(Vm, t, mask, thr):
    """(node, time) of every True entry of the (F-1, N) crossing mask, in
    frame order; float32 interpolation as the reference."""
    f, n = np.nonzero(mask)
    if f.size == 0:
        return n, np.zeros(0, np.float32)
    v0, v1 = Vm[f, n], Vm[f + 1, n]
    den = v1 - v0
    den = np.where(den == 0, 1e-9, den)
    frac = np.clip((thr - v0) / den, 0.0, 1.0)
    return n, (t[f] + frac * (t[f + 1] - t[f])).astype(np.float32)


def _table(node, tc, n_nodes):
    """NaN-padded (n_nodes, max_events) table, events in time order."""
    if node.size == 0:
        return np.zeros((n_nodes, 0), np.float32)
    o = np.argsort(node, kind="stable")
    node, tc = node[o], tc[o]
    cnt = np.bincount(node, minlength=n_nodes)
    pos = np.arange(node.size) - np.repeat(np.cumsum(cnt) - cnt, cnt)
    out = np.full((n_nodes, int(cnt.max())), np.nan, np.float32)
    out[node, pos] = tc
    return out


def _debounce(table, gap):
    """Drops events closer than ``gap`` ms to the previous kept one of the
    same node (activation_maps.py:119-152); None or one column: unchanged."""
    if gap is None or table.shape[1] <= 1:
        return table
    kept = []
    for row in table:
        k, last = [], -np.inf
        for v in row[~np.isnan(row)]:
            if v - last >= gap:
                k.append(v)
                last = v
        kept.append(k)
    out = np.full((table.shape[0], max((len(k) for k in kept), default=0)), np.nan, np.float32)
    for i, k in enumerate(kept):
        out[i, :len(k)] = k
    return out


def _grid_shape(S, vox_idx):
    if S is not None:
        S = np.asarray(S)
        inside = S[vox_idx[:, 0], vox_idx[:, 1], vox_idx[:, 2]] != 0
        if not inside.all():
            print(f"[compute_activation_maps] WARNING: {int((~inside).sum()):,} myocardial "
                  "nodes fall outside the provided S mask")
        return np.array(S.shape, dtype=np.int32)
    return (np.asarray(vox_idx).max(axis=0) + 1).astype(np.int32)


def _finish(act, dea, *, node_ids, coords_mm, vox_idx, grid_shape, act_threshold,
            deact_threshold, min_event_gap_ms, source, save_path):
    act = _debounce(act, min_event_gap_ms)
    dea = _debounce(dea, min_event_gap_ms)
    maps = ActivationMaps(
        node_ids=np.asarray(node_ids, np.int32), coords_mm=np.asarray(coords_mm, np.float32),
        vox_idx=np.asarray(vox_idx, np.int32), grid_shape=grid_shape,
        activation_times=act, deactivation_times=dea,
        n_activations=(~np.isnan(act)).sum(axis=1).astype(np.int32),
        n_deactivations=(~np.isnan(dea)).sum(axis=1).astype(np.int32),
        act_threshold=float(act_threshold), deact_threshold=float(deact_threshold),
        source_vm_path=str(source),
        path=Path(save_path) if save_path is not None else Path("."))
    if save_path is not None:
        save_activation_maps(maps, save_path)
    return maps


def compute_activation_maps(vm_snapshots, S=None, *, act_threshold: float = -40.0,
                            deact_threshold: float = -40.0, min_event_gap_ms=None,
                            save_path=None) -> ActivationMaps:
    """Maps from a ``VmSnapshots`` (activation_maps.py:295-413)."""
    Vm, t, n = vm_snapshots.Vm, vm_snapshots.time_vm, vm_snapshots.N_myo
    if vm_snapshots.n_frames < 2:
        raise ValueError("vm_snapshots has fewer than 2 frames -- cannot detect threshold "
                         "crossings. Re-run the simulation with a smaller vm_save_dt / longer T.")
    up = np.diff((Vm >= act_threshold).astype(np.int8), axis=0) == 1
    down = np.diff((Vm >= deact_threshold).astype(np.int8), axis=0) == -1
    act = _table(*_crossings(Vm, t, up, act_threshold), n)
    dea = _table(*_crossings(Vm, t, down, deact_threshold), n)
    return _finish(act, dea, node_ids=vm_snapshots.node_ids, coords_mm=vm_snapshots.coords_mm,
                   vox_idx=vm_snapshots.vox_idx,
                   grid_shape=_grid_shape(S, vm_snapshots.vox_idx),
                   act_threshold=act_threshold, deact_threshold=deact_threshold,
                   min_event_gap_ms=min_event_gap_ms, source=vm_snapshots.path,
                   save_path=save_path)


def activation_maps_from_run(results, S, *, act_threshold: float, deact_threshold: float,
                             min_event_gap_ms=None, save_path=None) -> ActivationMaps:
    """Maps from the in-loop event tables of a monodomain run (the dict
    ``run_coupled`` / ``purkinje_myocardium_anisotropic_solver`` return:
    ``activation_times``, ``deactivation_times``, ``node_ids``,
    ``coords_mm``, ``vox_idx``).  The thresholds must be the ones the run
    recorded with."""
    vox = np.asarray(results["vox_idx"])
    return _finish(np.asarray(results["activation_times"], np.float32),
                   np.asarray(results["deactivation_times"], np.float32),
                   node_ids=results["node_ids"], coords_mm=results["coords_mm"], vox_idx=vox,
                   grid_shape=_grid_shape(S, vox), act_threshold=act_threshold,
                   deact_threshold=deact_threshold, min_event_gap_ms=min_event_gap_ms,
                   source=results.get("vm_snapshots_path", ""), save_path=save_path)


def save_activation_maps(maps: ActivationMaps, path) -> None:
    path = _npz_path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    d = dict(node_ids=maps.node_ids.astype(np.int32), coords_mm=maps.coords_mm.astype(np.float32),
             vox_idx=maps.vox_idx.astype(np.int32),
             activation_times=maps.activation_times.astype(np.float32),
             deactivation_times=maps.deactivation_times.astype(np.float32),
             n_activations=maps.n_activations.astype(np.int32),
             n_deactivations=maps.n_deactivations.astype(np.int32),
             act_threshold=np.float32(maps.act_threshold),
             deact_threshold=np.float32(maps.deact_threshold),
             source_vm_path=str(maps.source_vm_path))
    if maps.grid_shape is not None:
        d["grid_shape"] = np.asarray(maps.grid_shape, np.int32)
    np.savez_compressed(path, **d)
    maps.path = path


def load_activation_maps(path) -> ActivationMaps:
    """FileNotFoundError if absent, KeyError if a required array is missing."""
    path = _npz_path(path)
    if not path.exists():
        raise FileNotFoundError(f"activation_maps file not found: {path}")
    d = np.load(str(path), allow_pickle=False)
    missing = set(REQUIRED) - set(d.files)
    if missing:
        raise KeyError(f"activation_maps NPZ is missing keys: {missing} (found: {d.files})")
    return ActivationMaps(
        node_ids=d["node_ids"], coords_mm=d["coords_mm"], vox_idx=d["vox_idx"],
        activation_times=d["activation_times"], deactivation_times=d["deactivation_times"],
        n_activations=d["n_activations"], n_deactivations=d["n_deactivations"],
        act_threshold=float(d["act_threshold"]), deact_threshold=float(d["deact_threshold"]),
        grid_shape=d["grid_shape"] if "grid_shape" in d.files else None,
        source_vm_path=str(d["source_vm_path"]) if "source_vm_path" in d.files else "",
        path=path)
