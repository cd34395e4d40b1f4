"""Vm snapshot files: the container and loader of the reference's
simulation/functions/load_vm_snapshots.py:49-240, for the npz files that
``monodomain.save_vm_snapshots`` writes (same schema, load_vm_snapshots.py
:7-16): node_ids (N_myo,) int32, coords_mm (N_myo, 3) float32, vox_idx
(N_myo, 3) int32, Vm (n_frames, N_myo) float32, time_vm (n_frames,) float32,
dt_solver and vm_save_dt float32 scalars.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

REQUIRED = ("node_ids", "coords_mm", "vox_idx", "Vm", "time_vm", "dt_solver", "vm_save_dt")


@dataclass
class VmSnapshots:
    node_ids: np.ndarray
    coords_mm: np.ndarray
    vox_idx: np.ndarray
    Vm: np.ndarray
    time_vm: np.ndarray
    dt_solver: float
    vm_save_dt: float
    path: Path = field(default_factory=lambda: Path("."))

    @property
    def n_frames(self) -> int:
        return int(self.Vm.shape[0])

    @property
    def N_myo(self) -> int:
        return int(self.Vm.shape[1])

    def __repr__(self) -> str:
        t = self.time_vm
        return (f"VmSnapshots(N_myo={self.N_myo:,}, n_frames={self.n_frames}, "
                f"t=[{t[0]:.2f}…{t[-1]:.2f}] ms, vm_save_dt={self.vm_save_dt:.4g} ms, "
                f"Vm=[{self.Vm.min():.1f}, {self.Vm.max():.1f}] mV)")

    def vm_at_node(self, local_id: int) -> np.ndarray:
        """Vm time series of myocardial node ``local_id`` (0 .. N_myo-1)."""
        if not 0 <= local_id < self.N_myo:
            raise IndexError(f"local_id {local_id} out of range [0, {self.N_myo})")
        return self.Vm[:, local_id]

    def _dist(self, p):
        p = np.asarray(p, dtype=np.float32)
        return np.linalg.norm(self.coords_mm - p[None, :], axis=1)

    def nearest_node(self, point_mm) -> int:
        """Local index of the node closest to ``point_mm`` (x, y, z mm)."""
        return int(self._dist(point_mm).argmin())

    def field_at_time(self, t_ms: float):
        """(Vm field, its time) of the frame closest to ``t_ms``."""
        i = int(np.argmin(np.abs(self.time_vm - t_ms)))
        return self.Vm[i], float(self.time_vm[i])

    def nodes_in_sphere(self, centre_mm, radius_mm: float) -> np.ndarray:
        return np.nonzero(self._dist(centre_mm) <= radius_mm)[0].astype(np.int32)

    def mean_vm_in_sphere(self, centre_mm, radius_mm: float) -> np.ndarray:
        ids = self.nodes_in_sphere(centre_mm, radius_mm)
        if ids.size == 0:
            return np.zeros(self.n_frames, dtype=np.float32)
        return self.Vm[:, ids].mean(axis=1)


def _npz_path(path) -> Path:
    path = Path(path)
    return path if path.suffix else path.with_suffix(".npz")


def load_vm_snapshots(path) -> VmSnapshots:
    """Loads a vm_snapshots npz.  FileNotFoundError if absent, KeyError if a
    required array is missing (load_vm_snapshots.py:198-240)."""
    path = _npz_path(path)
    if not path.exists():
        raise FileNotFoundError(f"vm_snapshots file not found: {path}")
    d = np.load(str(path))
    missing = set(REQUIRED) - set(d.files)
    if missing:
        raise KeyError(f"vm_snapshots NPZ is missing keys: {missing} (found: {d.files})")
    return VmSnapshots(node_ids=d["node_ids"], coords_mm=d["coords_mm"], vox_idx=d["vox_idx"],
                       Vm=d["Vm"], time_vm=d["time_vm"], dt_solver=float(d["dt_solver"]),
                       vm_save_dt=float(d["vm_save_dt"]), path=path)
