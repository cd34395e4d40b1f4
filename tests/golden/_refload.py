"""Loader for the upstream HrdayaPy sources, used only by make_golden.py.

The upstream package cannot be imported as a whole here (its coordinate
stage needs pynrrd/pyvista/skimage), so the hot-path modules are loaded by
file path under stub parent packages.  `build_surface_mesh` (marching cubes,
animation-only) is replaced by a stub because skimage is absent.
"""
from __future__ import annotations

import importlib.util
import os
import sys
import types
from pathlib import Path

import numpy as np

# root of the upstream HrdayaPy checkout (the directory holding hrdayapy/)
REF_ROOT = Path(os.environ.get("HRDAYAPY_REF_ROOT", "/root/reference"))


def _pkg(name: str, path: Path) -> None:
    if name in sys.modules:
        return
    m = types.ModuleType(name)
    m.__path__ = [str(path)]
    sys.modules[name] = m


def _load(modname: str, path: Path):
    if modname in sys.modules:
        return sys.modules[modname]
    spec = importlib.util.spec_from_file_location(modname, str(path))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[modname] = mod
    spec.loader.exec_module(mod)
    return mod


def _stub_surface(Z, myo, voxel_size):
    return (np.zeros((0, 3), np.float32), np.zeros((0, 3), np.int32),
            np.zeros(0, np.int32))


def load():
    """Return a namespace with the upstream hot-path modules."""
    hp = REF_ROOT / "hrdayapy"
    _pkg("hrdayapy", hp)
    ns = types.SimpleNamespace()
    for stage in ("simulation", "anisotropic_simulation"):
        _pkg(f"hrdayapy.{stage}", hp / stage)
        _pkg(f"hrdayapy.{stage}.functions", hp / stage / "functions")
        _pkg(f"hrdayapy.{stage}.functions.ionic_models",
             hp / stage / "functions" / "ionic_models")
        base = f"hrdayapy.{stage}.functions"
        im = f"{base}.ionic_models"
        _load(f"{im}.ttp06_phenotype_constants",
              hp / stage / "functions" / "ionic_models" / "ttp06_phenotype_constants.py")
        g = _load(f"{im}.gpu_ttp06", hp / stage / "functions" / "ionic_models" / "gpu_ttp06.py")
        _load(f"{im}.hetero_solver", hp / stage / "functions" / "ionic_models" / "hetero_solver.py")
        if stage == "simulation":
            ns.gpu_ttp06 = g
            ns.pipeline = _load(f"{base}.purkinje_myocardium_pipeline",
                                hp / stage / "functions" / "purkinje_myocardium_pipeline.py")
            ns.pipeline.build_surface_mesh = _stub_surface
            ns.activation_maps = _load(f"{base}.activation_maps",
                                       hp / stage / "functions" / "activation_maps.py")
            ns.load_vm_snapshots = _load(f"{base}.load_vm_snapshots",
                                         hp / stage / "functions" / "load_vm_snapshots.py")
        else:
            ns.aniso = _load(f"{base}.purkinje_myocardium_anisotropic_solver",
                             hp / stage / "functions" / "purkinje_myocardium_anisotropic_solver.py")
            ns.aniso.build_surface_mesh = _stub_surface
    _pkg("hrdayapy.ecg", hp / "ecg")
    _pkg("hrdayapy.ecg.functions", hp / "ecg" / "functions")
    ns.compute_bspm = _load("hrdayapy.ecg.functions.compute_bspm",
                            hp / "ecg" / "functions" / "compute_bspm.py")
    ns.build_torso_grid = _load("hrdayapy.ecg.functions.build_torso_grid",
                                hp / "ecg" / "functions" / "build_torso_grid.py")
    return ns
