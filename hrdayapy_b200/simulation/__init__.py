"""Drop-in for hrdayapy.simulation (isotropic coupled monodomain), with the
reference's snapshot loader and activation-map helpers
(simulation/__init__.py of the reference)."""
from .activation_maps import (ActivationMaps, activation_maps_from_run, compute_activation_maps,
                              load_activation_maps, save_activation_maps)
from .coupled import compute_coupled, load_coupled, run_coupled
from .vm_snapshots import VmSnapshots, load_vm_snapshots

__all__ = ["compute_coupled", "load_coupled", "run_coupled", "load_vm_snapshots", "VmSnapshots",
           "compute_activation_maps", "load_activation_maps", "save_activation_maps",
           "ActivationMaps", "activation_maps_from_run"]
