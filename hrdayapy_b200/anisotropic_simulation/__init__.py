"""Drop-in for hrdayapy.anisotropic_simulation (fibre-tensor monodomain)."""
from .coupled import (compute_anisotropic_coupled, load_anisotropic_coupled,
                      purkinje_myocardium_anisotropic_solver)

__all__ = ["compute_anisotropic_coupled", "load_anisotropic_coupled",
           "purkinje_myocardium_anisotropic_solver"]
