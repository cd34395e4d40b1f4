"""Drop-in for hrdayapy.simulation (isotropic coupled monodomain)."""
from .coupled import compute_coupled, load_coupled, run_coupled

__all__ = ["compute_coupled", "load_coupled", "run_coupled"]
