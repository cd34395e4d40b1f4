"""Drop-in for hrdayapy.ecg: torso grid and body-surface potential maps."""
from .bspm import compute_bspm, load_bspm, run_bspm_loop
from .torso_grid import compute_torso_grid, load_torso_grid, torso_grid_from_labels

__all__ = ["compute_bspm", "load_bspm", "run_bspm_loop", "compute_torso_grid",
           "load_torso_grid", "torso_grid_from_labels"]
