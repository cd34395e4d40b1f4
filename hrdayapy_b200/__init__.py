"""hrdayapy_b200 -- B200-native (sm_100a) implementation of HrdayaPy's
monodomain time-stepping and body-surface ECG forward solve.

Sub-packages mirror the reference's stage API:
    hrdayapy_b200.simulation              compute_coupled / run_coupled
    hrdayapy_b200.anisotropic_simulation  compute_anisotropic_coupled
    hrdayapy_b200.ecg                     compute_bspm / compute_torso_grid
All compute runs in libhrdaya_b200.so (CUDA, sm_100a); there is no CPU path.
"""
__version__ = "0.1.0"
