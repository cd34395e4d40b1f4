"""ORACLE -- test infrastructure, not product code.

FP64 CPU restatements of HrdayaPy's monodomain and torso-ECG hot path.
Only tests/, ``__graft_entry__.smoke()`` (as the checker) and ``bench.py``'s
CPU-baseline leg may import this package; the product never does.
"""
