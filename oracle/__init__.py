"""CPU FP64 oracle for PBT far-field diffraction (test infrastructure only).

Only tests/, __graft_entry__.smoke() (as the checker) and bench.py's CPU
baseline leg use this package.  The product library never imports it.
"""
