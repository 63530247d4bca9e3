"""B200 (sm_100a) implementation of GITM's vertical advance.

The compute path is the CUDA library ``libgitmvert.so`` built from
``gitm_b200/csrc``; this package holds its ctypes binding, the host-side
mirror of the reference's calling interface and the synthetic workloads.
"""
__version__ = "0.1.0"
