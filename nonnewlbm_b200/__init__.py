"""nonnewlbm_b200 -- B200-native fused D3Q27 stream + collide step of the TCPC
lattice-Boltzmann solver (buresjan/nonnewlbm), behind the C ABI of include/nnlbm.h.

The compute path is libnnlbm.so (hand-written sm_100a kernels, built in-tree by
``nonnewlbm_b200.build``); this package holds the ctypes binding and the host layer that
mirrors the reference's Python scripts and configuration.
"""
from . import capi, geometry
from .lattice import CaseSpec, Lattice

__all__ = ["capi", "geometry", "CaseSpec", "Lattice"]
