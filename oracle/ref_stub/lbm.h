// Stand-in for solver/lbm3d/lbm.h when solver/lbm3d/core.h is compiled on the host by
// oracle/ref_shim.cpp (test infrastructure only).  The real header holds the TNL-backed
// LBM storage class, which the shim replaces by its own plain arrays (ShimData); nothing
// of it is needed to compile core.h's per-cell kernels.
#pragma once
