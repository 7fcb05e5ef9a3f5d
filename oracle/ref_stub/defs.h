// Stand-in for solver/lbm3d/defs.h of buresjan/nonnewlbm when its headers are compiled on
// the host by oracle/ref_shim.cpp (test infrastructure only).
//
// The real defs.h pulls TNL, libpng and MPI, none of which is needed by the per-cell
// kernels.  This file declares what solver/lbm3d/core.h and the collision / equilibrium /
// streaming / boundary headers expect from it, with the reference's member names and
// values: the CUDA_HOSTDEV macros (defs.h:26-32), the df_cur/df_out enum (:34-40), the
// Traits template (:42-60), KernelStruct with the Carreau-Yasuda members of the production
// build (USE_CYMODEL, :143-160), the 27-direction enum (:215-247) and the helper macros.
// oracle/Makefile puts this directory before the reference's with -I-, so that core.h's
// own #include "defs.h" lands here.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <utility>

#include "ciselnik.h"

#ifndef USE_CYMODEL
#define USE_CYMODEL
#endif
#define CUDA_HOSTDEV
#define CUDA_HOSTDEV_NOINLINE

enum : uint8_t { df_cur, df_out, DFMAX };

template <typename _dreal = float, typename _real = double, typename _idx = long int, typename _map_t = short int>
struct Traits {
    using real = _real;
    using dreal = _dreal;
    using idx = _idx;
    using map_t = _map_t;
};

template <typename REAL>
struct KernelStruct {
    REAL fz = 0, fx = 0, fy = 0;
    REAL f[27];
    REAL vz = 0, vx = 0, vy = 0, rho = 1.0, lbmViscosity = 1.0;
    REAL S11 = 0., S12 = 0., S22 = 0., S32 = 0., S13 = 0., S33 = 0.;
    REAL lbm_nu0 = 0, lbm_lambda = 0, lbm_a = 0, lbm_n = 0;
    REAL mu;
};

enum {
    mmm = 0, mmz, mmp, mzm, mzz, mzp, mpm, mpz, mpp,
    zmm, zmz, zmp, zzm, zzz, zzp, zpm, zpz, zpp,
    pmm, pmz, pmp, pzm, pzz, pzp, ppm, ppz, ppp
};

#define MAX(a, b) (((a) > (b)) ? (a) : (b))
#define MIN(a, b) (((a) < (b)) ? (a) : (b))
#define SQ(x) ((x) * (x))
#define NORM(x, y, z) sqrt(SQ(x) + SQ(y) + SQ(z))

// The Carreau-Yasuda law of core.h:765 calls powf with double arguments when dreal is
// double.  C's powf rounds its arguments to float and glibc returns a result within an
// ulp of the exact power, not always the correctly rounded one; the FP64 GPU mode and the
// C oracle both use the correctly rounded float power, so this overload (chosen over C's
// powf(float, float) for double arguments) returns that: arguments rounded to float, the
// power taken in double and rounded once.  Single-precision builds call glibc's powf.
inline float powf(double b, double e) { return (float)std::pow((double)(float)b, (double)(float)e); }
