// ref_shim.cpp -- builds the reference's own collision, equilibrium, streaming and generic
// boundary-condition headers (solver/lbm3d/*.h of buresjan/nonnewlbm, included unmodified
// from the reference checkout) into oracle/_ref/libnnlbm_ref.so.
//
// TEST INFRASTRUCTURE ONLY: used to pin the C oracle (known-answer vectors under
// tests/golden/) and, in its single-precision build, as the timed CPU baseline of
// bench.py.  Nothing in the product links it.
//
// The reference's defs.h cannot be included (it pulls TNL, libpng and MPI), so this file
// declares the few interface types those headers expect: the CUDA_HOSTDEV macros, the
// df_cur/df_out enum, the 27-direction enum and a KernelStruct with the member names the
// headers use (solver/lbm3d/defs.h:26-40,143-160,215-247).  The kernel driver at the end
// is a restatement of the single-rank host loop (solver/lbm3d/core.h:1312-1320) around
// LBMKernel (core.h:578-800) and the TCPC policies (solver/sim_tcpc/sim_tcpc.cu:187-354),
// calling the reference templates for every per-cell operation.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <utility>
#ifdef _OPENMP
#include <omp.h>
#endif

#define CUDA_HOSTDEV
#define CUDA_HOSTDEV_NOINLINE
#define USE_CYMODEL

enum : uint8_t { df_cur, df_out, DFMAX };

enum {
    mmm = 0, mmz, mmp, mzm, mzz, mzp, mpm, mpz, mpp,
    zmm, zmz, zmp, zzm, zzz, zzp, zpm, zpz, zpp,
    pmm, pmz, pmp, pzm, pzz, pzp, ppm, ppz, ppp
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

template <typename DREAL>
struct ShimTraits {
    using real = double;
    using dreal = DREAL;
    using idx = long;
    using map_t = short;
};

#include "ciselnik.h"
#include "lbm_eq.h"
#include "lbm_eq_inv_cum.h"
#include "lbm_eq_entropic.h"
#include "lbm_common.h"
#include "lbm_streaming.h"
#include "lbm_col_cum.h"
#include "lbm_col_mrt.h"
#include "lbm_col_bgk.h"
#include "lbm_col_kbc_n.h"
#include "lbm_col_kbc_c.h"
#include "lbm_bc.h"

namespace {

// equilibrium selector: 0 = LBM_EQ_INV_CUM (as shipped), 2 = LBM_EQ_DEFAULT,
// 3 = LBM_EQ_ENTROPIC.  (1, the corrected factorised equilibrium, has no reference
// counterpart and is not provided here.)
template <typename T, int EQ> struct EqSel;
template <typename T> struct EqSel<T, 0> { using type = LBM_EQ_INV_CUM<ShimTraits<T>>; };
template <typename T> struct EqSel<T, 2> { using type = LBM_EQ_DEFAULT<ShimTraits<T>>; };
template <typename T> struct EqSel<T, 3> { using type = LBM_EQ_ENTROPIC<ShimTraits<T>>; };

template <typename T, int COL, typename EQ> struct ColSel;
template <typename T, typename EQ> struct ColSel<T, 0, EQ> { using type = LBM_CUM<ShimTraits<T>, EQ>; };
template <typename T, typename EQ> struct ColSel<T, 1, EQ> { using type = LBM_KBC_N1<ShimTraits<T>, EQ>; };
template <typename T, typename EQ> struct ColSel<T, 2, EQ> { using type = LBM_KBC_N2<ShimTraits<T>, EQ>; };
template <typename T, typename EQ> struct ColSel<T, 3, EQ> { using type = LBM_KBC_N3<ShimTraits<T>, EQ>; };
template <typename T, typename EQ> struct ColSel<T, 4, EQ> { using type = LBM_KBC_N4<ShimTraits<T>, EQ>; };
template <typename T, typename EQ> struct ColSel<T, 5, EQ> { using type = LBM_KBC_C1<ShimTraits<T>, EQ>; };
template <typename T, typename EQ> struct ColSel<T, 6, EQ> { using type = LBM_KBC_C2<ShimTraits<T>, EQ>; };
template <typename T, typename EQ> struct ColSel<T, 7, EQ> { using type = LBM_KBC_C3<ShimTraits<T>, EQ>; };
template <typename T, typename EQ> struct ColSel<T, 8, EQ> { using type = LBM_KBC_C4<ShimTraits<T>, EQ>; };
template <typename T, typename EQ> struct ColSel<T, 9, EQ> { using type = LBM_MRT<ShimTraits<T>, EQ>; };
template <typename T, typename EQ> struct ColSel<T, 10, EQ> { using type = LBM_BGK<ShimTraits<T>, EQ>; };

// ---------------------------------------------------------------------------------
// lattice data adaptor with the reference index map y + Y*(z + Z*(q + 27*x))
// (solver/lbm3d/lbm_data.h:296-312)
// ---------------------------------------------------------------------------------
template <typename T>
struct ShimData {
    T* dfs[DFMAX];
    long X_, Y_, Z_;
    long X() const { return X_; }
    long Y() const { return Y_; }
    long Z() const { return Z_; }
    T& df(uint8_t type, int q, long x, long y, long z) { return dfs[type][y + Y_ * (z + Z_ * (q + 27 * x))]; }
    // inflow data (LBM_Data_Tcpc, sim_tcpc.cu:288-309; generic per-cell inflow)
    T inflow_left = 0, inflow_right = 0, inflow_rho_left = 1, inflow_rho_right = 1, inflow_rho_eq = 1;
    long inflow_left_area = 0, inflow_right_area = 0;
    const double* prof = nullptr; // [3][N], N over x fastest
    void inflowConditionLeft(KernelStruct<T>& KS, long, long, long)
    {
        KS.rho = inflow_rho_left;
        KS.vx = inflow_left_area > 0 ? inflow_left / (T)inflow_left_area : (T)0;
        KS.vy = (T)0;
        KS.vz = (T)0;
    }
    void inflowConditionRight(KernelStruct<T>& KS, long, long, long)
    {
        KS.rho = inflow_rho_right;
        KS.vx = inflow_right_area > 0 ? inflow_right / (T)inflow_right_area : (T)0;
        KS.vy = (T)0;
        KS.vz = (T)0;
    }
    void inflow(KernelStruct<T>& KS, long x, long y, long z)
    {
        long c = x + X_ * (y + Y_ * z), N = X_ * Y_ * Z_;
        KS.rho = inflow_rho_eq;
        KS.vx = (T)prof[c];
        KS.vy = (T)prof[N + c];
        KS.vz = (T)prof[2 * N + c];
    }
};

enum { L_FLUID = 0, L_WALL = 1, L_PERIODIC = 2, L_IN_L = 3, L_IN_R = 4, L_OUT_F = 5, L_OUT_B = 6, L_IN_EQ = 7, L_OUT_REQ = 8 };

struct Lattice {
    int prec; // 8 or 4
    int col, eq;
    long X, Y, Z, N;
    double nu, fx, fy, fz;
    uint8_t* map;
    void* df[2];
    int cur;
    double* prof;
    void* macro; // [7 + 7 stats][N]: rho vx vy vz fx fy fz | vm+x vm-x vmy vmz vmxx vmyy vmzz
    double ivc_flux = 0, svc_flux = 0, rho_l = 1, rho_r = 1, rho_eq = 1;
    long left_area = 0, right_area = 0;
};

template <typename T, typename LT>
void cell_step(Lattice& L, ShimData<T>& SD, T* macro, long x, long y, long z, int acc)
{
    using S = LBM_STREAMING<ShimTraits<T>>;
    using BCG = LBM_BC_All<ShimTraits<T>>;
    using dreal = T;
    const long c = x + L.X * (y + L.Y * z);
    const int lab = L.map[c];
    KernelStruct<T> KS;
    KS.lbmViscosity = (T)L.nu;
    KS.fx = (T)L.fx; KS.fy = (T)L.fy; KS.fz = (T)L.fz;
    long xp, xm, yp, ym, zp, zm;
    if (lab == L_PERIODIC) {
        xp = x == L.X - 1 ? 0 : x + 1; xm = x == 0 ? L.X - 1 : x - 1;
        yp = y == L.Y - 1 ? 0 : y + 1; ym = y == 0 ? L.Y - 1 : y - 1;
        zp = z == L.Z - 1 ? 0 : z + 1; zm = z == 0 ? L.Z - 1 : z - 1;
    } else {
        xp = std::min(x + 1, L.X - 1); xm = std::max(x - 1, 0L);
        yp = std::min(y + 1, L.Y - 1); ym = std::max(y - 1, 0L);
        zp = std::min(z + 1, L.Z - 1); zm = std::max(z - 1, 0L);
    }
    if (lab == L_FLUID || lab == L_PERIODIC) {
        S::streaming(SD, KS, xm, x, xp, ym, y, yp, zm, z, zp);
        LT::computeDensityAndVelocity(KS);
        LT::collision(KS);
    } else if (lab == L_WALL) {
        BCG::template BC<LT, S, ShimData<T>>(SD, KS, BCG::GEO_WALL, xm, x, xp, ym, y, yp, zm, z, zp);
    } else if (lab == L_IN_L) {
        SD.inflowConditionLeft(KS, x, y, z);
        KernelStruct<T> KS_loc;
        S::streaming(SD, KS_loc, x, xp, xp + 1, ym, y, yp, zm, z, zp);
        LT::computeDensityAndVelocity(KS_loc);
        KS.rho = KS_loc.rho;
        LT::setEquilibrium(KS);
    } else if (lab == L_IN_R) {
        SD.inflowConditionRight(KS, x, y, z);
        KernelStruct<T> KS_loc;
        S::streaming(SD, KS_loc, xm - 1, xm, x, ym, y, yp, zm, z, zp);
        LT::computeDensityAndVelocity(KS_loc);
        KS.rho = KS_loc.rho;
        LT::setEquilibrium(KS);
    } else if (lab == L_OUT_F) {
        S::streaming(SD, KS, xm, x, xp, y, yp, yp + 1, zm, z, zp);
        LT::computeDensityAndVelocity(KS);
        KS.rho = no1;
        LT::setEquilibrium(KS);
    } else if (lab == L_OUT_B) {
        S::streaming(SD, KS, xm, x, xp, ym - 1, ym, y, zm, z, zp);
        LT::computeDensityAndVelocity(KS);
        KS.rho = no1;
        LT::setEquilibrium(KS);
    } else if (lab == L_IN_EQ) {
        // GEO_INFLOW streams first (isStreaming) and then overwrites everything
        BCG::template BC<LT, S, ShimData<T>>(SD, KS, BCG::GEO_INFLOW, xm, x, xp, ym, y, yp, zm, z, zp);
    } else if (lab == L_OUT_REQ) {
        S::streaming(SD, KS, xm, x, xp, ym, y, yp, zm, z, zp);
        LT::computeDensityAndVelocity(KS);
        BCG::template BC<LT, S, ShimData<T>>(SD, KS, BCG::GEO_OUTFLOW_RIGHT_EQ, xm, x, xp, ym, y, yp, zm, z, zp);
    }
    LT::copyKS2DFout(SD, KS, x, y, z);
    const long N = L.N;
    macro[0 * N + c] = KS.rho; macro[1 * N + c] = KS.vx; macro[2 * N + c] = KS.vy; macro[3 * N + c] = KS.vz;
    macro[4 * N + c] = KS.fx; macro[5 * N + c] = KS.fy; macro[6 * N + c] = KS.fz;
    if (acc) {
        macro[7 * N + c] += (KS.vx > 0) ? KS.rho * KS.vx : 0;
        macro[8 * N + c] += (KS.vx < 0) ? KS.rho * KS.vx : 0;
        macro[9 * N + c] += KS.rho * KS.vy;
        macro[10 * N + c] += KS.rho * KS.vz;
        macro[11 * N + c] += KS.rho * KS.rho * KS.vx * KS.vx;
        macro[12 * N + c] += KS.rho * KS.rho * KS.vy * KS.vy;
        macro[13 * N + c] += KS.rho * KS.rho * KS.vz * KS.vz;
    }
}

template <typename T, typename LT>
void lattice_step(Lattice& L, int acc)
{
    ShimData<T> SD;
    SD.dfs[df_cur] = (T*)L.df[L.cur];
    SD.dfs[df_out] = (T*)L.df[1 - L.cur];
    SD.X_ = L.X; SD.Y_ = L.Y; SD.Z_ = L.Z;
    SD.inflow_left = (T)L.ivc_flux;
    SD.inflow_right = (T)(-L.svc_flux);
    SD.inflow_rho_left = (T)L.rho_l;
    SD.inflow_rho_right = (T)L.rho_r;
    SD.inflow_rho_eq = (T)L.rho_eq;
    SD.inflow_left_area = L.left_area;
    SD.inflow_right_area = L.right_area;
    SD.prof = L.prof;
    T* macro = (T*)L.macro;
    // core.h:1313-1320 loop order
#pragma omp parallel for schedule(static) collapse(2) firstprivate(SD)
    for (long x = 0; x < L.X; x++)
        for (long z = 0; z < L.Z; z++)
            for (long y = 0; y < L.Y; y++) cell_step<T, LT>(L, SD, macro, x, y, z, acc);
    L.cur = 1 - L.cur;
}

template <typename T, typename LT>
void lattice_init(Lattice& L, double rho, double vx, double vy, double vz)
{
    KernelStruct<T> KS;
    KS.rho = (T)rho; KS.vx = (T)vx; KS.vy = (T)vy; KS.vz = (T)vz;
    LT::setEquilibrium(KS);
    for (int k = 0; k < 2; ++k) {
        T* a = (T*)L.df[k];
        for (long x = 0; x < L.X; ++x)
            for (int q = 0; q < 27; ++q)
                for (long z = 0; z < L.Z; ++z)
                    for (long y = 0; y < L.Y; ++y) a[y + L.Y * (z + L.Z * (q + 27 * x))] = KS.f[q];
    }
    L.cur = 0;
}

template <typename T, int COL, int EQ>
struct Ops {
    using LT = typename ColSel<T, COL, typename EqSel<T, EQ>::type>::type;
    static void step(Lattice& L, int acc) { lattice_step<T, LT>(L, acc); }
    static void init(Lattice& L, double r, double a, double b, double c) { lattice_init<T, LT>(L, r, a, b, c); }
    static void collide(double nu, double* f, double rho, double vx, double vy, double vz, double fx, double fy, double fz)
    {
        KernelStruct<T> KS;
        for (int q = 0; q < 27; ++q) KS.f[q] = (T)f[q];
        KS.rho = (T)rho; KS.vx = (T)vx; KS.vy = (T)vy; KS.vz = (T)vz;
        KS.fx = (T)fx; KS.fy = (T)fy; KS.fz = (T)fz;
        KS.lbmViscosity = (T)nu;
        LT::collision(KS);
        for (int q = 0; q < 27; ++q) f[q] = (double)KS.f[q];
    }
    static void feq(double rho, double vx, double vy, double vz, double* f)
    {
        KernelStruct<T> KS;
        KS.rho = (T)rho; KS.vx = (T)vx; KS.vy = (T)vy; KS.vz = (T)vz;
        LT::setEquilibrium(KS);
        for (int q = 0; q < 27; ++q) f[q] = (double)KS.f[q];
    }
    static void dv(const double* f, double fx, double fy, double fz, double* out)
    {
        KernelStruct<T> KS;
        for (int q = 0; q < 27; ++q) KS.f[q] = (T)f[q];
        KS.fx = (T)fx; KS.fy = (T)fy; KS.fz = (T)fz;
        LT::computeDensityAndVelocity(KS);
        out[0] = KS.rho; out[1] = KS.vx; out[2] = KS.vy; out[3] = KS.vz;
    }
};

template <typename T, int COL, int EQ>
void dispatch_eq_col(int what, Lattice* L, int acc, double* a, double* b)
{
    using O = Ops<T, COL, EQ>;
    switch (what) {
    case 0: O::step(*L, acc); break;
    case 1: O::init(*L, a[0], a[1], a[2], a[3]); break;
    case 2: O::collide(a[0], b, a[1], a[2], a[3], a[4], a[5], a[6], a[7]); break;
    case 3: O::feq(a[0], a[1], a[2], a[3], b); break;
    case 4: O::dv(b, a[0], a[1], a[2], a + 3); break;
    }
}

template <typename T, int COL>
int dispatch_eq(int eq, int what, Lattice* L, int acc, double* a, double* b)
{
    switch (eq) {
    case 0: dispatch_eq_col<T, COL, 0>(what, L, acc, a, b); return 0;
    case 2: dispatch_eq_col<T, COL, 2>(what, L, acc, a, b); return 0;
    case 3: dispatch_eq_col<T, COL, 3>(what, L, acc, a, b); return 0;
    }
    return -1;
}

template <typename T>
int dispatch(int col, int eq, int what, Lattice* L, int acc, double* a, double* b)
{
    switch (col) {
    case 0: return dispatch_eq<T, 0>(eq, what, L, acc, a, b);
    case 1: return dispatch_eq<T, 1>(eq, what, L, acc, a, b);
    case 2: return dispatch_eq<T, 2>(eq, what, L, acc, a, b);
    case 3: return dispatch_eq<T, 3>(eq, what, L, acc, a, b);
    case 4: return dispatch_eq<T, 4>(eq, what, L, acc, a, b);
    case 5: return dispatch_eq<T, 5>(eq, what, L, acc, a, b);
    case 6: return dispatch_eq<T, 6>(eq, what, L, acc, a, b);
    case 7: return dispatch_eq<T, 7>(eq, what, L, acc, a, b);
    case 8: return dispatch_eq<T, 8>(eq, what, L, acc, a, b);
    case 9: return dispatch_eq<T, 9>(eq, what, L, acc, a, b);
    case 10: return dispatch_eq<T, 10>(eq, what, L, acc, a, b);
    }
    return -1;
}

int run(int prec, int col, int eq, int what, Lattice* L, int acc, double* a, double* b)
{
    return prec == 4 ? dispatch<float>(col, eq, what, L, acc, a, b) : dispatch<double>(col, eq, what, L, acc, a, b);
}

} // namespace

extern "C" {

// per-cell known answers (FP64 or FP32 reference arithmetic; inputs/outputs in double)
int ref_feq(int prec, int eq, double rho, double vx, double vy, double vz, double* f)
{
    double a[4] = {rho, vx, vy, vz};
    return run(prec, 0, eq, 3, nullptr, 0, a, f);
}

int ref_density_velocity(int prec, const double* f, double fx, double fy, double fz, double* out)
{
    double a[7] = {fx, fy, fz, 0, 0, 0, 0};
    double fb[27];
    memcpy(fb, f, sizeof fb);
    int rc = run(prec, 0, 0, 4, nullptr, 0, a, fb);
    memcpy(out, a + 3, 4 * sizeof(double));
    return rc;
}

int ref_collide(int prec, int col, double nu, double* f, double rho, double vx, double vy, double vz,
                double fx, double fy, double fz)
{
    double a[8] = {nu, rho, vx, vy, vz, fx, fy, fz};
    return run(prec, col, 0, 2, nullptr, 0, a, f);
}

// lattice: map labels 0..8 as in the C oracle; df exported as [27][N], x fastest
void* ref_create(int prec, int nx, int ny, int nz, int col, int eq, double nu, double fx, double fy, double fz)
{
    if (nx < 3 || ny < 3 || nz < 3 || (prec != 4 && prec != 8)) return nullptr;
    Lattice* L = new Lattice();
    L->prec = prec; L->col = col; L->eq = eq;
    L->X = nx; L->Y = ny; L->Z = nz; L->N = (long)nx * ny * nz;
    L->nu = nu; L->fx = fx; L->fy = fy; L->fz = fz;
    L->map = (uint8_t*)calloc(L->N, 1);
    L->df[0] = calloc(L->N * 27, prec);
    L->df[1] = calloc(L->N * 27, prec);
    L->macro = calloc(L->N * 14, prec);
    L->prof = (double*)calloc(L->N * 3, sizeof(double));
    L->cur = 0;
    return L;
}

void ref_destroy(void* h)
{
    Lattice* L = (Lattice*)h;
    if (!L) return;
    free(L->map); free(L->df[0]); free(L->df[1]); free(L->macro); free(L->prof);
    delete L;
}

int ref_set_map(void* h, const uint8_t* map)
{
    Lattice* L = (Lattice*)h;
    memcpy(L->map, map, L->N);
    L->left_area = L->right_area = 0;
    for (long c = 0; c < L->N; ++c) {
        L->left_area += map[c] == L_IN_L;
        L->right_area += map[c] == L_IN_R;
    }
    return 0;
}

void ref_set_inflow(void* h, double ivc, double svc, double rl, double rr, double re)
{
    Lattice* L = (Lattice*)h;
    L->ivc_flux = ivc; L->svc_flux = svc; L->rho_l = rl; L->rho_r = rr; L->rho_eq = re;
}

void ref_set_inflow_profile(void* h, const double* u3)
{
    Lattice* L = (Lattice*)h;
    memcpy(L->prof, u3, sizeof(double) * 3 * L->N);
}

int ref_init(void* h, double rho, double vx, double vy, double vz)
{
    Lattice* L = (Lattice*)h;
    double a[4] = {rho, vx, vy, vz};
    memset(L->macro, 0, L->N * 14 * L->prec);
    return run(L->prec, L->col, L->eq, 1, L, 0, a, nullptr);
}

int ref_step(void* h, int accumulate)
{
    Lattice* L = (Lattice*)h;
    return run(L->prec, L->col, L->eq, 0, L, accumulate, nullptr, nullptr);
}

void ref_get_df(void* h, double* out)
{
    Lattice* L = (Lattice*)h;
    for (long x = 0; x < L->X; ++x)
        for (int q = 0; q < 27; ++q)
            for (long z = 0; z < L->Z; ++z)
                for (long y = 0; y < L->Y; ++y) {
                    long s = y + L->Y * (z + L->Z * (q + 27 * x));
                    long d = (long)q * L->N + x + L->X * (y + L->Y * z);
                    out[d] = L->prec == 4 ? (double)((float*)L->df[L->cur])[s] : ((double*)L->df[L->cur])[s];
                }
}

void ref_get_macro(void* h, int field, double* out)
{
    Lattice* L = (Lattice*)h;
    for (long c = 0; c < L->N; ++c)
        out[c] = L->prec == 4 ? (double)((float*)L->macro)[field * L->N + c] : ((double*)L->macro)[field * L->N + c];
}

void ref_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int ref_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

} // extern "C"
