// ref_shim.cpp -- the reference's own per-cell kernels of solver/lbm3d/core.h (buresjan/nonnewlbm),
// compiled unmodified on the host into oracle/_ref/libnnlbm_ref.so (FP64 parity build) and
// oracle/_ref/libnnlbm_ref_fast.so (timing build).
//
// TEST INFRASTRUCTURE ONLY: it pins the C oracle (known-answer vectors under tests/golden/),
// is compared with the GPU step directly by the GPU tests, and its single-precision build is
// the timed CPU baseline of bench.py.  Nothing in the product links it.
//
// core.h is included as it ships.  Its own #include "defs.h" / "state.h" / "lbm.h" land on
// the stand-ins of oracle/ref_stub/ (oracle/Makefile searches that directory first, with
// -I-), which declare the interface types those headers take from TNL-bound code.  Every
// per-cell operation therefore runs the reference's code: LBMKernel (core.h:578-800) with its
// finite-difference Carreau-Yasuda force, the multi-rank pre-kernels LBMKernelVelocity
// (core.h:273-384) and LBMKernelStress (core.h:387-576), LBMKernelInit (core.h:833-863), the
// streaming, collision and equilibrium templates, the generic boundary blocks of lbm_bc.h and
// MacroDefault of lbm_macro.h.  Written here are only what sim_tcpc.cu and TNL would supply:
//   ShimData  the LBM_DATA policy over plain arrays (index map y + Y*(z + Z*(q + 27*x)) of
//             solver/lbm3d/lbm_data.h:61-71) with LBM_Data_Tcpc's inflow rules
//             (sim_tcpc.cu:281-320) and the per-cell inflow of LBM_Data_ConstInflow
//             (lbm_data.h:352-367);
//   ShimBC    the LBM_BC policy: the predicates and BC switch of LBM_BC_Tcpc
//             (sim_tcpc.cu:187-279), which lives in sim_tcpc.cu next to its main() and VTK
//             reader and cannot be included, extended by the generic GEO_INFLOW and
//             GEO_OUTFLOW_RIGHT_EQ blocks, which it takes from LBM_BC_All (lbm_bc.h:126-152);
//   the loops: the host loop of core.h:1312-1320 (x, z, y order, collapse(2)) around each
//             kernel, and for the finite-difference Carreau-Yasuda mode the three phases of
//             the multi-rank step (core.h:1169-1310) on one rank, with the pointer swap of
//             lbm.hpp:392-418 after each step.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "core.h"

namespace {

// solver map labels of this repository: 0..6 are LBM_BC_Tcpc::GEO (sim_tcpc.cu:194-203); 7 and 8
// stand for LBM_BC_All's GEO_INFLOW and GEO_OUTFLOW_RIGHT_EQ
enum { L_FLUID = 0, L_WALL = 1, L_PERIODIC = 2, L_IN_L = 3, L_IN_R = 4, L_OUT_F = 5, L_OUT_B = 6, L_IN_EQ = 7, L_OUT_REQ = 8 };
enum { CY_NONE = 0, CY_REF_FD = 1 };

template <typename T>
using ShimTraits = Traits<T, double, long, short>;

// LBM_DATA policy over plain host arrays
template <typename T>
struct ShimData {
    T* dfs[DFMAX];
    T* mac;                 // [MacroDefault::N][N], x fastest
    const uint8_t* lab;     // [N] labels, x fastest
    const double* prof;     // [3][N] prescribed velocity of L_IN_EQ cells
    long X_, Y_, Z_, N_;
    T lbmViscosity = 1, fx = 0, fy = 0, fz = 0;
    T lbm_nu0 = 0, lbm_lambda = 0, lbm_a = 1, lbm_n = 1;
    T inflow_rho_left = 1, inflow_rho_right = 1, inflow_rho_eq = 1;
    T inflow_left = 0, inflow_right = 0;
    long inflow_left_area = 0, inflow_right_area = 0;

    long X() const { return X_; }
    long Y() const { return Y_; }
    long Z() const { return Z_; }
    long cell(long x, long y, long z) const { return x + X_ * (y + Y_ * z); }
    T& df(uint8_t type, int q, long x, long y, long z) { return dfs[type][y + Y_ * (z + Z_ * (q + 27 * x))]; }
    short map(long x, long y, long z) const { return (short)lab[cell(x, y, z)]; }
    T& macro(int id, long x, long y, long z) { return mac[(long)id * N_ + cell(x, y, z)]; }

    // LBM_Data_Tcpc::inflowCondition{Left,Right} (sim_tcpc.cu:295-309)
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
    // LBM_Data_Tcpc::inflow (sim_tcpc.cu:311-319) for the two TCPC planes; the prescribed
    // per-cell velocity (LBM_Data_ConstInflow) for GEO_INFLOW cells
    void inflow(KernelStruct<T>& KS, long x, long y, long z)
    {
        const int l = map(x, y, z);
        if (l == L_IN_R) { inflowConditionRight(KS, x, y, z); return; }
        if (l == L_IN_L) { inflowConditionLeft(KS, x, y, z); return; }
        const long c = cell(x, y, z);
        KS.rho = inflow_rho_eq;
        KS.vx = (T)prof[c];
        KS.vy = (T)prof[N_ + c];
        KS.vz = (T)prof[2 * N_ + c];
    }
};

// LBM_BC policy: LBM_BC_Tcpc's predicates and switch plus the two generic blocks
template <typename TRAITS>
struct ShimBC {
    using dreal = typename TRAITS::dreal;
    using idx = typename TRAITS::idx;
    using map_t = typename TRAITS::map_t;
    using G = LBM_BC_All<TRAITS>;

    static bool isPeriodic(map_t m) { return m == L_PERIODIC; }
    static bool isFluid(map_t m) { return m == L_FLUID; }
    static bool isNotFluid(map_t m) { return m != L_FLUID; }
    static bool isWall(map_t m) { return m == L_WALL; }
    static bool isInflow(map_t m) { return m == L_IN_L || m == L_IN_R || m == L_IN_EQ; }
    static bool isOutflowR(map_t m) { return m == L_OUT_F || m == L_OUT_B || m == L_OUT_REQ; }
    static bool isStreaming(map_t m) { return m == L_FLUID || m == L_PERIODIC; }
    static bool isComputeDensityAndVelocity(map_t m) { return m == L_FLUID || m == L_PERIODIC; }

    template <typename L, typename S, typename LBM_DATA>
    static bool BC(LBM_DATA& SD, KernelStruct<dreal>& KS, idx m, idx xm, idx x, idx xp, idx ym, idx y, idx yp, idx zm,
                   idx z, idx zp)
    {
        switch (m) {
        case L_WALL: // sim_tcpc.cu:235-241
            S::streamingBounceBack(SD, KS, xm, x, xp, ym, y, yp, zm, z, zp);
            KS.rho = no1;
            KS.vx = KS.vy = KS.vz = (dreal)0;
            return true;
        case L_IN_L:
        case L_IN_R: { // sim_tcpc.cu:242-261: rho of the post-streaming state one cell inward
            if (m == L_IN_L) SD.inflowConditionLeft(KS, x, y, z);
            else SD.inflowConditionRight(KS, x, y, z);
            KernelStruct<dreal> inward;
            if (m == L_IN_L) S::streaming(SD, inward, x, xp, xp + 1, ym, y, yp, zm, z, zp);
            else S::streaming(SD, inward, xm - 1, xm, x, ym, y, yp, zm, z, zp);
            L::computeDensityAndVelocity(inward);
            KS.rho = inward.rho;
            L::setEquilibrium(KS);
            return true;
        }
        case L_OUT_F:
        case L_OUT_B: // sim_tcpc.cu:262-273: velocity one cell inward, rho = 1
            if (m == L_OUT_F) S::streaming(SD, KS, xm, x, xp, y, yp, yp + 1, zm, z, zp);
            else S::streaming(SD, KS, xm, x, xp, ym - 1, ym, y, zm, z, zp);
            L::computeDensityAndVelocity(KS);
            KS.rho = no1;
            L::setEquilibrium(KS);
            return true;
        case L_IN_EQ:
            return G::template BC<L, S, LBM_DATA>(SD, KS, G::GEO_INFLOW, xm, x, xp, ym, y, yp, zm, z, zp);
        case L_OUT_REQ:
            return G::template BC<L, S, LBM_DATA>(SD, KS, G::GEO_OUTFLOW_RIGHT_EQ, xm, x, xp, ym, y, yp, zm, z, zp);
        default:
            return false;
        }
    }
};

// LBMKernelInit's view of the lattice (core.h:839-863): the map, the host populations and
// the kernel data
template <typename T>
struct ShimHostDF {
    const T* a;
    long Y, Z;
    T operator()(int q, long x, long y, long z) const { return a[y + Y * (z + Z * (q + 27 * x))]; }
};
template <typename T>
struct ShimLBM {
    ShimData<T> data;
    ShimHostDF<T> hfs[DFMAX];
    short map(long x, long y, long z) const { return data.map(x, y, z); }
};

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

using MacroF = MacroDefault<ShimTraits<float>>;
// macro fields in the C oracle's numbering (oracle/nnlbm_oracle.h), as MacroDefault ids
const int kMacroOf[20] = {MacroF::e_rho, MacroF::e_vx, MacroF::e_vy, MacroF::e_vz,
                          MacroF::e_vm_plus_x, MacroF::e_vm_minus_x, MacroF::e_vm_y, MacroF::e_vm_z,
                          MacroF::e_vm_xx, MacroF::e_vm_yy, MacroF::e_vm_zz,
                          MacroF::e_fx, MacroF::e_fy, MacroF::e_fz,
                          MacroF::e_S11, MacroF::e_S12, MacroF::e_S13, MacroF::e_S22, MacroF::e_S32, MacroF::e_S33};
// the mean/rms sums, which MacroDefault::outputMacro adds to on every call
const int kStatFields[7] = {MacroF::e_vm_plus_x, MacroF::e_vm_minus_x, MacroF::e_vm_y, MacroF::e_vm_z,
                            MacroF::e_vm_xx, MacroF::e_vm_yy, MacroF::e_vm_zz};

struct Lattice {
    int prec; // 8 or 4
    int col, eq, cy_mode = CY_NONE;
    long X, Y, Z, N;
    double nu, fx, fy, fz;
    double nu0 = 0, lam = 0, a = 1, n = 1;
    uint8_t* map;
    void* df[2];
    int cur;
    double* prof;
    void* macro; // [MacroDefault::N][N]
    double ivc_flux = 0, svc_flux = 0, rho_l = 1, rho_r = 1, rho_eq = 1;
    long left_area = 0, right_area = 0;
};

template <typename T>
ShimData<T> make_data(Lattice& L)
{
    ShimData<T> SD;
    SD.dfs[df_cur] = (T*)L.df[L.cur];
    SD.dfs[df_out] = (T*)L.df[1 - L.cur];
    SD.mac = (T*)L.macro;
    SD.lab = L.map;
    SD.prof = L.prof;
    SD.X_ = L.X; SD.Y_ = L.Y; SD.Z_ = L.Z; SD.N_ = L.N;
    SD.lbmViscosity = (T)L.nu;
    SD.fx = (T)L.fx; SD.fy = (T)L.fy; SD.fz = (T)L.fz;
    if (L.cy_mode == CY_REF_FD) {
        SD.lbm_nu0 = (T)L.nu0; SD.lbm_lambda = (T)L.lam; SD.lbm_a = (T)L.a; SD.lbm_n = (T)L.n;
    } else {
        // a Newtonian law: with the zero strain of the single-rank step the force term of
        // core.h:779-781 is exactly zero, as in the deployed sim_tcpc
        SD.lbm_nu0 = (T)L.nu; SD.lbm_lambda = 0; SD.lbm_a = 1; SD.lbm_n = 1;
    }
    // sim_tcpc.cu:657-663: inflow_right = -svc_flux
    SD.inflow_left = (T)L.ivc_flux;
    SD.inflow_right = (T)(-L.svc_flux);
    SD.inflow_rho_left = (T)L.rho_l;
    SD.inflow_rho_right = (T)L.rho_r;
    SD.inflow_rho_eq = (T)L.rho_eq;
    SD.inflow_left_area = L.left_area;
    SD.inflow_right_area = L.right_area;
    return SD;
}

// the host loop of core.h:1312-1320 around one kernel
template <typename F>
void for_cells(const Lattice& L, F&& body)
{
#pragma omp parallel for schedule(static) collapse(2)
    for (long x = 0; x < L.X; x++)
        for (long z = 0; z < L.Z; z++)
            for (long y = 0; y < L.Y; y++) body(x, y, z);
}

template <typename T, typename LT>
void lattice_step(Lattice& L, int acc)
{
    using TR = ShimTraits<T>;
    using S = LBM_STREAMING<TR>;
    using M = MacroDefault<TR>;
    using D = ShimData<T>;
    using BC = ShimBC<TR>;
    const D SD = make_data<T>(L);
    T* mac = (T*)L.macro;
    std::vector<T> keep;
    if (!acc) keep.assign(mac + (long)kStatFields[0] * L.N, mac + (long)(kStatFields[6] + 1) * L.N);
    if (L.cy_mode == CY_REF_FD) {
        // core.h:1169-1258 on one rank: the velocity of the post-streaming state, then the
        // finite-difference strain, then the step with the force of that strain
        for_cells(L, [&](long x, long y, long z) { LBMKernelVelocity<LT, S, M, D, BC>(SD, x, y, z, 0, 1); });
        for_cells(L, [&](long x, long y, long z) { LBMKernelStress<LT, S, M, D, BC>(SD, x, y, z, 0, 1); });
    }
    for_cells(L, [&](long x, long y, long z) { LBMKernel<LT, S, M, D, BC>(SD, x, y, z, 0, 1); });
    if (!acc) std::copy(keep.begin(), keep.end(), mac + (long)kStatFields[0] * L.N);
    L.cur = 1 - L.cur; // lbm.hpp:392-418
}

template <typename T, typename LT>
void lattice_init(Lattice& L, double rho, double vx, double vy, double vz)
{
    // resetLattice / setEqLat (sim_tcpc.cu:647-655, lbm.hpp:1-39): both lattices at feq
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
    // the initial macro fields (LBMKernelInit over every cell, core.h:1531-1536); its call of
    // outputMacro also adds the initial state to the mean/rms sums, which start at zero here
    using TR = ShimTraits<T>;
    using M = MacroDefault<TR>;
    using BC = ShimBC<TR>;
    memset(L.macro, 0, (size_t)L.N * M::N * L.prec);
    ShimLBM<T> lbm;
    lbm.data = make_data<T>(L);
    lbm.hfs[df_cur] = {(const T*)L.df[L.cur], L.Y, L.Z};
    lbm.hfs[df_out] = {(const T*)L.df[1 - L.cur], L.Y, L.Z};
    for_cells(L, [&](long x, long y, long z) { LBMKernelInit<LT, BC, M, ShimLBM<T>>(lbm, x, y, z); });
    for (int f : kStatFields) memset((T*)L.macro + (long)f * L.N, 0, (size_t)L.N * sizeof(T));
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
    if (nx < 3 || ny < 3 || nz < 3 || (prec != 4 && prec != 8) || col < 0 || col > 10 || (eq != 0 && eq != 2 && eq != 3))
        return nullptr;
    Lattice* L = new Lattice();
    L->prec = prec; L->col = col; L->eq = eq;
    L->X = nx; L->Y = ny; L->Z = nz; L->N = (long)nx * ny * nz;
    L->nu = nu; L->fx = fx; L->fy = fy; L->fz = fz;
    L->map = (uint8_t*)calloc(L->N, 1);
    L->df[0] = calloc(L->N * 27, prec);
    L->df[1] = calloc(L->N * 27, prec);
    L->macro = calloc(L->N * MacroF::N, prec);
    L->prof = (double*)calloc(L->N * 3, sizeof(double));
    L->cur = 0;
    return L;
}

// Carreau-Yasuda coupling: 0 = none (the deployed single-rank step), 1 = the
// finite-difference force of the multi-rank step; lattice-unit nu0, lambda, a, n
int ref_set_cy(void* h, int mode, double nu0, double lam, double a, double n)
{
    Lattice* L = (Lattice*)h;
    if (mode != CY_NONE && mode != CY_REF_FD) return -1;
    if (mode == CY_REF_FD && !(a > 0)) return -1;
    L->cy_mode = mode; L->nu0 = nu0; L->lam = lam; L->a = a; L->n = n;
    return 0;
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

// one macro field, numbered as in the C oracle (oracle/nnlbm_oracle.h: rho vx vy vz, the
// seven mean/rms sums, fx fy fz, S11 S12 S13 S22 S32 S33)
int ref_get_macro(void* h, int field, double* out)
{
    Lattice* L = (Lattice*)h;
    if (field < 0 || field >= 20) return -1;
    const long off = (long)kMacroOf[field] * L->N;
    for (long c = 0; c < L->N; ++c)
        out[c] = L->prec == 4 ? (double)((float*)L->macro)[off + c] : ((double*)L->macro)[off + c];
    return 0;
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
