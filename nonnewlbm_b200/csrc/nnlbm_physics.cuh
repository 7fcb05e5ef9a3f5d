// nnlbm_physics.cuh -- per-cell D3Q27 physics for the sm_100a step kernels.
//
// Direction q = 9*(cx+1) + 3*(cy+1) + (cz+1) (the reference enum, solver/lbm3d/defs.h:215-247),
// opposite direction 26-q.  CT is the arithmetic type: float for F32/F16/BF16 storage and
// double for F64 storage.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <type_traits>

namespace nnlbm {

__host__ __device__ constexpr int cxq(int q) { return q / 9 - 1; }
__host__ __device__ constexpr int cyq(int q) { return (q / 3) % 3 - 1; }
__host__ __device__ constexpr int czq(int q) { return q % 3 - 1; }
__host__ __device__ constexpr int oppq(int q) { return 26 - q; }
__host__ __device__ constexpr int nnzq(int q) { return (cxq(q) != 0) + (cyq(q) != 0) + (czq(q) != 0); }

// lattice weights 8/27, 2/27, 1/54, 1/216 by the number of non-zero velocity components
template <class CT>
__host__ __device__ constexpr CT weight(int q)
{
    return nnzq(q) == 0 ? CT(8.0 / 27.0) : nnzq(q) == 1 ? CT(2.0 / 27.0) : nnzq(q) == 2 ? CT(1.0 / 54.0) : CT(1.0 / 216.0);
}

enum : int { EQ_INV_CUM_REF = 0, EQ_INV_CUM = 1, EQ_DEFAULT = 2, EQ_ENTROPIC = 3 };
enum : int { COL_CUM = 0, COL_KBC_N1 = 1, COL_KBC_N2, COL_KBC_N3, COL_KBC_N4, COL_KBC_C1, COL_KBC_C2,
             COL_KBC_C3, COL_KBC_C4, COL_MRT = 9, COL_BGK = 10 };

template <class CT> __device__ __forceinline__ CT dsqrt(CT v);
template <> __device__ __forceinline__ float dsqrt<float>(float v) { return sqrtf(v); }
template <> __device__ __forceinline__ double dsqrt<double>(double v) { return sqrt(v); }
template <class CT> __device__ __forceinline__ CT dpow(CT b, CT e);
template <> __device__ __forceinline__ float dpow<float>(float b, float e) { return powf(b, e); }
template <> __device__ __forceinline__ double dpow<double>(double b, double e) { return pow(b, e); }

// ---------------------------------------------------------------------------------------
// f2: one quantity of two cells at once on the packed FP32 pipe of sm_100 (FADD2, FMUL2,
// FFMA2), so that the step of two cells issues the arithmetic instructions of one.  Each
// half is rounded exactly as the scalar float operation; division is per half.
// ---------------------------------------------------------------------------------------
struct f2 {
    float2 v;
    __device__ __forceinline__ f2() {}
    __device__ __forceinline__ f2(float2 a) : v(a) {}
    __device__ __forceinline__ f2(float a, float b) : v(make_float2(a, b)) {}
    __device__ __forceinline__ explicit f2(double s) : v(make_float2((float)s, (float)s)) {}
};
__device__ __forceinline__ f2 operator+(f2 a, f2 b) { return __fadd2_rn(a.v, b.v); }
__device__ __forceinline__ f2 operator*(f2 a, f2 b) { return __fmul2_rn(a.v, b.v); }
__device__ __forceinline__ f2 operator-(f2 a, f2 b) { return __ffma2_rn(b.v, make_float2(-1.f, -1.f), a.v); }
__device__ __forceinline__ f2 operator-(f2 a) { return __fmul2_rn(a.v, make_float2(-1.f, -1.f)); }
__device__ __forceinline__ f2 operator/(f2 a, f2 b) { return f2(a.v.x / b.v.x, a.v.y / b.v.y); }
__device__ __forceinline__ f2& operator+=(f2& a, f2 b) { return a = a + b; }
__device__ __forceinline__ f2& operator-=(f2& a, f2 b) { return a = a - b; }
template <> __device__ __forceinline__ f2 dsqrt<f2>(f2 v) { return f2(sqrtf(v.v.x), sqrtf(v.v.y)); }

// a b + c: one rounding for f2 (FFMA2); for float the compiler contracts it under
// --use_fast_math; for double (built with -fmad=false) it is the product, then the sum,
// so an expression rewritten with mad keeps its FP64 rounding
template <class CT>
__device__ __forceinline__ CT mad(CT a, CT b, CT c) { return a * b + c; }
template <>
__device__ __forceinline__ f2 mad<f2>(f2 a, f2 b, f2 c) { return __ffma2_rn(a.v, b.v, c.v); }

// ---------------------------------------------------------------------------------------
// density and velocity with the F/2 shift, in the pairwise order of Geier 2015 Appendix J
// (the order of LBM_COMMON::computeDensityAndVelocity, solver/lbm3d/lbm_common.h:31-38)
// ---------------------------------------------------------------------------------------
template <class CT>
__device__ __forceinline__ void density_velocity(const CT* f, CT fx, CT fy, CT fz, CT& rho, CT& ux, CT& uy, CT& uz)
{
    enum { mmm = 0, mmz, mmp, mzm, mzz, mzp, mpm, mpz, mpp, zmm, zmz, zmp, zzm, zzz, zzp, zpm, zpz, zpp,
           pmm, pmz, pmp, pzm, pzz, pzp, ppm, ppz, ppp };
    rho = ((((f[ppp] + f[mmm]) + (f[pmp] + f[mpm])) + ((f[ppm] + f[mmp]) + (f[mpp] + f[pmm])))
           + (((f[zpp] + f[zmm]) + (f[zpm] + f[zmp])) + ((f[pzp] + f[mzm]) + (f[pzm] + f[mzp]))
              + ((f[ppz] + f[mmz]) + (f[pmz] + f[mpz])))
           + ((f[pzz] + f[mzz]) + (f[zpz] + f[zmz]) + (f[zzp] + f[zzm]))) + f[zzz];
    const CT ir = CT(1) / rho;
    uz = ((((f[ppp] - f[mmm]) + (f[mpp] - f[pmm])) + ((f[pmp] - f[mpm]) + (f[mmp] - f[ppm])))
          + (((f[zpp] - f[zmm]) + (f[zmp] - f[zpm])) + ((f[pzp] - f[mzm]) + (f[mzp] - f[pzm])))
          + (f[zzp] - f[zzm]) + fz * CT(0.5)) * ir;
    ux = ((((f[ppp] - f[mmm]) + (f[pmp] - f[mpm])) + ((f[ppm] - f[mmp]) + (f[pmm] - f[mpp])))
          + (((f[pzp] - f[mzm]) + (f[pzm] - f[mzp])) + ((f[ppz] - f[mmz]) + (f[pmz] - f[mpz])))
          + (f[pzz] - f[mzz]) + fx * CT(0.5)) * ir;
    uy = ((((f[ppp] - f[mmm]) + (f[ppm] - f[mmp])) + ((f[mpp] - f[pmm]) + (f[mpm] - f[pmp])))
          + (((f[ppz] - f[mmz]) + (f[mpz] - f[pmz])) + ((f[zpp] - f[zmm]) + (f[zpm] - f[zmp])))
          + (f[zpz] - f[zmz]) + fy * CT(0.5)) * ir;
}

template <class CT>
__device__ __forceinline__ CT density(const CT* f)
{
    CT r, a, b, c;
    density_velocity<CT>(f, CT(0), CT(0), CT(0), r, a, b, c);
    return r;
}

// ---------------------------------------------------------------------------------------
// equilibria for boundary nodes and initial states
// ---------------------------------------------------------------------------------------
template <class CT>
__device__ __forceinline__ CT inv_cum_factor(int c, CT v)
{
    return c == 0 ? CT(3) * v * v - CT(2) : (c > 0 ? CT(3) * v * v + CT(3) * v + CT(1) : CT(3) * v * v - CT(3) * v + CT(1));
}

// population q of the equilibrium of kind `eq` (q and eq may be runtime values; equilibrium()
// below evaluates the same expression for every q)
template <class CT>
__device__ __forceinline__ CT feq_one(int eq, int q, CT rho, CT ux, CT uy, CT uz)
{
    const int cx = cxq(q), cy = cyq(q), cz = czq(q);
    if (eq == EQ_DEFAULT) {
        // LBM_EQ_DEFAULT, lbm_eq.h:12-47
        const CT u2 = ux * ux + uy * uy + uz * uz;
        const CT cu = CT(cx) * ux + CT(cy) * uy + CT(cz) * uz;
        return weight<CT>(q) * rho * (CT(1) - CT(1.5) * u2 + CT(3) * cu + CT(4.5) * cu * cu);
    }
    if (eq == EQ_ENTROPIC) {
        // LBM_EQ_ENTROPIC, lbm_eq_entropic.h:12-38: per axis weight (2/3 or 1/6) times
        // (2 - sqrt(1+3v^2)) times B^c with B = (2v + sqrt(1+3v^2)) / (1 - v)
        const CT sx = dsqrt<CT>(CT(1) + CT(3) * ux * ux), sy = dsqrt<CT>(CT(1) + CT(3) * uy * uy);
        const CT sz = dsqrt<CT>(CT(1) + CT(3) * uz * uz);
        const CT bx = (CT(2) * ux + sx) / (CT(1) - ux), by = (CT(2) * uy + sy) / (CT(1) - uy), bz = (CT(2) * uz + sz) / (CT(1) - uz);
        const CT base = (CT(2) - sx) * (CT(2) - sy) * (CT(2) - sz);
        CT v = (cx ? CT(1.0 / 6.0) : CT(2.0 / 3.0)) * (cy ? CT(1.0 / 6.0) : CT(2.0 / 3.0)) * (cz ? CT(1.0 / 6.0) : CT(2.0 / 3.0)) * base;
        if (cx > 0) v *= bx; else if (cx < 0) v *= CT(1) / bx;
        if (cy > 0) v *= by; else if (cy < 0) v *= CT(1) / by;
        if (cz > 0) v *= bz; else if (cz < 0) v *= CT(1) / bz;
        return rho * v;
    }
    // factorised equilibrium of LBM_EQ_INV_CUM (lbm_eq_inv_cum.h:71-101): prefactor by the
    // number of zero components 3: -1/27, 2: 1/54, 1: -1/108, 0: 1/216
    const int nz0 = nnzq(q);
    const CT pre = nz0 == 0 ? CT(-1.0 / 27.0) : nz0 == 1 ? CT(1.0 / 54.0) : nz0 == 2 ? CT(-1.0 / 108.0) : CT(1.0 / 216.0);
    CT v = pre * rho * (inv_cum_factor<CT>(cx, ux) * inv_cum_factor<CT>(cy, uy) * inv_cum_factor<CT>(cz, uz));
    // the shipped feq_pmm multiplies by rho twice (lbm_eq_inv_cum.h:49)
    if (eq == EQ_INV_CUM_REF && q == 18) v *= rho;
    return v;
}

// feq of kind `eq` (runtime-uniform switch) into f[27]
template <class CT>
__device__ __forceinline__ void equilibrium(int eq, CT rho, CT ux, CT uy, CT uz, CT* f)
{
#pragma unroll
    for (int q = 0; q < 27; ++q) f[q] = feq_one<CT>(eq, q, rho, ux, uy, uz);
}

// ---------------------------------------------------------------------------------------
// cumulant collision (Geier et al. 2015) with the reference configuration of
// solver/lbm3d/lbm_col_cum.h:166-282: shear rate omega1 = 1/(3 nu + 1/2), every other rate
// 1, A = B = 0, no limiter.  With those rates all cumulants of order >= 3 are reset to
// zero, so only the central moments up to second order are needed from the forward
// transform; the backward transform rebuilds orders 4..6 from products of second order
// ones (G2015 Eq 81-84).
// ---------------------------------------------------------------------------------------
template <class CT>
__device__ __forceinline__ void fwd3(CT m, CT z, CT p, CT u, CT& k0, CT& k1, CT& k2)
{
    // k0 = (p+m)+z, k1 = (p-m) - u k0, k2 = (p+m) - 2u (p-m) + u^2 k0
    const CT s = p + m, d = p - m;
    k0 = s + z;
    k1 = mad(-u, k0, d);
    k2 = mad(u * u, k0, mad(-(CT(2) * u), d, s));
}

// the coefficients of one axis of the backward transform:
// z = k0 (1-u^2) - 2u k1 - k2, m = k0 (u^2-u)/2 + k1 (u - 1/2) + k2/2,
// p = k0 (u^2+u)/2 + k1 (u + 1/2) + k2/2
template <class CT>
struct Bwd {
    CT a, b, c, d, e, ntu;
    __device__ __forceinline__ explicit Bwd(CT u)
    {
        const CT uu = u * u;
        a = CT(1) - uu; b = CT(0.5) * (uu - u); c = u - CT(0.5); d = CT(0.5) * (uu + u); e = u + CT(0.5); ntu = CT(-2) * u;
    }
};

template <class CT>
__device__ __forceinline__ void bwd3(CT k0, CT k1, CT k2, const Bwd<CT>& w, CT& m, CT& z, CT& p)
{
    const CT h = CT(0.5) * k2;
    z = mad(k0, w.a, mad(w.ntu, k1, -k2));
    m = mad(k0, w.b, mad(k1, w.c, h));
    p = mad(k0, w.d, mad(k1, w.e, h));
}

template <class CT>
struct CYParams;
template <class CT>
__device__ __forceinline__ CT cy_nu_from_central(CT Cxx, CT Cyy, CT Czz, CT Cxy, CT Cxz, CT Cyz, CT rho, const CYParams<CT>& p,
                                                 CT* S);

// the first half of the forward z pass, which needs no velocity: per (x, y) column of
// populations (m, z, p) at f[9 ix + 3 iy + 0..2], its sum k0 = (p + m) + z, d = p - m and
// s = p + m, in place
template <class CT>
__device__ __forceinline__ void cum_columns(CT* f)
{
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        const CT m = f[3 * c], z = f[3 * c + 1], p = f[3 * c + 2];
        const CT sp = p + m, d = p - m;
        f[3 * c] = sp + z;
        f[3 * c + 1] = d;
        f[3 * c + 2] = sp;
    }
}

// density and velocity u = (j + F/2) / rho from the columns of cum_columns: rho sums the
// column sums, j_z their d, j_y and j_x the column sums' differences across y and x
template <class CT>
__device__ __forceinline__ void cum_density_velocity(const CT* k, CT fx, CT fy, CT fz, CT& rho, CT& ux, CT& uy, CT& uz)
{
    auto k0 = [&](int ix, int iy) { return k[9 * ix + 3 * iy]; };
    auto d = [&](int ix, int iy) { return k[9 * ix + 3 * iy + 1]; };
    const CT rx0 = (k0(0, 0) + k0(0, 2)) + k0(0, 1), rx1 = (k0(1, 0) + k0(1, 2)) + k0(1, 1), rx2 = (k0(2, 0) + k0(2, 2)) + k0(2, 1);
    rho = (rx0 + rx2) + rx1;
    const CT ir = CT(1) / rho;
    ux = ((rx2 - rx0) + fx * CT(0.5)) * ir;
    uy = (((k0(0, 2) - k0(0, 0)) + (k0(2, 2) - k0(2, 0))) + (k0(1, 2) - k0(1, 0)) + fy * CT(0.5)) * ir;
    uz = ((((d(0, 0) + d(0, 2)) + (d(2, 0) + d(2, 2))) + ((d(0, 1) + d(2, 1)) + (d(1, 0) + d(1, 2)))) + d(1, 1) + fz * CT(0.5)) * ir;
}

// the relaxation of the cumulant (lbm_col_cum.h:205-235 with omega2 = 1 and no anti-aliasing
// terms) from the central moments k of total order <= 2: s receives the post-collision
// cumulants as central moments (orders 3 and 5 zero).  `cy` non-null: the shear viscosity
// comes from the Carreau-Yasuda law on k's second moments, S receives the strain rate
template <class CT, class PT = CT>
__device__ __forceinline__ void cum_relax(const CT (&k)[3][3][3], CT rho, CT nu, const CYParams<PT>* cy, CT* S, CT (&s)[3][3][3])
{
    const CT ir = CT(1) / rho;
    if (cy) nu = cy_nu_from_central(k[2][0][0], k[0][2][0], k[0][0][2], k[1][1][0], k[1][0][1], k[0][1][1], rho, *cy, S);
    const CT om = CT(1) / (CT(3) * nu + CT(0.5));
    const CT k000 = k[0][0][0];
    // relaxation (lbm_col_cum.h:205-235 with omega2 = 1 and no anti-aliasing terms)
    const CT s110 = (CT(1) - om) * k[1][1][0];
    const CT s101 = (CT(1) - om) * k[1][0][1];
    const CT s011 = (CT(1) - om) * k[0][1][1];
    const CT e33 = (CT(1) - om) * (k[2][0][0] - k[0][2][0]);
    const CT e34 = (CT(1) - om) * (k[2][0][0] - k[0][0][2]);
    const CT s200 = CT(1.0 / 3.0) * (e33 + e34 + k000);
    const CT s020 = CT(1.0 / 3.0) * (CT(-2) * e33 + e34 + k000);
    const CT s002 = CT(1.0 / 3.0) * (e33 - CT(2) * e34 + k000);
    // fourth order from products (Eq 81-82); third and fifth order vanish
    const CT s211 = (s200 * s011 + CT(2) * s101 * s110) * ir;
    const CT s121 = (s020 * s101 + CT(2) * s110 * s011) * ir;
    const CT s112 = (s002 * s110 + CT(2) * s011 * s101) * ir;
    const CT s220 = (s020 * s200 + CT(2) * s110 * s110) * ir;
    const CT s022 = (s002 * s020 + CT(2) * s011 * s011) * ir;
    const CT s202 = (s200 * s002 + CT(2) * s101 * s101) * ir;
    // sixth order (Eq 84 with the odd orders at zero)
    const CT s222 = (s200 * s022 + s020 * s202 + s002 * s220 + CT(4) * (s011 * s211 + s101 * s121 + s110 * s112)) * ir
                    - (CT(16) * s110 * s101 * s011 + CT(4) * (s101 * s101 * s020 + s011 * s011 * s200 + s110 * s110 * s002)
                       + CT(2) * s200 * s020 * s002) * ir * ir;

#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int l = 0; l < 3; ++l) s[i][j][l] = CT(0);
    s[0][0][0] = k000;
    s[1][0][0] = -k[1][0][0]; s[0][1][0] = -k[0][1][0]; s[0][0][1] = -k[0][0][1];
    s[1][1][0] = s110; s[1][0][1] = s101; s[0][1][1] = s011;
    s[2][0][0] = s200; s[0][2][0] = s020; s[0][0][2] = s002;
    s[2][1][1] = s211; s[1][2][1] = s121; s[1][1][2] = s112;
    s[2][2][0] = s220; s[0][2][2] = s022; s[2][0][2] = s202;
    s[2][2][2] = s222;
}

// `cy` non-null: the shear viscosity comes from the Carreau-Yasuda law evaluated on this
// cell's own central second moments (k_200 ... k_011 of the forward transform); S receives
// the strain rate.  `f`: the columns of cum_columns; the post-collision populations replace
// them
template <class CT, class PT = CT>
__device__ __forceinline__ void collide_cum_columns(CT* f, CT rho, CT ux, CT uy, CT uz, CT nu, const CYParams<PT>* cy = nullptr,
                                                    CT* S = nullptr)
{
    // forward: the z pass's second half over the 9 (x,y) columns (fwd3 from k0, d, s)
    CT a[3][3][3];
    const CT uzz = uz * uz, m2uz = CT(-2) * uz;
#pragma unroll
    for (int ix = 0; ix < 3; ++ix)
#pragma unroll
        for (int iy = 0; iy < 3; ++iy) {
            const CT c0 = f[9 * ix + 3 * iy], d = f[9 * ix + 3 * iy + 1], sp = f[9 * ix + 3 * iy + 2];
            a[ix][iy][0] = c0;
            a[ix][iy][1] = mad(-uz, c0, d);
            a[ix][iy][2] = mad(uzz, c0, mad(m2uz, d, sp));
        }
    // y pass
    CT b[3][3][3];
#pragma unroll
    for (int ix = 0; ix < 3; ++ix)
#pragma unroll
        for (int kz = 0; kz < 3; ++kz)
            fwd3<CT>(a[ix][0][kz], a[ix][1][kz], a[ix][2][kz], uy, b[ix][0][kz], b[ix][1][kz], b[ix][2][kz]);
    // x pass, only the moments of total order <= 2 are used below
    CT k[3][3][3];
#pragma unroll
    for (int ky = 0; ky < 3; ++ky)
#pragma unroll
        for (int kz = 0; kz < 3; ++kz)
            if (ky + kz <= 2) fwd3<CT>(b[0][ky][kz], b[1][ky][kz], b[2][ky][kz], ux, k[0][ky][kz], k[1][ky][kz], k[2][ky][kz]);

    CT s[3][3][3];
    cum_relax<CT, PT>(k, rho, nu, cy, S, s);
    // backward: x, y, z (G2015 Eq 88-96), each axis's coefficients made just before its pass
    {
        const Bwd<CT> wx(ux);
#pragma unroll
        for (int ky = 0; ky < 3; ++ky)
#pragma unroll
            for (int kz = 0; kz < 3; ++kz)
                bwd3<CT>(s[0][ky][kz], s[1][ky][kz], s[2][ky][kz], wx, b[0][ky][kz], b[1][ky][kz], b[2][ky][kz]);
    }
    {
        const Bwd<CT> wy(uy);
#pragma unroll
        for (int ix = 0; ix < 3; ++ix)
#pragma unroll
            for (int kz = 0; kz < 3; ++kz)
                bwd3<CT>(b[ix][0][kz], b[ix][1][kz], b[ix][2][kz], wy, a[ix][0][kz], a[ix][1][kz], a[ix][2][kz]);
    }
    {
        const Bwd<CT> wz(uz);
#pragma unroll
        for (int ix = 0; ix < 3; ++ix)
#pragma unroll
            for (int iy = 0; iy < 3; ++iy)
                bwd3<CT>(a[ix][iy][0], a[ix][iy][1], a[ix][iy][2], wz, f[9 * ix + 3 * iy], f[9 * ix + 3 * iy + 1],
                         f[9 * ix + 3 * iy + 2]);
    }
}

// The cumulant step of one cell in single precision with the columns of x = -1 and x = 0
// packed into f2 (the packed FP32 pipe runs both at once): the z and y passes of both
// transforms treat the 18 populations of those two x planes as 9 pairs, the x passes (which
// combine the planes) and the relaxation run scalar.  The operations and their order are
// those of cum_columns / collide_cum_columns, so the results are bitwise the same.
#ifndef NNLBM_CUM_PACKED
#define NNLBM_CUM_PACKED 1
#endif
__device__ __forceinline__ void step_cell_cum_packed(float* f, float fx, float fy, float fz, float nu, const CYParams<float>* cy,
                                                     float* S, float& rho, float& ux, float& uy, float& uz)
{
    // z pass, first half: per column (iy) of the planes ix = 0, 1 (P) and ix = 2 (Q)
    f2 c0P[3], dP[3], spP[3];
    float c0Q[3], dQ[3], spQ[3];
#pragma unroll
    for (int iy = 0; iy < 3; ++iy) {
        const f2 m(f[3 * iy], f[9 + 3 * iy]), z(f[3 * iy + 1], f[9 + 3 * iy + 1]), p(f[3 * iy + 2], f[9 + 3 * iy + 2]);
        spP[iy] = p + m;
        dP[iy] = p - m;
        c0P[iy] = spP[iy] + z;
        const float mq = f[18 + 3 * iy], zq = f[18 + 3 * iy + 1], pq = f[18 + 3 * iy + 2];
        spQ[iy] = pq + mq;
        dQ[iy] = pq - mq;
        c0Q[iy] = spQ[iy] + zq;
    }
    {
        float k[27];
#pragma unroll
        for (int iy = 0; iy < 3; ++iy) {
            k[3 * iy] = c0P[iy].v.x; k[9 + 3 * iy] = c0P[iy].v.y; k[18 + 3 * iy] = c0Q[iy];
            k[3 * iy + 1] = dP[iy].v.x; k[9 + 3 * iy + 1] = dP[iy].v.y; k[18 + 3 * iy + 1] = dQ[iy];
        }
        cum_density_velocity<float>(k, fx, fy, fz, rho, ux, uy, uz);
    }
    // z pass, second half
    f2 aP[3][3];
    float aQ[3][3];
    {
        const f2 nuz(-uz), uzz(uz * uz), m2uz(-2.f * uz);
#pragma unroll
        for (int iy = 0; iy < 3; ++iy) {
            aP[iy][0] = c0P[iy];
            aP[iy][1] = mad(nuz, c0P[iy], dP[iy]);
            aP[iy][2] = mad(uzz, c0P[iy], mad(m2uz, dP[iy], spP[iy]));
            aQ[iy][0] = c0Q[iy];
            aQ[iy][1] = mad(-uz, c0Q[iy], dQ[iy]);
            aQ[iy][2] = mad(uz * uz, c0Q[iy], mad(-2.f * uz, dQ[iy], spQ[iy]));
        }
    }
    // y pass
    f2 bP[3][3];
    float bQ[3][3];
#pragma unroll
    for (int kz = 0; kz < 3; ++kz) {
        fwd3<f2>(aP[0][kz], aP[1][kz], aP[2][kz], f2(uy), bP[0][kz], bP[1][kz], bP[2][kz]);
        fwd3<float>(aQ[0][kz], aQ[1][kz], aQ[2][kz], uy, bQ[0][kz], bQ[1][kz], bQ[2][kz]);
    }
    // x pass (scalar), orders <= 2
    float k[3][3][3];
#pragma unroll
    for (int ky = 0; ky < 3; ++ky)
#pragma unroll
        for (int kz = 0; kz < 3; ++kz)
            if (ky + kz <= 2) fwd3<float>(bP[ky][kz].v.x, bP[ky][kz].v.y, bQ[ky][kz], ux, k[0][ky][kz], k[1][ky][kz], k[2][ky][kz]);
    float s[3][3][3];
    cum_relax<float, float>(k, rho, nu, cy, S, s);
    // backward x (scalar): the planes ix = 0, 1 of each (ky, kz) land as one pair
    {
        const Bwd<float> wx(ux);
#pragma unroll
        for (int ky = 0; ky < 3; ++ky)
#pragma unroll
            for (int kz = 0; kz < 3; ++kz) {
                float m, z, p;
                bwd3<float>(s[0][ky][kz], s[1][ky][kz], s[2][ky][kz], wx, m, z, p);
                bP[ky][kz] = f2(m, z);
                bQ[ky][kz] = p;
            }
    }
    // backward y
    {
        const Bwd<f2> wy2{f2(uy)};
        const Bwd<float> wy(uy);
#pragma unroll
        for (int kz = 0; kz < 3; ++kz) {
            bwd3<f2>(bP[0][kz], bP[1][kz], bP[2][kz], wy2, aP[0][kz], aP[1][kz], aP[2][kz]);
            bwd3<float>(bQ[0][kz], bQ[1][kz], bQ[2][kz], wy, aQ[0][kz], aQ[1][kz], aQ[2][kz]);
        }
    }
    // backward z, into the populations
    {
        const Bwd<f2> wz2{f2(uz)};
        const Bwd<float> wz(uz);
#pragma unroll
        for (int iy = 0; iy < 3; ++iy) {
            f2 m, z, p;
            bwd3<f2>(aP[iy][0], aP[iy][1], aP[iy][2], wz2, m, z, p);
            f[3 * iy] = m.v.x; f[9 + 3 * iy] = m.v.y;
            f[3 * iy + 1] = z.v.x; f[9 + 3 * iy + 1] = z.v.y;
            f[3 * iy + 2] = p.v.x; f[9 + 3 * iy + 2] = p.v.y;
            bwd3<float>(aQ[iy][0], aQ[iy][1], aQ[iy][2], wz, f[18 + 3 * iy], f[18 + 3 * iy + 1], f[18 + 3 * iy + 2]);
        }
    }
}

// the cumulant collision from populations f and a given density and velocity
template <class CT, class PT = CT>
__device__ __forceinline__ void collide_cum(CT* f, CT rho, CT ux, CT uy, CT uz, CT nu, const CYParams<PT>* cy = nullptr,
                                            CT* S = nullptr)
{
    cum_columns<CT>(f);
    collide_cum_columns<CT, PT>(f, rho, ux, uy, uz, nu, cy, S);
}

// ---------------------------------------------------------------------------------------
// factorised equilibrium of the BGK / KBC schemes (lbm_col_bgk.h:43-53, 85-111):
// feq_q = -rho X_cx Y_cy Z_cz with Xz = u^2 - 2/3, Xp = -(u^2 + u + 1/3)/2, Xm = Xp + u
// ---------------------------------------------------------------------------------------
template <class CT>
struct FactEq {
    CT X[3], Y[3], Z[3];
    __device__ __forceinline__ FactEq(CT ux, CT uy, CT uz)
    {
        X[1] = CT(1.0 / 3.0) - CT(1) + ux * ux; X[2] = CT(-0.5) * (X[1] + CT(1) + ux); X[0] = X[2] + ux;
        Y[1] = CT(1.0 / 3.0) - CT(1) + uy * uy; Y[2] = CT(-0.5) * (Y[1] + CT(1) + uy); Y[0] = Y[2] + uy;
        Z[1] = CT(1.0 / 3.0) - CT(1) + uz * uz; Z[2] = CT(-0.5) * (Z[1] + CT(1) + uz); Z[0] = Z[2] + uz;
    }
    __device__ __forceinline__ CT operator()(int q, CT rho) const { return -rho * X[q / 9] * Y[(q / 3) % 3] * Z[q % 3]; }
};

// forcing source S_q of lbm_col_bgk.h:57-83
template <class CT>
__device__ __forceinline__ CT force_src(int q, CT ir, CT ux, CT uy, CT uz, CT fx, CT fy, CT fz)
{
    return (CT(3) * ((CT(cxq(q)) - ux) * fx + (CT(cyq(q)) - uy) * fy + (CT(czq(q)) - uz) * fz)) * ir;
}

// BGK, solver/lbm3d/lbm_col_bgk.h:14-140
template <class CT>
__device__ __forceinline__ void collide_bgk(CT* f, CT rho, CT ux, CT uy, CT uz, CT fx, CT fy, CT fz, CT nu)
{
    const CT om = CT(1) / (CT(3) * nu + CT(0.5));
    const CT ir = CT(1) / rho;
    const FactEq<CT> E(ux, uy, uz);
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const CT feq = E(q, rho);
        f[q] += (feq - f[q]) * om + (CT(1) - CT(0.5) * om) * force_src<CT>(q, ir, ux, uy, uz, fx, fy, fz) * feq;
    }
}

// density and velocity of one cell in single precision from its column sums (the z pass's
// first half, cum_columns, with the columns of the planes x = -1, 0 as packed pairs), f
// unchanged
__device__ __forceinline__ void packed_density_velocity(const float* f, float fx, float fy, float fz, float& rho, float& ux,
                                                        float& uy, float& uz)
{
    float k[27];
#pragma unroll
    for (int iy = 0; iy < 3; ++iy) {
        const f2 m(f[3 * iy], f[9 + 3 * iy]), z(f[3 * iy + 1], f[9 + 3 * iy + 1]), p(f[3 * iy + 2], f[9 + 3 * iy + 2]);
        const f2 d = p - m, c0 = (p + m) + z;
        const float mq = f[18 + 3 * iy], zq = f[18 + 3 * iy + 1], pq = f[18 + 3 * iy + 2];
        k[3 * iy] = c0.v.x; k[9 + 3 * iy] = c0.v.y; k[18 + 3 * iy] = (pq + mq) + zq;
        k[3 * iy + 1] = d.v.x; k[9 + 3 * iy + 1] = d.v.y; k[18 + 3 * iy + 1] = pq - mq;
    }
    cum_density_velocity<float>(k, fx, fy, fz, rho, ux, uy, uz);
}

// BGK of one cell in single precision with the populations of the planes x = -1 and x = 0
// packed into f2 pairs (the same operations in the same order as collide_bgk; the x = +1
// plane runs scalar)
__device__ __forceinline__ void collide_bgk_packed(float* f, float rho, float ux, float uy, float uz, float fx, float fy,
                                                   float fz, float nu)
{
    const float om = 1.f / (3.f * nu + 0.5f);
    const float ir = 1.f / rho;
    const float k = 1.f - 0.5f * om;
    const FactEq<float> E(ux, uy, uz);
    const f2 rX(-rho * E.X[0], -rho * E.X[1]);
    const float rX2 = -rho * E.X[2];
    const f2 A((-1.f - ux) * fx, (0.f - ux) * fx);
    const float A2 = (1.f - ux) * fx;
    const f2 om2(om), k2(k), three(3.0), ir2(ir);
#pragma unroll
    for (int iy = 0; iy < 3; ++iy)
#pragma unroll
        for (int iz = 0; iz < 3; ++iz) {
            const int j = 3 * iy + iz;
            const float Y = E.Y[iy], Z = E.Z[iz];
            const float B = ((float)(iy - 1) - uy) * fy, C = ((float)(iz - 1) - uz) * fz;
            const f2 feq = (rX * f2(Y, Y)) * f2(Z, Z);
            const f2 src = (three * ((A + f2(B, B)) + f2(C, C))) * ir2;
            const f2 fv(f[j], f[9 + j]);
            const f2 nv = fv + mad(feq - fv, om2, (k2 * src) * feq);
            f[j] = nv.v.x;
            f[9 + j] = nv.v.y;
            const float feq1 = (rX2 * Y) * Z;
            const float src1 = (3.f * ((A2 + B) + C)) * ir;
            f[18 + j] += (feq1 - f[18 + j]) * om + (k * src1) * feq1;
        }
}

// MRT_LES, solver/lbm3d/lbm_col_mrt.h:12-78: second moments relaxed with a Smagorinsky rate,
// everything rebuilt as w_q [rho (1 + 3 c.u) + 9/2 (c c - I/3) : (P - rho I/3)] form
// the relaxed second moments of MRT_LES (P, and tr = trace P) from the populations
template <class CT>
__device__ __forceinline__ void mrt_moments(const CT* f, CT rho, CT ux, CT uy, CT uz, CT nu, CT& Pxx, CT& Pyy, CT& Pzz, CT& Pxy,
                                            CT& Pxz, CT& Pyz, CT& tr)
{
    Pxx = CT(0); Pyy = CT(0); Pzz = CT(0); Pxy = CT(0); Pxz = CT(0); Pyz = CT(0);
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const int cx = cxq(q), cy = cyq(q), cz = czq(q);
        if (cx) Pxx += f[q];
        if (cy) Pyy += f[q];
        if (cz) Pzz += f[q];
        if (cx * cy > 0) Pxy += f[q]; else if (cx * cy < 0) Pxy -= f[q];
        if (cx * cz > 0) Pxz += f[q]; else if (cx * cz < 0) Pxz -= f[q];
        if (cy * cz > 0) Pyz += f[q]; else if (cy * cz < 0) Pyz -= f[q];
    }
    const CT Pnxx = Pxx - rho * (CT(1.0 / 3.0) + ux * ux);
    const CT Pnyy = Pyy - rho * (CT(1.0 / 3.0) + uy * uy);
    const CT Pnzz = Pzz - rho * (CT(1.0 / 3.0) + uz * uz);
    const CT Pnxz = Pxz - rho * ux * uz;
    const CT Pnxy = Pxy - rho * ux * uy;
    const CT Pnyz = Pyz - rho * uy * uz;
    const CT Qs = CT(2) * (Pnxx * Pnxx + Pnyy * Pnyy + Pnzz * Pnzz + CT(2) * (Pnxy * Pnxy + Pnxz * Pnxz + Pnyz * Pnyz));
    const CT tau = CT(3) * nu + CT(0.5);
    const CT om = CT(2) / (dsqrt<CT>(tau * tau + CT(2) * CT(0.0342) * CT(9) * dsqrt<CT>(Qs) / rho) + tau);
    Pxx -= om * Pnxx; Pyy -= om * Pnyy; Pzz -= om * Pnzz;
    Pxy -= om * Pnxy; Pxz -= om * Pnxz; Pyz -= om * Pnyz;
    tr = Pxx + Pyy + Pzz;
}

template <class CT>
__device__ __forceinline__ void collide_mrt(CT* f, CT rho, CT ux, CT uy, CT uz, CT nu)
{
    CT Pxx, Pyy, Pzz, Pxy, Pxz, Pyz, tr;
    mrt_moments<CT>(f, rho, ux, uy, uz, nu, Pxx, Pyy, Pzz, Pxy, Pxz, Pyz, tr);
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const int cx = cxq(q), cy = cyq(q), cz = czq(q);
        const int c2 = cx * cx + cy * cy + cz * cz;
        const CT cu = CT(cx) * ux + CT(cy) * uy + CT(cz) * uz;
        const CT pp = CT(cx * cx) * Pxx + CT(cy * cy) * Pyy + CT(cz * cz) * Pzz
                      + CT(2) * (CT(cx * cy) * Pxy + CT(cx * cz) * Pxz + CT(cy * cz) * Pyz);
        f[q] = weight<CT>(q) * (rho * (CT(2.5) - CT(1.5) * CT(c2) + CT(3) * cu) + CT(4.5) * pp - CT(1.5) * tr);
    }
}

// MRT_LES of one cell in single precision, its rebuild with the planes x = -1 and x = 0 as
// packed f2 pairs (the terms without c_x are shared by the pair; the x = +1 plane runs
// scalar)
__device__ __forceinline__ void collide_mrt_packed(float* f, float rho, float ux, float uy, float uz, float nu)
{
    float Pxx, Pyy, Pzz, Pxy, Pxz, Pyz, tr;
    mrt_moments<float>(f, rho, ux, uy, uz, nu, Pxx, Pyy, Pzz, Pxy, Pxz, Pyz, tr);
    const f2 rho2(rho, rho), ux0(-ux, 0.f), three(3.0), p45(4.5), tr15(1.5f * tr, 1.5f * tr);
#pragma unroll
    for (int iy = 0; iy < 3; ++iy)
#pragma unroll
        for (int iz = 0; iz < 3; ++iz) {
            const int cy = iy - 1, cz = iz - 1, j = 3 * iy + iz;
            const float s_cu = (float)cy * uy + (float)cz * uz;
            const float s_pp = (float)(cy * cy) * Pyy + (float)(cz * cz) * Pzz + 2.f * (float)(cy * cz) * Pyz;
            const float x_pp = 2.f * ((float)cy * Pxy + (float)cz * Pxz);
            const int s_c2 = cy * cy + cz * cz;
            // x = -1 (c_x^2 = 1) and x = 0
            const f2 cu = ux0 + f2(s_cu, s_cu);
            const f2 pp = f2(Pxx - x_pp, 0.f) + f2(s_pp, s_pp);
            const f2 k(2.5f - 1.5f * (float)(1 + s_c2), 2.5f - 1.5f * (float)s_c2);
            const f2 w(weight<float>(j), weight<float>(9 + j));
            const f2 v = w * (mad(rho2, mad(three, cu, k), p45 * pp) - tr15);
            f[j] = v.v.x;
            f[9 + j] = v.v.y;
            // x = +1
            const float cu1 = ux + s_cu, pp1 = Pxx + x_pp + s_pp;
            f[18 + j] = weight<float>(18 + j) * (rho * (2.5f - 1.5f * (float)(1 + s_c2) + 3.f * cu1) + 4.5f * pp1 - 1.5f * tr);
        }
}

// ---------------------------------------------------------------------------------------
// KBC (Karlin, Boesch, Chikatamarla 2015), lbm_col_kbc_n.h / lbm_col_kbc_c.h: shear part
// s = D [+T] [+Q] of raw (N) or central (C) moments, entropic stabiliser gamma,
// f -= beta (2 ds + gamma dh) - (1-beta) S feq.  Two passes over q keep the per-direction
// temporaries out of registers.
// ---------------------------------------------------------------------------------------
template <class CT>
struct KbcMom { CT T, Nxz, Nyz, Pxy, Pxz, Pyz, Qxxy, Qxxz, Qxyy, Qyyz, Qxzz, Qyzz, Qxyz; };

template <class CT, bool USE_T, bool USE_Q>
__device__ __forceinline__ CT kbc_shear(int q, const KbcMom<CT>& m)
{
    const int cx = cxq(q), cy = cyq(q), cz = czq(q), nz0 = nnzq(q);
    CT D = CT(0), T = CT(0), Qv = CT(0);
    if (nz0 == 1) {
        if (cx) D = (CT(2) * m.Nxz - m.Nyz) * CT(1.0 / 6.0);
        if (cy) D = (-m.Nxz + CT(2) * m.Nyz) * CT(1.0 / 6.0);
        if (cz) D = (-m.Nxz - m.Nyz) * CT(1.0 / 6.0);
        T = m.T * CT(1.0 / 6.0);
        if (cx) Qv = CT(-cx) * (m.Qxyy + m.Qxzz) * CT(0.5);
        if (cy) Qv = CT(-cy) * (m.Qxxy + m.Qyzz) * CT(0.5);
        if (cz) Qv = CT(-cz) * (m.Qxxz + m.Qyyz) * CT(0.5);
    } else if (nz0 == 2) {
        if (!cz) { D = CT(cx * cy) * m.Pxy * CT(0.25); Qv = (CT(cx) * m.Qxyy + CT(cy) * m.Qxxy) * CT(0.25); }
        if (!cy) { D = CT(cx * cz) * m.Pxz * CT(0.25); Qv = (CT(cx) * m.Qxzz + CT(cz) * m.Qxxz) * CT(0.25); }
        if (!cx) { D = CT(cy * cz) * m.Pyz * CT(0.25); Qv = (CT(cy) * m.Qyzz + CT(cz) * m.Qyyz) * CT(0.25); }
    } else if (nz0 == 3) {
        Qv = CT(cx * cy * cz) * m.Qxyz * CT(0.125);
    } else {
        T = -m.T;
    }
    return D + (USE_T ? T : CT(0)) + (USE_Q ? Qv : CT(0));
}

// the entropic stabiliser gamma = 1/beta - (2 - 1/beta) num/den; the reference divides 0/0
// when dh vanishes identically, where gamma*dh is zero for any finite gamma and the
// regularised limit 1/beta is taken
template <class CT>
__device__ __forceinline__ CT kbc_gamma(CT num, CT den, CT beta)
{
    return den != CT(0) ? CT(1) / beta - (CT(2) - CT(1) / beta) * num / den : CT(1) / beta;
}
__device__ __forceinline__ f2 kbc_gamma(f2 num, f2 den, f2 beta)
{
    return f2(kbc_gamma<float>(num.v.x, den.v.x, beta.v.x), kbc_gamma<float>(num.v.y, den.v.y, beta.v.y));
}

template <class CT, bool CENTRAL, bool USE_T, bool USE_Q>
__device__ __forceinline__ void collide_kbc(CT* f, CT rho, CT ux, CT uy, CT uz, CT fx, CT fy, CT fz, CT nu)
{
    CT M200 = CT(0), M020 = CT(0), M002 = CT(0), M110 = CT(0), M101 = CT(0), M011 = CT(0), M111 = CT(0);
    CT M201 = CT(0), M102 = CT(0), M210 = CT(0), M120 = CT(0), M021 = CT(0), M012 = CT(0);
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const int cx = cxq(q), cy = cyq(q), cz = czq(q);
        const CT v = f[q];
        if (cx) { M200 += v; if (cz) M201 += CT(cz) * v; if (cy) M210 += CT(cy) * v; }
        if (cy) { M020 += v; if (cz) M021 += CT(cz) * v; if (cx) M120 += CT(cx) * v; }
        if (cz) { M002 += v; if (cx) M102 += CT(cx) * v; if (cy) M012 += CT(cy) * v; }
        if (cx && cy) M110 += CT(cx * cy) * v;
        if (cx && cz) M101 += CT(cx * cz) * v;
        if (cy && cz) M011 += CT(cy * cz) * v;
        if (cx && cy && cz) M111 += CT(cx * cy * cz) * v;
    }
    const CT cs2 = CT(1.0 / 3.0);
    KbcMom<CT> m, e;
    const CT rT = M200 + M020 + M002, rNxz = M200 - M002, rNyz = M020 - M002;
    if (!CENTRAL) {
        m = {rT, rNxz, rNyz, M110, M101, M011, M210, M201, M120, M021, M102, M012, M111};
        e.T = rho * (CT(3) * cs2 + ux * ux + uy * uy + uz * uz);
        e.Nxz = rho * (ux * ux - uz * uz); e.Nyz = rho * (uy * uy - uz * uz);
        e.Pxy = rho * ux * uy; e.Pxz = rho * ux * uz; e.Pyz = rho * uy * uz;
        e.Qxxy = rho * uy * (cs2 + ux * ux); e.Qxxz = rho * uz * (cs2 + ux * ux);
        e.Qxyy = rho * ux * (cs2 + uy * uy); e.Qyyz = rho * uz * (cs2 + uy * uy);
        e.Qxzz = rho * ux * (cs2 + uz * uz); e.Qyzz = rho * uy * (cs2 + uz * uz);
        e.Qxyz = rho * ux * uy * uz;
    } else {
        const CT cT = rT - rho * (ux * ux + uy * uy + uz * uz);
        const CT cNxz = rNxz + rho * (uz * uz - ux * ux), cNyz = rNyz + rho * (uz * uz - uy * uy);
        const CT cPxy = M110 - rho * ux * uy, cPxz = M101 - rho * ux * uz, cPyz = M011 - rho * uy * uz;
        m.T = cT; m.Nxz = cNxz; m.Nyz = cNyz; m.Pxy = cPxy; m.Pxz = cPxz; m.Pyz = cPyz;
        m.Qxxy = M210 - CT(1.0 / 3.0) * (CT(6) * ux * cPxy + uy * (CT(3) * ux * ux + CT(2) * cNxz - cNyz + cT));
        m.Qxxz = M201 - CT(1.0 / 3.0) * (CT(6) * ux * cPxz + uz * (CT(3) * ux * ux + CT(2) * cNxz - cNyz + cT));
        m.Qxyy = M120 - CT(1.0 / 3.0) * (CT(6) * uy * cPxy + ux * (CT(3) * uy * uy + CT(2) * cNyz - cNxz + cT));
        m.Qyyz = M021 - CT(1.0 / 3.0) * (CT(6) * uy * cPyz + uz * (CT(3) * uy * uy + CT(2) * cNyz - cNxz + cT));
        m.Qxzz = M102 - CT(1.0 / 3.0) * (CT(6) * uz * cPxz + ux * (CT(3) * uz * uz - cNyz - cNxz + cT));
        m.Qyzz = M012 - CT(1.0 / 3.0) * (CT(6) * uz * cPyz + uy * (CT(3) * uz * uz - cNyz - cNxz + cT));
        m.Qxyz = M111 - ux * cPyz - uy * cPxz - uz * cPxy - ux * uy * uz;
        const CT z = CT(0);
        e = {rho * CT(3) * cs2, z, z, z, z, z, z, z, z, z, z, z, z};
    }
    const FactEq<CT> E(ux, uy, uz);
    const CT beta = CT(1) / (CT(2) * nu / cs2 + CT(1));
    // the shear part is linear in the moments: Delta s_q = s_q(m) - s_q(m_eq) = s_q(m - m_eq)
    const KbcMom<CT> dm = {m.T - e.T, m.Nxz - e.Nxz, m.Nyz - e.Nyz, m.Pxy - e.Pxy, m.Pxz - e.Pxz, m.Pyz - e.Pyz,
                           m.Qxxy - e.Qxxy, m.Qxxz - e.Qxxz, m.Qxyy - e.Qxyy, m.Qyyz - e.Qyyz, m.Qxzz - e.Qxzz,
                           m.Qyzz - e.Qyzz, m.Qxyz - e.Qxyz};
    CT num = CT(0), den = CT(0);
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const CT feq = E(q, rho);
        const CT ds = kbc_shear<CT, USE_T, USE_Q>(q, dm);
        const CT dh = f[q] - feq - ds;
        const CT ifeq = CT(1) / feq;
        num += ds * dh * ifeq;
        den += dh * dh * ifeq;
    }
    const CT gamma = kbc_gamma(num, den, beta);
    const CT ir = CT(1) / rho;
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const CT feq = E(q, rho);
        const CT ds = kbc_shear<CT, USE_T, USE_Q>(q, dm);
        const CT dh = f[q] - feq - ds;
        f[q] -= beta * (CT(2) * ds + gamma * dh) - (CT(1) - beta) * force_src<CT>(q, ir, ux, uy, uz, fx, fy, fz) * feq;
    }
}

template <class CT, class PT>
__device__ __forceinline__ CT local_nu(const CT* f, CT rho, CT ux, CT uy, CT uz, const CYParams<PT>& p, CT* S);

// one collision; with `cy` the shear viscosity is the local Carreau-Yasuda one.  CT is
// the arithmetic type (f2: two cells at once), PT that of the viscosity-law parameters
template <class CT, int COL, class PT = CT>
__device__ __forceinline__ void collide(CT* f, CT rho, CT ux, CT uy, CT uz, CT fx, CT fy, CT fz, CT nu,
                                        const CYParams<PT>* cy = nullptr, CT* S = nullptr)
{
    if constexpr (COL != COL_CUM) {
        if (cy) nu = local_nu<CT, PT>(f, rho, ux, uy, uz, *cy, S);
    }
    if constexpr (COL == COL_CUM) collide_cum<CT, PT>(f, rho, ux, uy, uz, nu, cy, S);
    else if constexpr (COL == COL_MRT) collide_mrt<CT>(f, rho, ux, uy, uz, nu);
    else if constexpr (COL == COL_BGK) collide_bgk<CT>(f, rho, ux, uy, uz, fx, fy, fz, nu);
    else {
        constexpr bool central = COL >= COL_KBC_C1;
        constexpr int v = central ? COL - COL_KBC_C1 + 1 : COL - COL_KBC_N1 + 1;
        collide_kbc<CT, central, (v == 2 || v == 4), (v == 3 || v == 4)>(f, rho, ux, uy, uz, fx, fy, fz, nu);
    }
}

// density, velocity (u = (j + F/2) / rho) and the collision of one cell's populations.  For
// the cumulant the first half of the forward transform's z pass sums the populations by
// column, and the density and momentum come from those sums instead of separate sums over
// all 27
// PACK_DT: the storage type of a one-cell step in single precision (0: none), which picks the
// forms with the planes x = -1, 0 as packed pairs: the cumulant and BGK with every
// single-precision storage, MRT_LES with 16-bit storage (with FP32 storage, bound by HBM,
// the packed rebuild measured 1 % slower).  KBC keeps the scalar sums: at its 128 registers
// the packed ones spill and measured 5 % slower
template <class CT, int COL, class PT = CT, int PACK_DT = 0>
__device__ __forceinline__ void step_cell(CT* f, CT fx, CT fy, CT fz, CT nu, const CYParams<PT>* cy, CT* S, CT& rho, CT& ux,
                                          CT& uy, CT& uz)
{
    constexpr bool PACK = PACK_DT != 0 && std::is_same<CT, float>::value;
    if constexpr (COL == COL_CUM && PACK && NNLBM_CUM_PACKED) {
        step_cell_cum_packed(f, fx, fy, fz, nu, cy, S, rho, ux, uy, uz);
    } else if constexpr (COL == COL_MRT && PACK && PACK_DT >= 2) {
        packed_density_velocity(f, fx, fy, fz, rho, ux, uy, uz);
        if (cy) nu = local_nu<CT, PT>(f, rho, ux, uy, uz, *cy, S);
        collide_mrt_packed(f, rho, ux, uy, uz, nu);
    } else if constexpr (COL == COL_BGK && PACK) {
        packed_density_velocity(f, fx, fy, fz, rho, ux, uy, uz);
        if (cy) nu = local_nu<CT, PT>(f, rho, ux, uy, uz, *cy, S);
        collide_bgk_packed(f, rho, ux, uy, uz, fx, fy, fz, nu);
    } else if constexpr (COL == COL_CUM) {
        cum_columns<CT>(f);
        cum_density_velocity<CT>(f, fx, fy, fz, rho, ux, uy, uz);
        collide_cum_columns<CT, PT>(f, rho, ux, uy, uz, nu, cy, S);
    } else {
        density_velocity<CT>(f, fx, fy, fz, rho, ux, uy, uz);
        collide<CT, COL, PT>(f, rho, ux, uy, uz, fx, fy, fz, nu, cy, S);
    }
}

// ---------------------------------------------------------------------------------------
// Carreau-Yasuda local viscosity from the non-equilibrium second moments:
// Pi = sum f (c-u)(c-u) - rho/3 I, S = -3/(2 rho tau) Pi, gamma_dot = sqrt(2 S:S),
// nu = nu_inf + (nu0-nu_inf)(1 + (lambda gamma_dot)^a)^((n-1)/a), tau = 3 nu + 1/2, solved by
// three Newton steps on g(tau) = tau - 3 nu_CY(K/tau) - 1/2 from tau = 3 nu0 + 1/2.
// The viscosity law is the reference's (solver/lbm3d/core.h:763-766).
// ---------------------------------------------------------------------------------------
template <class CT>
struct CYParams { CT nu_inf, nu0, lam, a, n; };

// from the central second moments Cxx.. (not yet reduced by rho/3 on the diagonal)
template <class CT>
__device__ __forceinline__ CT cy_nu_from_central(CT Cxx, CT Cyy, CT Czz, CT Cxy, CT Cxz, CT Cyz, CT rho, const CYParams<CT>& p,
                                                 CT* S)
{
    const CT Pxx = Cxx - rho * CT(1.0 / 3.0), Pyy = Cyy - rho * CT(1.0 / 3.0), Pzz = Czz - rho * CT(1.0 / 3.0);
    const CT pn = dsqrt<CT>(Pxx * Pxx + Pyy * Pyy + Pzz * Pzz + CT(2) * (Cxy * Cxy + Cxz * Cxz + Cyz * Cyz));
    const CT K = CT(3) * CT(1.4142135623730951) * pn / (CT(2) * rho);
    CT tau = CT(3) * p.nu0 + CT(0.5);
    if (K > CT(0)) {
        const CT e = (p.n - CT(1)) / p.a;
#pragma unroll
        for (int it = 0; it < 3; ++it) {
            const CT g = K / tau;
            // (lambda gamma)^a; in single precision the usual a = 2 is a product
            CT s;
            if constexpr (sizeof(CT) == 4) s = p.a == CT(2) ? (p.lam * g) * (p.lam * g) : dpow<CT>(p.lam * g, p.a);
            else s = dpow<CT>(p.lam * g, p.a);
            const CT pw = dpow<CT>(CT(1) + s, e);
            const CT nuc = p.nu_inf + (p.nu0 - p.nu_inf) * pw;
            const CT G = tau - CT(3) * nuc - CT(0.5);
            const CT gdn = (p.nu0 - p.nu_inf) * (p.n - CT(1)) * s * pw / (CT(1) + s);
            const CT Gp = CT(1) + CT(3) * gdn / tau;
            tau = tau - G / Gp;
        }
    }
    const CT sc = CT(-3) / (CT(2) * rho * tau);
    S[0] = sc * Pxx; S[1] = sc * Cxy; S[2] = sc * Cxz; S[3] = sc * Pyy; S[4] = sc * Cyz; S[5] = sc * Pzz;
    return (tau - CT(0.5)) * CT(1.0 / 3.0);
}

// two cells at once: the same Newton solve in packed arithmetic; the powers, square roots
// and divisions run per half, and a half whose strain is zero keeps tau = 3 nu0 + 1/2
__device__ __forceinline__ f2 cy_nu_from_central(f2 Cxx, f2 Cyy, f2 Czz, f2 Cxy, f2 Cxz, f2 Cyz, f2 rho,
                                                 const CYParams<float>& p, f2* S)
{
    const f2 third(1.0 / 3.0), half(0.5), three(3.0), one(1.0);
    const f2 Pxx = Cxx - rho * third, Pyy = Cyy - rho * third, Pzz = Czz - rho * third;
    const f2 pn = dsqrt<f2>(Pxx * Pxx + Pyy * Pyy + Pzz * Pzz + f2(2.0) * (Cxy * Cxy + Cxz * Cxz + Cyz * Cyz));
    const f2 K = three * f2(1.4142135623730951) * pn / (f2(2.0) * rho);
    const f2 tau0 = three * f2(p.nu0) + half;
    f2 tau = tau0;
    const bool ka = K.v.x > 0.f, kb = K.v.y > 0.f;
    if (ka || kb) {
        const float e = (p.n - 1.f) / p.a;
        const f2 dn(p.nu0 - p.nu_inf), ninf(p.nu_inf), lam(p.lam), nm1(p.n - 1.f);
#pragma unroll
        for (int it = 0; it < 3; ++it) {
            const f2 g = K / tau;
            const f2 lg = lam * g;
            // (lambda gamma)^a; the usual a = 2 is a product
            const f2 s = p.a == 2.f ? lg * lg : f2(dpow<float>(lg.v.x, p.a), dpow<float>(lg.v.y, p.a));
            const f2 s1 = one + s;
            const f2 pw(dpow<float>(s1.v.x, e), dpow<float>(s1.v.y, e));
            const f2 nuc = ninf + dn * pw;
            const f2 G = tau - three * nuc - half;
            const f2 gdn = dn * nm1 * s * pw / s1;
            const f2 Gp = one + three * gdn / tau;
            tau = tau - G / Gp;
        }
        tau = f2(ka ? tau.v.x : tau0.v.x, kb ? tau.v.y : tau0.v.y);
    }
    const f2 sc = f2(-3.0) / (f2(2.0) * rho * tau);
    S[0] = sc * Pxx; S[1] = sc * Cxy; S[2] = sc * Cxz; S[3] = sc * Pyy; S[4] = sc * Cyz; S[5] = sc * Pzz;
    return (tau - half) * third;
}

// the same from the populations: raw second moments by additions only (c in {-1,0,1}),
// shifted to central ones with the raw momentum j: C_ab = M_ab - u_a j_b - u_b j_a + rho u_a u_b
template <class CT, class PT>
__device__ __forceinline__ CT local_nu(const CT* f, CT rho, CT ux, CT uy, CT uz, const CYParams<PT>& p, CT* S)
{
    CT Mxx = CT(0), Myy = CT(0), Mzz = CT(0), Mxy = CT(0), Mxz = CT(0), Myz = CT(0), jx = CT(0), jy = CT(0), jz = CT(0);
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const int cx = cxq(q), cy = cyq(q), cz = czq(q);
        const CT v = f[q];
        if (cx) { Mxx += v; if (cx > 0) jx += v; else jx -= v; }
        if (cy) { Myy += v; if (cy > 0) jy += v; else jy -= v; }
        if (cz) { Mzz += v; if (cz > 0) jz += v; else jz -= v; }
        if (cx * cy > 0) Mxy += v; else if (cx * cy < 0) Mxy -= v;
        if (cx * cz > 0) Mxz += v; else if (cx * cz < 0) Mxz -= v;
        if (cy * cz > 0) Myz += v; else if (cy * cz < 0) Myz -= v;
    }
    const CT Cxx = Mxx - CT(2) * ux * jx + rho * ux * ux;
    const CT Cyy = Myy - CT(2) * uy * jy + rho * uy * uy;
    const CT Czz = Mzz - CT(2) * uz * jz + rho * uz * uz;
    const CT Cxy = Mxy - ux * jy - uy * jx + rho * ux * uy;
    const CT Cxz = Mxz - ux * jz - uz * jx + rho * ux * uz;
    const CT Cyz = Myz - uy * jz - uz * jy + rho * uy * uz;
    return cy_nu_from_central(Cxx, Cyy, Czz, Cxy, Cxz, Cyz, rho, p, S);
}

} // namespace nnlbm
