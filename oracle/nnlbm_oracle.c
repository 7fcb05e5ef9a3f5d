/*
 * nnlbm_oracle.c -- FP64 CPU oracle (test infrastructure only; see nnlbm_oracle.h).
 *
 * A plain-C restatement of the reference step.  Compiled with -ffp-contract=off so that
 * every product and sum is rounded as written.  Paths cited are relative to the
 * buresjan/nonnewlbm project root.
 */
#include "nnlbm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NQ 27

/* direction enum of solver/lbm3d/defs.h:215-247 */
enum {
    mmm = 0, mmz, mmp, mzm, mzz, mzp, mpm, mpz, mpp,
    zmm, zmz, zmp, zzm, zzz, zzp, zpm, zpz, zpp,
    pmm, pmz, pmp, pzm, pzz, pzp, ppm, ppz, ppp
};

static inline int CXq(int q) { return q / 9 - 1; }
static inline int CYq(int q) { return (q / 3) % 3 - 1; }
static inline int CZq(int q) { return q % 3 - 1; }
static inline int OPP(int q) { return 26 - q; }

struct orc_lattice {
    orc_desc d;
    int64_t N;
    uint8_t* map;
    double* df[2];   /* AoS: df[c*27 + q] */
    int cur;         /* index of the array holding the latest post-collision state */
    double* macro;   /* [ORC_M_N][N] */
    double* prof;    /* [3][N] */
    double ivc_flux, svc_flux, rho_left, rho_right, rho_eq;
    int64_t left_area, right_area;
    int64_t iterations;
};

static inline int64_t cidx(const orc_lattice* L, int x, int y, int z)
{
    return (int64_t)x + (int64_t)L->d.nx * ((int64_t)y + (int64_t)L->d.ny * z);
}

void orc_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------------------------ */
/* equilibria                                                                             */
/* ------------------------------------------------------------------------------------ */

/* LBM_EQ_DEFAULT, solver/lbm3d/lbm_eq.h:12-47 */
static double eq_default_1(int qx, int qy, int qz, double vx, double vy, double vz)
{
    double cu = qx * vx + qy * vy + qz * vz;
    return 1.0 - 1.5 * (vx * vx + vy * vy + vz * vz) + 3.0 * cu + 4.5 * cu * cu;
}

/* one-dimensional factors of the factorised equilibrium, solver/lbm3d/lbm_eq_inv_cum.h:71-101:
 * c=0 -> (3v^2-2), c=+1 -> (3v^2+3v+1), c=-1 -> (3v^2-3v+1) */
static inline double inv_cum_factor(int c, double v)
{
    if (c == 0) return 3.0 * v * v - 2.0;
    if (c > 0) return 3.0 * v * v + 3.0 * v + 1.0;
    return 3.0 * v * v - 3.0 * v + 1.0;
}

/* entropic 1-D pieces, solver/lbm3d/lbm_eq_entropic.h:12-38 */
static inline double ent_base(double v) { return 2.0 - sqrt(1.0 + 3.0 * v * v); }
static inline double ent_ratio(double v) { return (2.0 * v + sqrt(1.0 + 3.0 * v * v)) / (1.0 - v); }

void orc_feq(int eq, double rho, double vx, double vy, double vz, double f[27])
{
    for (int q = 0; q < NQ; ++q) {
        int cx = CXq(q), cy = CYq(q), cz = CZq(q);
        int nz0 = (cx != 0) + (cy != 0) + (cz != 0);
        if (eq == ORC_EQ_DEFAULT) {
            static const double w[4] = {8.0 / 27.0, 2.0 / 27.0, 1.0 / 54.0, 1.0 / 216.0};
            f[q] = w[nz0] * rho * eq_default_1(cx, cy, cz, vx, vy, vz);
        } else if (eq == ORC_EQ_ENTROPIC) {
            /* weights 2/3 (c=0) and 1/6 (c=+-1) per axis, times prod(2-sqrt(1+3v^2)),
             * times B^c with B=(2v+sqrt(1+3v^2))/(1-v) */
            double wx = cx == 0 ? 2.0 / 3.0 : 1.0 / 6.0;
            double wy = cy == 0 ? 2.0 / 3.0 : 1.0 / 6.0;
            double wz = cz == 0 ? 2.0 / 3.0 : 1.0 / 6.0;
            double v = wx * wy * wz * ent_base(vx) * ent_base(vy) * ent_base(vz);
            if (cx > 0) v = v * ent_ratio(vx); else if (cx < 0) v = v * (1.0 / ent_ratio(vx));
            if (cy > 0) v = v * ent_ratio(vy); else if (cy < 0) v = v * (1.0 / ent_ratio(vy));
            if (cz > 0) v = v * ent_ratio(vz); else if (cz < 0) v = v * (1.0 / ent_ratio(vz));
            f[q] = rho * v;
        } else {
            /* factorised ("inverse cumulant") equilibrium: sign/weight by number of
             * zero components: 3 -> -1/27, 2 -> 1/54, 1 -> -1/108, 0 -> 1/216 */
            static const double wc[4] = {-1.0 / 27.0, 1.0 / 54.0, -1.0 / 108.0, 1.0 / 216.0};
            double v = wc[nz0] * rho *
                       (inv_cum_factor(cx, vx) * inv_cum_factor(cy, vy) * inv_cum_factor(cz, vz));
            /* lbm_eq_inv_cum.h:49 multiplies feq_pmm by rho a second time */
            if (eq == ORC_EQ_INV_CUM_REF && q == pmm) v = v * rho;
            f[q] = v;
        }
    }
}

/* ------------------------------------------------------------------------------------ */
/* density and velocity: LBM_COMMON::computeDensityAndVelocity, lbm_common.h:16-39       */
/* (Geier 2015 Appendix J pairwise order, velocity shifted by F/2)                        */
/* ------------------------------------------------------------------------------------ */
void orc_density_velocity(const double* f, double fx, double fy, double fz, double out[4])
{
    double rho = ((((f[ppp] + f[mmm]) + (f[pmp] + f[mpm])) + ((f[ppm] + f[mmp]) + (f[mpp] + f[pmm])))
                  + (((f[zpp] + f[zmm]) + (f[zpm] + f[zmp])) + ((f[pzp] + f[mzm]) + (f[pzm] + f[mzp]))
                     + ((f[ppz] + f[mmz]) + (f[pmz] + f[mpz])))
                  + ((f[pzz] + f[mzz]) + (f[zpz] + f[zmz]) + (f[zzp] + f[zzm]))) + f[zzz];
    double vz = ((((f[ppp] - f[mmm]) + (f[mpp] - f[pmm])) + ((f[pmp] - f[mpm]) + (f[mmp] - f[ppm])))
                 + (((f[zpp] - f[zmm]) + (f[zmp] - f[zpm])) + ((f[pzp] - f[mzm]) + (f[mzp] - f[pzm])))
                 + (f[zzp] - f[zzm]) + fz * 0.5) / rho;
    double vx = ((((f[ppp] - f[mmm]) + (f[pmp] - f[mpm])) + ((f[ppm] - f[mmp]) + (f[pmm] - f[mpp])))
                 + (((f[pzp] - f[mzm]) + (f[pzm] - f[mzp])) + ((f[ppz] - f[mmz]) + (f[pmz] - f[mpz])))
                 + (f[pzz] - f[mzz]) + fx * 0.5) / rho;
    double vy = ((((f[ppp] - f[mmm]) + (f[ppm] - f[mmp])) + ((f[mpp] - f[pmm]) + (f[mpm] - f[pmp])))
                 + (((f[ppz] - f[mmz]) + (f[mpz] - f[pmz])) + ((f[zpp] - f[zmm]) + (f[zpm] - f[zmp])))
                 + (f[zpz] - f[zmz]) + fy * 0.5) / rho;
    out[0] = rho; out[1] = vx; out[2] = vy; out[3] = vz;
}

/* ------------------------------------------------------------------------------------ */
/* cumulant collision, solver/lbm3d/lbm_col_cum.h:12-455 (Geier et al. 2015), with the     */
/* reference's defaults: omega2..omega10 = 1, A = B = 0, no limiter, no anti-aliasing.     */
/* ------------------------------------------------------------------------------------ */
static void chimera_fwd(double m, double z, double p, double u, double out[3])
{
    /* Eq 6-8 (lbm_col_cum.h:50-80) */
    double k0 = (p + m) + z;
    out[0] = k0;
    out[1] = (p - m) - u * k0;
    out[2] = (p + m) - 2.0 * u * (p - m) + u * u * k0;
}

static void chimera_bwd(double k0, double k1, double k2, double u, double out[3])
{
    /* Eq 88-90 (lbm_col_cum.h:319-349): out = {m, z, p} */
    out[1] = k0 * (1.0 - u * u) - 2.0 * u * k1 - k2;
    out[0] = (k0 * (u * u - u) + k1 * (2.0 * u - 1.0) + k2) * 0.5;
    out[2] = (k0 * (u * u + u) + k1 * (2.0 * u + 1.0) + k2) * 0.5;
}

static void col_cum(double* f, double rho, double vx, double vy, double vz, double nu)
{
    double a[3][3][3], b[3][3][3], k[3][3][3], o[3];
    /* z pass: a[ix][iy][kz] */
    for (int ix = 0; ix < 3; ++ix)
        for (int iy = 0; iy < 3; ++iy) {
            chimera_fwd(f[9 * ix + 3 * iy + 0], f[9 * ix + 3 * iy + 1], f[9 * ix + 3 * iy + 2], vz, o);
            for (int t = 0; t < 3; ++t) a[ix][iy][t] = o[t];
        }
    /* y pass (Eq 9-11): b[ix][ky][kz] */
    for (int ix = 0; ix < 3; ++ix)
        for (int kz = 0; kz < 3; ++kz) {
            chimera_fwd(a[ix][0][kz], a[ix][1][kz], a[ix][2][kz], vy, o);
            for (int t = 0; t < 3; ++t) b[ix][t][kz] = o[t];
        }
    /* x pass (Eq 12-14): k[kx][ky][kz] */
    for (int ky = 0; ky < 3; ++ky)
        for (int kz = 0; kz < 3; ++kz) {
            chimera_fwd(b[0][ky][kz], b[1][ky][kz], b[2][ky][kz], vx, o);
            for (int t = 0; t < 3; ++t) k[t][ky][kz] = o[t];
        }
#define K(i, j, l) k[i][j][l]
    const double k_000 = K(0, 0, 0), k_100 = K(1, 0, 0), k_010 = K(0, 1, 0), k_001 = K(0, 0, 1);
    const double k_110 = K(1, 1, 0), k_101 = K(1, 0, 1), k_011 = K(0, 1, 1), k_111 = K(1, 1, 1);
    const double k_200 = K(2, 0, 0), k_020 = K(0, 2, 0), k_002 = K(0, 0, 2);
    const double k_210 = K(2, 1, 0), k_201 = K(2, 0, 1), k_120 = K(1, 2, 0), k_021 = K(0, 2, 1);
    const double k_102 = K(1, 0, 2), k_012 = K(0, 1, 2);
    const double k_211 = K(2, 1, 1), k_121 = K(1, 2, 1), k_112 = K(1, 1, 2);
    const double k_220 = K(2, 2, 0), k_202 = K(2, 0, 2), k_022 = K(0, 2, 2);
    const double k_122 = K(1, 2, 2), k_212 = K(2, 1, 2), k_221 = K(2, 2, 1), k_222 = K(2, 2, 2);
#undef K
    /* cumulants, G2015 Eq 51-54 (lbm_col_cum.h:148-163); orders 2 and 3 equal the central
     * moments (lbm_col_cum.h:15-29) */
    const double C_110 = k_110, C_101 = k_101, C_011 = k_011, C_111 = k_111;
    const double C_200 = k_200, C_020 = k_020, C_002 = k_002;
    const double C_210 = k_210, C_201 = k_201, C_120 = k_120, C_021 = k_021, C_102 = k_102, C_012 = k_012;
    const double C_211 = k_211 - (k_200 * k_011 + 2.0 * k_101 * k_110) / rho;
    const double C_121 = k_121 - (k_020 * k_101 + 2.0 * k_110 * k_011) / rho;
    const double C_112 = k_112 - (k_002 * k_110 + 2.0 * k_011 * k_101) / rho;
    const double C_220 = k_220 - (k_020 * k_200 + 2.0 * k_110 * k_110) / rho;
    const double C_022 = k_022 - (k_002 * k_020 + 2.0 * k_011 * k_011) / rho;
    const double C_202 = k_202 - (k_200 * k_002 + 2.0 * k_101 * k_101) / rho;
    const double C_122 = k_122 - (k_020 * k_102 + k_002 * k_120 + 4.0 * k_011 * k_111 + 2.0 * (k_110 * k_012 + k_101 * k_021)) / rho;
    const double C_212 = k_212 - (k_002 * k_210 + k_200 * k_012 + 4.0 * k_101 * k_111 + 2.0 * (k_011 * k_201 + k_110 * k_102)) / rho;
    const double C_221 = k_221 - (k_200 * k_021 + k_020 * k_201 + 4.0 * k_110 * k_111 + 2.0 * (k_101 * k_120 + k_011 * k_210)) / rho;
    const double C_222 = k_222 - (4.0 * k_111 * k_111 + k_200 * k_022 + k_020 * k_202 + k_002 * k_220
                                  + 4.0 * (k_011 * k_211 + k_101 * k_121 + k_110 * k_112)
                                  + 2.0 * (k_120 * k_102 + k_210 * k_012 + k_201 * k_021)) / rho
                         + (16.0 * k_110 * k_101 * k_011 + 4.0 * (k_101 * k_101 * k_020 + k_011 * k_011 * k_200 + k_110 * k_110 * k_002)
                            + 2.0 * k_200 * k_020 * k_002) / rho / rho;
    (void)C_111; (void)C_211; (void)C_121; (void)C_112; (void)C_220; (void)C_022; (void)C_202;
    (void)C_122; (void)C_212; (void)C_221; (void)C_222;

    /* relaxation, lbm_col_cum.h:166-282 (non-2017 branch) */
    const double omega1 = 1.0 / (3.0 * nu + 0.5);
    const double omega2 = 1.0, omega3 = 1.0, omega4 = 1.0;
    const double Cs_110 = (1.0 - omega1) * C_110;
    const double Cs_101 = (1.0 - omega1) * C_101;
    const double Cs_011 = (1.0 - omega1) * C_011;
    const double Eq33RHS = (1.0 - omega1) * (C_200 - C_020);
    const double Eq34RHS = (1.0 - omega1) * (C_200 - C_002);
    const double Eq35RHS = k_000 * omega2 + (1.0 - omega2) * (C_200 + C_020 + C_002);
    const double Cs_200 = (1.0 / 3.0) * (Eq33RHS + Eq34RHS + Eq35RHS);
    const double Cs_020 = (1.0 / 3.0) * (-2.0 * Eq33RHS + Eq34RHS + Eq35RHS);
    const double Cs_002 = (1.0 / 3.0) * (Eq33RHS - 2.0 * Eq34RHS + Eq35RHS);
    const double Cs_120 = (-C_102 - C_120) * omega3 * 0.5 + (C_102 - C_120) * omega4 * 0.5 + C_120;
    const double Cs_102 = (-C_102 - C_120) * omega3 * 0.5 + (-C_102 + C_120) * omega4 * 0.5 + C_102;
    const double Cs_210 = (-C_012 - C_210) * omega3 * 0.5 + (C_012 - C_210) * omega4 * 0.5 + C_210;
    const double Cs_012 = (-C_012 - C_210) * omega3 * 0.5 + (-C_012 + C_210) * omega4 * 0.5 + C_012;
    const double Cs_021 = (-C_021 - C_201) * omega3 * 0.5 + (-C_021 + C_201) * omega4 * 0.5 + C_021;
    const double Cs_201 = (-C_021 - C_201) * omega3 * 0.5 + (C_021 - C_201) * omega4 * 0.5 + C_201;
    const double Cs_111 = 0.0; /* (1-omega5)*C_111 with omega5 = 1 */
    /* orders 4..6 relax to zero: omega6..omega10 = 1 and A = B = 0 */
    const double Cs_220 = 0.0, Cs_202 = 0.0, Cs_022 = 0.0;
    const double Cs_211 = 0.0, Cs_121 = 0.0, Cs_112 = 0.0;
    const double Cs_221 = 0.0, Cs_212 = 0.0, Cs_122 = 0.0, Cs_222 = 0.0;

    /* backward cumulant transformation, G2015 Eq 81-84 (lbm_col_cum.h:289-307) */
    const double ks_110 = Cs_110, ks_101 = Cs_101, ks_011 = Cs_011, ks_111 = Cs_111;
    const double ks_200 = Cs_200, ks_020 = Cs_020, ks_002 = Cs_002;
    const double ks_120 = Cs_120, ks_102 = Cs_102, ks_210 = Cs_210, ks_012 = Cs_012, ks_021 = Cs_021, ks_201 = Cs_201;
    const double ks_211 = Cs_211 + (ks_200 * ks_011 + 2.0 * ks_101 * ks_110) / rho;
    const double ks_121 = Cs_121 + (ks_020 * ks_101 + 2.0 * ks_110 * ks_011) / rho;
    const double ks_112 = Cs_112 + (ks_002 * ks_110 + 2.0 * ks_011 * ks_101) / rho;
    const double ks_220 = Cs_220 + (ks_020 * ks_200 + 2.0 * ks_110 * ks_110) / rho;
    const double ks_022 = Cs_022 + (ks_002 * ks_020 + 2.0 * ks_011 * ks_011) / rho;
    const double ks_202 = Cs_202 + (ks_200 * ks_002 + 2.0 * ks_101 * ks_101) / rho;
    const double ks_122 = Cs_122 + (ks_020 * ks_102 + ks_002 * ks_120 + 4.0 * ks_011 * ks_111 + 2.0 * (ks_110 * ks_012 + ks_101 * ks_021)) / rho;
    const double ks_212 = Cs_212 + (ks_002 * ks_210 + ks_200 * ks_012 + 4.0 * ks_101 * ks_111 + 2.0 * (ks_011 * ks_201 + ks_110 * ks_102)) / rho;
    const double ks_221 = Cs_221 + (ks_200 * ks_021 + ks_020 * ks_201 + 4.0 * ks_110 * ks_111 + 2.0 * (ks_101 * ks_120 + ks_011 * ks_210)) / rho;
    const double ks_222 = Cs_222 + (4.0 * ks_111 * ks_111 + ks_200 * ks_022 + ks_020 * ks_202 + ks_002 * ks_220
                                    + 4.0 * (ks_011 * ks_211 + ks_101 * ks_121 + ks_110 * ks_112)
                                    + 2.0 * (ks_120 * ks_102 + ks_210 * ks_012 + ks_201 * ks_021)) / rho
                          - (16.0 * ks_110 * ks_101 * ks_011 + 4.0 * (ks_101 * ks_101 * ks_020 + ks_011 * ks_011 * ks_200 + ks_110 * ks_110 * ks_002)
                             + 2.0 * ks_200 * ks_020 * ks_002) / rho / rho;
    /* first order flips sign (forcing), lbm_col_cum.h:311-315 */
    double s[3][3][3];
    s[0][0][0] = k_000; s[1][0][0] = -k_100; s[0][1][0] = -k_010; s[0][0][1] = -k_001;
    s[1][1][0] = ks_110; s[1][0][1] = ks_101; s[0][1][1] = ks_011; s[1][1][1] = ks_111;
    s[2][0][0] = ks_200; s[0][2][0] = ks_020; s[0][0][2] = ks_002;
    s[1][2][0] = ks_120; s[1][0][2] = ks_102; s[2][1][0] = ks_210; s[0][1][2] = ks_012;
    s[0][2][1] = ks_021; s[2][0][1] = ks_201;
    s[2][1][1] = ks_211; s[1][2][1] = ks_121; s[1][1][2] = ks_112;
    s[2][2][0] = ks_220; s[0][2][2] = ks_022; s[2][0][2] = ks_202;
    s[1][2][2] = ks_122; s[2][1][2] = ks_212; s[2][2][1] = ks_221; s[2][2][2] = ks_222;

    /* backward central moment transformation x, y, z (Eq 88-96, lbm_col_cum.h:319-415) */
    for (int ky = 0; ky < 3; ++ky)
        for (int kz = 0; kz < 3; ++kz) {
            chimera_bwd(s[0][ky][kz], s[1][ky][kz], s[2][ky][kz], vx, o);
            for (int ix = 0; ix < 3; ++ix) b[ix][ky][kz] = o[ix];
        }
    for (int ix = 0; ix < 3; ++ix)
        for (int kz = 0; kz < 3; ++kz) {
            chimera_bwd(b[ix][0][kz], b[ix][1][kz], b[ix][2][kz], vy, o);
            for (int iy = 0; iy < 3; ++iy) a[ix][iy][kz] = o[iy];
        }
    for (int ix = 0; ix < 3; ++ix)
        for (int iy = 0; iy < 3; ++iy) {
            chimera_bwd(a[ix][iy][0], a[ix][iy][1], a[ix][iy][2], vz, o);
            for (int iz = 0; iz < 3; ++iz) f[9 * ix + 3 * iy + iz] = o[iz];
        }
}

/* ------------------------------------------------------------------------------------ */
/* MRT_LES, solver/lbm3d/lbm_col_mrt.h:12-78: regularised rebuild with Smagorinsky omega  */
/* ------------------------------------------------------------------------------------ */
static void col_mrt(double* f, double rho, double vx, double vy, double vz, double nu)
{
    double Pxx = 0, Pyy = 0, Pzz = 0, Pxy = 0, Pxz = 0, Pyz = 0;
    for (int q = 0; q < NQ; ++q) {
        int cx = CXq(q), cy = CYq(q), cz = CZq(q);
        Pxx += cx * cx * f[q]; Pyy += cy * cy * f[q]; Pzz += cz * cz * f[q];
        Pxy += cx * cy * f[q]; Pxz += cx * cz * f[q]; Pyz += cy * cz * f[q];
    }
    const double Pnxx = Pxx - rho * (1.0 / 3.0 + vx * vx);
    const double Pnyy = Pyy - rho * (1.0 / 3.0 + vy * vy);
    const double Pnzz = Pzz - rho * (1.0 / 3.0 + vz * vz);
    const double Pnxz = Pxz - rho * vx * vz;
    const double Pnxy = Pxy - rho * vx * vy;
    const double Pnyz = Pyz - rho * vy * vz;
    const double Qs = 2.0 * (Pnxx * Pnxx + Pnyy * Pnyy + Pnzz * Pnzz + 2.0 * (Pnxy * Pnxy + Pnxz * Pnxz + Pnyz * Pnyz));
    const double tau = 3.0 * nu + 0.5;
    const double C = 0.0342;
    const double omega = 2.0 / (sqrt(tau * tau + 2.0 * C * 3.0 * 3.0 * sqrt(Qs) / rho) + tau);
    Pxx -= omega * Pnxx; Pyy -= omega * Pnyy; Pzz -= omega * Pnzz;
    Pxy -= omega * Pnxy; Pxz -= omega * Pnxz; Pyz -= omega * Pnyz;
    const double tr = Pxx + Pyy + Pzz;
    for (int q = 0; q < NQ; ++q) {
        int cx = CXq(q), cy = CYq(q), cz = CZq(q);
        int c2 = cx * cx + cy * cy + cz * cz;
        static const double w[4] = {8.0 / 27.0, 2.0 / 27.0, 1.0 / 54.0, 1.0 / 216.0};
        f[q] = w[c2] * (rho * (2.5 - 1.5 * c2 + 3.0 * (vx * cx + vy * cy + vz * cz))
                        + 4.5 * (Pxx * (cx * cx) + Pyy * (cy * cy) + Pzz * (cz * cz)
                                 + 2.0 * (Pxy * (cx * cy) + Pxz * (cx * cz) + Pyz * (cy * cz)))
                        - 1.5 * tr);
    }
}

/* forcing source of the factorised BGK/KBC schemes, lbm_col_bgk.h:57-83 */
static inline double force_src(int cx, int cy, int cz, double rho, double vx, double vy, double vz,
                               double fx, double fy, double fz)
{
    return (3.0 * ((cx - vx) * fx + (cy - vy) * fy + (cz - vz) * fz)) / rho;
}

/* factorised equilibrium factors X/Y/Z of lbm_col_bgk.h:43-53 and lbm_col_kbc_n.h:329-339 */
static void fact_eq(double rho, double vx, double vy, double vz, double feq[27])
{
    double X[3], Y[3], Z[3];
    double Xz = 1.0 / 3.0 - 1.0 + vx * vx, Xp = -0.5 * (Xz + 1.0 + vx), Xm = Xp + vx;
    double Yz = 1.0 / 3.0 - 1.0 + vy * vy, Yp = -0.5 * (Yz + 1.0 + vy), Ym = Yp + vy;
    double Zz = 1.0 / 3.0 - 1.0 + vz * vz, Zp = -0.5 * (Zz + 1.0 + vz), Zm = Zp + vz;
    X[0] = Xm; X[1] = Xz; X[2] = Xp; Y[0] = Ym; Y[1] = Yz; Y[2] = Yp; Z[0] = Zm; Z[1] = Zz; Z[2] = Zp;
    for (int q = 0; q < NQ; ++q) feq[q] = -rho * X[q / 9] * Y[(q / 3) % 3] * Z[q % 3];
}

/* BGK (Geier 2017 factorised), solver/lbm3d/lbm_col_bgk.h:14-140 */
static void col_bgk(double* f, double rho, double vx, double vy, double vz, double fx, double fy,
                    double fz, double nu)
{
    const double omega1 = 1.0 / (3.0 * nu + 0.5);
    double feq[27];
    fact_eq(rho, vx, vy, vz, feq);
    for (int q = 0; q < NQ; ++q) {
        double S = force_src(CXq(q), CYq(q), CZq(q), rho, vx, vy, vz, fx, fy, fz);
        f[q] += (feq[q] - f[q]) * omega1 + (1.0 - 0.5 * omega1) * S * feq[q];
    }
}

/* ------------------------------------------------------------------------------------ */
/* KBC N1..N4 / C1..C4, solver/lbm3d/lbm_col_kbc_n.h:21-289,296-1260 and                 */
/* lbm_col_kbc_c.h:21-318,324-1290.  Shear part s = D [+T] [+Q] of raw (N) or central (C)  */
/* moments; f -= beta(2 ds + gamma dh) - (1-beta) S feq.                                   */
/* ------------------------------------------------------------------------------------ */
typedef struct { double T, Nxz, Nyz, Pxy, Pxz, Pyz, Qxxy, Qxxz, Qxyy, Qyyz, Qxzz, Qyzz, Qxyz; } kbc_mom;

static double kbc_shear_dir(int q, const kbc_mom* m, int useT, int useQ)
{
    int cx = CXq(q), cy = CYq(q), cz = CZq(q);
    int nz0 = (cx != 0) + (cy != 0) + (cz != 0);
    double D = 0, T = 0, Qv = 0;
    if (nz0 == 1) {
        if (cx) D = (2.0 * m->Nxz - m->Nyz) / 6.0;
        if (cy) D = (-m->Nxz + 2.0 * m->Nyz) / 6.0;
        if (cz) D = (-m->Nxz - m->Nyz) / 6.0;
        T = m->T / 6.0;
        if (cx) Qv = -cx * (m->Qxyy + m->Qxzz) / 2.0;
        if (cy) Qv = -cy * (m->Qxxy + m->Qyzz) / 2.0;
        if (cz) Qv = -cz * (m->Qxxz + m->Qyyz) / 2.0;
    } else if (nz0 == 2) {
        if (!cz) { D = cx * cy * m->Pxy / 4.0; Qv = (cx * m->Qxyy + cy * m->Qxxy) / 4.0; }
        if (!cy) { D = cx * cz * m->Pxz / 4.0; Qv = (cx * m->Qxzz + cz * m->Qxxz) / 4.0; }
        if (!cx) { D = cy * cz * m->Pyz / 4.0; Qv = (cy * m->Qyzz + cz * m->Qyyz) / 4.0; }
    } else if (nz0 == 3) {
        Qv = cx * cy * cz * m->Qxyz / 8.0;
    } else {
        T = -m->T;
    }
    return D + (useT ? T : 0.0) + (useQ ? Qv : 0.0);
}

static void col_kbc(double* f, double rho, double vx, double vy, double vz, double fx, double fy,
                    double fz, double nu, int central, int useT, int useQ)
{
    double ffeq[27];
    fact_eq(rho, vx, vy, vz, ffeq);
    double M200 = 0, M020 = 0, M002 = 0, M110 = 0, M101 = 0, M011 = 0, M111 = 0;
    double M201 = 0, M102 = 0, M210 = 0, M120 = 0, M021 = 0, M012 = 0;
    for (int q = 0; q < NQ; ++q) {
        int cx = CXq(q), cy = CYq(q), cz = CZq(q);
        double v = f[q];
        M200 += cx * cx * v; M020 += cy * cy * v; M002 += cz * cz * v;
        M110 += cx * cy * v; M101 += cx * cz * v; M011 += cy * cz * v; M111 += cx * cy * cz * v;
        M201 += cx * cx * cz * v; M102 += cx * cz * cz * v; M210 += cx * cx * cy * v;
        M120 += cx * cy * cy * v; M021 += cy * cy * cz * v; M012 += cy * cz * cz * v;
    }
    const double cs2 = 1.0 / 3.0;
    kbc_mom m, e;
    /* raw moments and their equilibria (lbm_col_kbc_n.h:25-50) */
    double rT = M200 + M020 + M002, rNxz = M200 - M002, rNyz = M020 - M002;
    if (!central) {
        m.T = rT; m.Nxz = rNxz; m.Nyz = rNyz; m.Pxy = M110; m.Pxz = M101; m.Pyz = M011;
        m.Qxxy = M210; m.Qxxz = M201; m.Qxyy = M120; m.Qyyz = M021; m.Qxzz = M102; m.Qyzz = M012; m.Qxyz = M111;
        e.T = rho * (3.0 * cs2 + vx * vx + vy * vy + vz * vz);
        e.Nxz = rho * (vx * vx - vz * vz); e.Nyz = rho * (vy * vy - vz * vz);
        e.Pxy = rho * vx * vy; e.Pxz = rho * vx * vz; e.Pyz = rho * vy * vz;
        e.Qxxy = rho * vy * (cs2 + vx * vx); e.Qxxz = rho * vz * (cs2 + vx * vx);
        e.Qxyy = rho * vx * (cs2 + vy * vy); e.Qyyz = rho * vz * (cs2 + vy * vy);
        e.Qxzz = rho * vx * (cs2 + vz * vz); e.Qyzz = rho * vy * (cs2 + vz * vz);
        e.Qxyz = rho * vx * vy * vz;
    } else {
        /* central moments (lbm_col_kbc_c.h:53-79) */
        double cT = rT - rho * (vx * vx + vy * vy + vz * vz);
        double cNxz = rNxz + rho * (vz * vz - vx * vx);
        double cNyz = rNyz + rho * (vz * vz - vy * vy);
        double cPxy = M110 - rho * vx * vy, cPxz = M101 - rho * vx * vz, cPyz = M011 - rho * vy * vz;
        m.T = cT; m.Nxz = cNxz; m.Nyz = cNyz; m.Pxy = cPxy; m.Pxz = cPxz; m.Pyz = cPyz;
        m.Qxxy = M210 - (1.0 / 3.0) * (6.0 * vx * cPxy + vy * (3.0 * vx * vx + 2.0 * cNxz - cNyz + cT));
        m.Qxxz = M201 - (1.0 / 3.0) * (6.0 * vx * cPxz + vz * (3.0 * vx * vx + 2.0 * cNxz - cNyz + cT));
        m.Qxyy = M120 - (1.0 / 3.0) * (6.0 * vy * cPxy + vx * (3.0 * vy * vy + 2.0 * cNyz - cNxz + cT));
        m.Qyyz = M021 - (1.0 / 3.0) * (6.0 * vy * cPyz + vz * (3.0 * vy * vy + 2.0 * cNyz - cNxz + cT));
        m.Qxzz = M102 - (1.0 / 3.0) * (6.0 * vz * cPxz + vx * (3.0 * vz * vz - cNyz - cNxz + cT));
        m.Qyzz = M012 - (1.0 / 3.0) * (6.0 * vz * cPyz + vy * (3.0 * vz * vz - cNyz - cNxz + cT));
        m.Qxyz = M111 - vx * cPyz - vy * cPxz - vz * cPxy - vx * vy * vz;
        memset(&e, 0, sizeof e);
        e.T = rho * 3.0 * cs2;
    }
    double ds[27], dh[27];
    for (int q = 0; q < NQ; ++q) {
        ds[q] = kbc_shear_dir(q, &m, useT, useQ) - kbc_shear_dir(q, &e, useT, useQ);
        dh[q] = f[q] - ffeq[q] - ds[q];
    }
    const double beta = 1.0 / (2.0 * nu / cs2 + 1.0);
    double num = 0, den = 0;
    for (int q = 0; q < NQ; ++q) {
        double ifeq = 1.0 / ffeq[q];
        num += ds[q] * dh[q] * ifeq;
        den += dh[q] * dh[q] * ifeq;
    }
    /* the reference divides 0/0 when dh vanishes identically; then gamma*dh is zero for
     * any finite gamma, and the regularised limit 1/beta is used here */
    const double gamma = den != 0.0 ? 1.0 / beta - (2.0 - 1.0 / beta) * num / den : 1.0 / beta;
    for (int q = 0; q < NQ; ++q) {
        double S = force_src(CXq(q), CYq(q), CZq(q), rho, vx, vy, vz, fx, fy, fz);
        f[q] -= beta * (2.0 * ds[q] + gamma * dh[q]) - (1.0 - beta) * S * ffeq[q];
    }
}

void orc_collide(int col, double nu, double* f, double rho, double ux, double uy, double uz,
                 double fx, double fy, double fz)
{
    switch (col) {
    case ORC_COL_CUM: col_cum(f, rho, ux, uy, uz, nu); break;
    case ORC_COL_MRT: col_mrt(f, rho, ux, uy, uz, nu); break;
    case ORC_COL_BGK: col_bgk(f, rho, ux, uy, uz, fx, fy, fz, nu); break;
    default: {
        int central = col >= ORC_COL_KBC_C1;
        int v = central ? col - ORC_COL_KBC_C1 + 1 : col - ORC_COL_KBC_N1 + 1; /* 1..4 */
        int useT = (v == 2 || v == 4), useQ = (v == 3 || v == 4);
        col_kbc(f, rho, ux, uy, uz, fx, fy, fz, nu, central, useT, useQ);
    }
    }
}

/* ------------------------------------------------------------------------------------ */
/* Carreau-Yasuda local viscosity from the non-equilibrium second moments.                */
/* New model (no reference counterpart): Pi = sum f (c-u)(c-u) - rho/3 I,                 */
/* S = -3/(2 rho tau) Pi, gamma_dot = sqrt(2 S:S), nu solves                              */
/* nu = nu_inf + (nu0-nu_inf)(1+(lambda gamma_dot)^a)^((n-1)/a) with tau = 3 nu + 1/2.   */
/* Three Newton steps on g(tau) = tau - 3 nu_CY(K/tau) - 1/2 from tau = 3 nu0 + 1/2.      */
/* The viscosity law is the one of solver/lbm3d/core.h:763-766.                            */
/* ------------------------------------------------------------------------------------ */
double orc_local_nu(const double* f, double rho, double ux, double uy, double uz, double nu_inf,
                    double nu0, double lambda, double a, double n, double S[6])
{
    double Cxx = 0, Cyy = 0, Czz = 0, Cxy = 0, Cxz = 0, Cyz = 0;
    for (int q = 0; q < NQ; ++q) {
        double dx = CXq(q) - ux, dy = CYq(q) - uy, dz = CZq(q) - uz, v = f[q];
        Cxx += dx * dx * v; Cyy += dy * dy * v; Czz += dz * dz * v;
        Cxy += dx * dy * v; Cxz += dx * dz * v; Cyz += dy * dz * v;
    }
    const double Pxx = Cxx - rho / 3.0, Pyy = Cyy - rho / 3.0, Pzz = Czz - rho / 3.0;
    const double pn = sqrt(Pxx * Pxx + Pyy * Pyy + Pzz * Pzz + 2.0 * (Cxy * Cxy + Cxz * Cxz + Cyz * Cyz));
    const double K = 3.0 * sqrt(2.0) * pn / (2.0 * rho);
    double tau = 3.0 * nu0 + 0.5;
    if (K > 0.0) {
        const double e = (n - 1.0) / a;
        for (int it = 0; it < 3; ++it) {
            double g = K / tau;
            double s = pow(lambda * g, a);
            double p = pow(1.0 + s, e);
            double nuc = nu_inf + (nu0 - nu_inf) * p;
            double G = tau - 3.0 * nuc - 0.5;
            double gdn = (nu0 - nu_inf) * (n - 1.0) * s * p / (1.0 + s);
            double Gp = 1.0 + 3.0 * gdn / tau;
            tau = tau - G / Gp;
        }
    }
    const double sc = -3.0 / (2.0 * rho * tau);
    S[0] = sc * Pxx; S[1] = sc * Cxy; S[2] = sc * Cxz; S[3] = sc * Pyy; S[4] = sc * Cyz; S[5] = sc * Pzz;
    return (tau - 0.5) / 3.0;
}

/* ------------------------------------------------------------------------------------ */
/* lattice                                                                                */
/* ------------------------------------------------------------------------------------ */
orc_lattice* orc_create(const orc_desc* d)
{
    if (d->nx < 3 || d->ny < 3 || d->nz < 3) return NULL;
    orc_lattice* L = (orc_lattice*)calloc(1, sizeof *L);
    L->d = *d;
    L->N = (int64_t)d->nx * d->ny * d->nz;
    L->map = (uint8_t*)calloc((size_t)L->N, 1);
    L->df[0] = (double*)calloc((size_t)L->N * NQ, sizeof(double));
    L->df[1] = (double*)calloc((size_t)L->N * NQ, sizeof(double));
    L->macro = (double*)calloc((size_t)L->N * ORC_M_N, sizeof(double));
    L->prof = (double*)calloc((size_t)L->N * 3, sizeof(double));
    L->rho_left = L->rho_right = L->rho_eq = 1.0;
    return L;
}

void orc_destroy(orc_lattice* L)
{
    if (!L) return;
    free(L->map); free(L->df[0]); free(L->df[1]); free(L->macro); free(L->prof); free(L);
}

int orc_set_map(orc_lattice* L, const uint8_t* map)
{
    memcpy(L->map, map, (size_t)L->N);
    int64_t la = 0, ra = 0;
    for (int64_t c = 0; c < L->N; ++c) {
        if (map[c] > ORC_OUTFLOW_RIGHT_EQ) return -1;
        la += map[c] == ORC_INFLOW_LEFT;
        ra += map[c] == ORC_INFLOW_RIGHT;
    }
    L->left_area = la; L->right_area = ra;
    return 0;
}

int orc_get_map(const orc_lattice* L, uint8_t* map)
{
    memcpy(map, L->map, (size_t)L->N);
    return 0;
}

/* StateTcpc::setupBoundaries (sim_tcpc.cu:494-645) followed by LBM::projectWall
 * (lbm.hpp:144-155); wall[] is the geometry's cell array, x fastest (sim_tcpc.cu:508-512) */
int orc_setup_tcpc(orc_lattice* L, const int32_t* wall, int64_t counts[10])
{
    const int X = L->d.nx, Y = L->d.ny, Z = L->d.nz;
    uint8_t* wf = (uint8_t*)calloc((size_t)L->N, 1);
    int64_t in3 = 0, in4 = 0, in5 = 0, in6 = 0;
    for (int z = 0; z < Z; ++z)
        for (int y = 0; y < Y; ++y)
            for (int x = 0; x < X; ++x) {
                int64_t c = cidx(L, x, y, z);
                int lab = wall[c];
                in3 += lab == 3; in4 += lab == 4; in5 += lab == 5; in6 += lab == 6;
                L->map[c] = ORC_FLUID;
                wf[c] = lab == ORC_WALL;
            }
    for (int z = 0; z < Z; ++z)
        for (int y = 0; y < Y; ++y) {
            L->map[cidx(L, 0, y, z)] = ORC_INFLOW_LEFT;
            L->map[cidx(L, X - 1, y, z)] = ORC_INFLOW_RIGHT;
        }
    for (int z = 0; z < Z; ++z)
        for (int x = 0; x < X; ++x) {
            L->map[cidx(L, x, 0, z)] = ORC_OUTFLOW_FRONT;
            L->map[cidx(L, x, Y - 1, z)] = ORC_OUTFLOW_BACK;
        }
    for (int y = 0; y < Y; ++y)
        for (int x = 0; x < X; ++x) {
            L->map[cidx(L, x, y, 0)] = ORC_WALL;
            L->map[cidx(L, x, y, Z - 1)] = ORC_WALL;
        }
    /* openBoundaryX / openBoundaryY (sim_tcpc.cu:531-586) */
    for (int side = 0; side < 2; ++side) {
        int bx = side == 0 ? 0 : X - 1, st = side == 0 ? 1 : -1;
        int sx = bx + st;
        for (;;) {
            if (!(sx > 0 && sx < X - 1)) break;
            int64_t open = 0;
            for (int z = 0; z < Z; ++z)
                for (int y = 0; y < Y; ++y) open += !wf[cidx(L, sx, y, z)];
            if (open != 0) break;
            sx += st;
        }
        if (sx <= 0 || sx >= X - 1) continue;
        for (int z = 0; z < Z; ++z)
            for (int y = 0; y < Y; ++y)
                if (!wf[cidx(L, sx, y, z)])
                    for (int x = bx; x != sx + st; x += st) wf[cidx(L, x, y, z)] = 0;
    }
    for (int side = 0; side < 2; ++side) {
        int by = side == 0 ? 0 : Y - 1, st = side == 0 ? 1 : -1;
        int sy = by + st;
        for (;;) {
            if (!(sy > 0 && sy < Y - 1)) break;
            int64_t open = 0;
            for (int z = 0; z < Z; ++z)
                for (int x = 0; x < X; ++x) open += !wf[cidx(L, x, sy, z)];
            if (open != 0) break;
            sy += st;
        }
        if (sy <= 0 || sy >= Y - 1) continue;
        for (int z = 0; z < Z; ++z)
            for (int x = 0; x < X; ++x)
                if (!wf[cidx(L, x, sy, z)])
                    for (int y = by; y != sy + st; y += st) wf[cidx(L, x, y, z)] = 0;
    }
    int64_t la = 0, ra = 0, of = 0, ob = 0, wc = 0, fc = 0;
    for (int64_t c = 0; c < L->N; ++c) {
        int lab = L->map[c];
        int is_wall = wf[c] || lab == ORC_WALL;
        la += lab == ORC_INFLOW_LEFT && !is_wall;
        ra += lab == ORC_INFLOW_RIGHT && !is_wall;
        of += lab == ORC_OUTFLOW_FRONT && !is_wall;
        ob += lab == ORC_OUTFLOW_BACK && !is_wall;
        wc += is_wall;
        fc += lab == ORC_FLUID && !is_wall;
    }
    for (int64_t c = 0; c < L->N; ++c)
        if (wf[c]) L->map[c] = ORC_WALL;
    free(wf);
    L->left_area = la; L->right_area = ra;
    if (counts) {
        counts[0] = la; counts[1] = ra; counts[2] = of; counts[3] = ob; counts[4] = wc; counts[5] = fc;
        counts[6] = in3; counts[7] = in4; counts[8] = in5; counts[9] = in6;
    }
    return (la <= 0 || ra <= 0 || of <= 0 || ob <= 0) ? 1 : 0;
}

/* resetLattice (sim_tcpc.cu:647-655, lbm.hpp:1-39) then LBMKernelInit (core.h:833-863) */
void orc_init_equilibrium(orc_lattice* L, double rho, double ux, double uy, double uz)
{
    double feq[27];
    orc_feq(L->d.equilibrium, rho, ux, uy, uz, feq);
    for (int64_t c = 0; c < L->N; ++c)
        for (int q = 0; q < NQ; ++q) L->df[0][c * NQ + q] = L->df[1][c * NQ + q] = feq[q];
    L->cur = 0;
    L->iterations = 0;
    memset(L->macro, 0, sizeof(double) * (size_t)L->N * ORC_M_N);
    for (int64_t c = 0; c < L->N; ++c) {
        int lab = L->map[c];
        double r[4] = {1.0, 0.0, 0.0, 0.0};
        if (lab == ORC_FLUID || lab == ORC_PERIODIC)
            orc_density_velocity(&L->df[0][c * NQ], L->d.fx, L->d.fy, L->d.fz, r);
        L->macro[ORC_M_RHO * L->N + c] = r[0];
        L->macro[ORC_M_VX * L->N + c] = r[1];
        L->macro[ORC_M_VY * L->N + c] = r[2];
        L->macro[ORC_M_VZ * L->N + c] = r[3];
        L->macro[ORC_M_FX * L->N + c] = L->d.fx;
        L->macro[ORC_M_FY * L->N + c] = L->d.fy;
        L->macro[ORC_M_FZ * L->N + c] = L->d.fz;
    }
}

void orc_set_inflow(orc_lattice* L, double ivc_flux, double svc_flux, double rho_left,
                    double rho_right, double rho_eq)
{
    L->ivc_flux = ivc_flux; L->svc_flux = svc_flux;
    L->rho_left = rho_left; L->rho_right = rho_right; L->rho_eq = rho_eq;
}

void orc_set_inflow_profile(orc_lattice* L, const double* u3)
{
    memcpy(L->prof, u3, sizeof(double) * 3 * (size_t)L->N);
}

/* neighbour indices, core.h:639-661 (single rank: x is clamped unless periodic) */
static void neighbours(const orc_lattice* L, int x, int y, int z, int lab, int xs[3], int ys[3], int zs[3])
{
    const int X = L->d.nx, Y = L->d.ny, Z = L->d.nz;
    xs[1] = x; ys[1] = y; zs[1] = z;
    if (lab == ORC_PERIODIC) {
        xs[2] = x == X - 1 ? 0 : x + 1; xs[0] = x == 0 ? X - 1 : x - 1;
        ys[2] = y == Y - 1 ? 0 : y + 1; ys[0] = y == 0 ? Y - 1 : y - 1;
        zs[2] = z == Z - 1 ? 0 : z + 1; zs[0] = z == 0 ? Z - 1 : z - 1;
    } else {
        xs[2] = x + 1 < X - 1 ? x + 1 : X - 1; xs[0] = x - 1 > 0 ? x - 1 : 0;
        ys[2] = y + 1 < Y - 1 ? y + 1 : Y - 1; ys[0] = y - 1 > 0 ? y - 1 : 0;
        zs[2] = z + 1 < Z - 1 ? z + 1 : Z - 1; zs[0] = z - 1 > 0 ? z - 1 : 0;
    }
}

/* LBM_STREAMING::streaming (lbm_streaming.h:10-39): f_q <- src at x - c_q, taken from the
 * supplied (xm,x,xp) triples; a triple may be re-centred on a neighbour by the BCs.
 * With halfway bounce-back (no reference counterpart: the reference has wall nodes only,
 * lbm_streaming.h:78-107) a population that would come from a WALL cell is the centre's own
 * post-collision population of the opposite direction, f_q <- src_opp(q) at the centre; the
 * rule holds for every pull, the re-centred stencils of the open planes included. */
static void pull(const orc_lattice* L, const double* src, const int xs[3], const int ys[3],
                 const int zs[3], double* f)
{
    const int64_t centre = cidx(L, xs[1], ys[1], zs[1]);
    for (int q = 0; q < NQ; ++q) {
        const int64_t s = cidx(L, xs[1 - CXq(q)], ys[1 - CYq(q)], zs[1 - CZq(q)]);
        f[q] = (L->d.halfway_bounce_back && L->map[s] == ORC_WALL) ? src[centre * NQ + OPP(q)] : src[s * NQ + q];
    }
}

/* streamingBounceBack (lbm_streaming.h:78-107): f_{opp q} <- incoming f_q */
static void pull_bounce_back(const orc_lattice* L, const double* src, const int xs[3],
                             const int ys[3], const int zs[3], double* f)
{
    for (int q = 0; q < NQ; ++q)
        f[OPP(q)] = src[cidx(L, xs[1 - CXq(q)], ys[1 - CYq(q)], zs[1 - CZq(q)]) * NQ + q];
}

static inline double MACRO(const orc_lattice* L, int fld, int64_t c) { return L->macro[(int64_t)fld * L->N + c]; }
static inline double* MACROP(orc_lattice* L, int fld, int64_t c) { return &L->macro[(int64_t)fld * L->N + c]; }

static inline int is_fluid(int lab) { return lab == ORC_FLUID; }

/* one-sided / central first derivative of a macro component along one axis, following
 * the branch structure of core.h:677-761 and core.h:489-573 */
static double fd1(const orc_lattice* L, int fld, int64_t cm, int64_t c0, int64_t cp, int labm, int labp,
                  double wgt_center)
{
    if (!is_fluid(labm)) {
        if (!is_fluid(labp)) return 0.0;
        return MACRO(L, fld, cp) - MACRO(L, fld, c0);
    } else if (!is_fluid(labp)) {
        return MACRO(L, fld, c0) - MACRO(L, fld, cm);
    }
    return wgt_center * (MACRO(L, fld, cp) - MACRO(L, fld, cm));
}

/* cudaLBMKernelVelocity restricted to FLUID cells (core.h:273-384): the only values that
 * the strain stencil reads (it skips every non-FLUID neighbour) */
static void phase_velocity(orc_lattice* L, const double* src)
{
    const int X = L->d.nx, Y = L->d.ny, Z = L->d.nz;
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < Z; ++z)
        for (int y = 0; y < Y; ++y)
            for (int x = 0; x < X; ++x) {
                int64_t c = cidx(L, x, y, z);
                int lab = L->map[c];
                if (!is_fluid(lab)) continue;
                int xs[3], ys[3], zs[3];
                double f[27], r[4];
                neighbours(L, x, y, z, lab, xs, ys, zs);
                pull(L, src, xs, ys, zs, f);
                orc_density_velocity(f, MACRO(L, ORC_M_FX, c), MACRO(L, ORC_M_FY, c), MACRO(L, ORC_M_FZ, c), r);
                *MACROP(L, ORC_M_RHO, c) = r[0];
                *MACROP(L, ORC_M_VX, c) = r[1];
                *MACROP(L, ORC_M_VY, c) = r[2];
                *MACROP(L, ORC_M_VZ, c) = r[3];
            }
}

/* cudaLBMKernelStress (core.h:387-576): finite-difference strain of the macro velocity */
static void phase_stress(orc_lattice* L)
{
    const int X = L->d.nx, Y = L->d.ny, Z = L->d.nz;
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < Z; ++z)
        for (int y = 0; y < Y; ++y)
            for (int x = 0; x < X; ++x) {
                int64_t c = cidx(L, x, y, z);
                int lab = L->map[c];
                double S11 = 0, S12 = 0, S13 = 0, S22 = 0, S32 = 0, S33 = 0;
                if (is_fluid(lab)) {
                    int xs[3], ys[3], zs[3];
                    neighbours(L, x, y, z, lab, xs, ys, zs);
                    int64_t cxm = cidx(L, xs[0], y, z), cxp = cidx(L, xs[2], y, z);
                    int64_t cym = cidx(L, x, ys[0], z), cyp = cidx(L, x, ys[2], z);
                    int64_t czm = cidx(L, x, y, zs[0]), czp = cidx(L, x, y, zs[2]);
                    int lxm = L->map[cxm], lxp = L->map[cxp], lym = L->map[cym], lyp = L->map[cyp];
                    int lzm = L->map[czm], lzp = L->map[czp];
                    /* x: S11 and the x-halves of S12, S13 (core.h:489-517) */
                    S11 = fd1(L, ORC_M_VX, cxm, c, cxp, lxm, lxp, 0.5);
                    S12 += 0.5 * fd1(L, ORC_M_VY, cxm, c, cxp, lxm, lxp, 0.5);
                    S13 += 0.5 * fd1(L, ORC_M_VZ, cxm, c, cxp, lxm, lxp, 0.5);
                    /* y: S22 and the y-halves of S12, S32 (core.h:519-544) */
                    S22 = fd1(L, ORC_M_VY, cym, c, cyp, lym, lyp, 0.5);
                    S12 += 0.5 * fd1(L, ORC_M_VX, cym, c, cyp, lym, lyp, 0.5);
                    S32 += 0.5 * fd1(L, ORC_M_VZ, cym, c, cyp, lym, lyp, 0.5);
                    /* z: S33 and the z-halves of S13, S32 (core.h:546-572) */
                    S33 = fd1(L, ORC_M_VZ, czm, c, czp, lzm, lzp, 0.5);
                    S13 += 0.5 * fd1(L, ORC_M_VX, czm, c, czp, lzm, lzp, 0.5);
                    S32 += 0.5 * fd1(L, ORC_M_VY, czm, c, czp, lzm, lzp, 0.5);
                }
                *MACROP(L, ORC_M_S11, c) = S11; *MACROP(L, ORC_M_S12, c) = S12; *MACROP(L, ORC_M_S13, c) = S13;
                *MACROP(L, ORC_M_S22, c) = S22; *MACROP(L, ORC_M_S32, c) = S32; *MACROP(L, ORC_M_S33, c) = S33;
            }
}

/* the fused step for one cell: cudaLBMKernel (core.h:578-800) with LBM_BC_Tcpc
 * (sim_tcpc.cu:228-278), the generic inflow / outflow blocks (lbm_bc.h:126-152) and
 * MacroTcpc::outputMacro (sim_tcpc.cu:337-354) */
static void cell_step(orc_lattice* L, const double* src, double* dst, int x, int y, int z, int acc)
{
    const orc_desc* d = &L->d;
    const int64_t c = cidx(L, x, y, z);
    const int lab = L->map[c];
    double f[27];
    double rho = 1.0, vx = 0.0, vy = 0.0, vz = 0.0;
    double fx = d->fx, fy = d->fy, fz = d->fz;
    double nu = d->nu;
    int xs[3], ys[3], zs[3];
    neighbours(L, x, y, z, lab, xs, ys, zs);

    if (d->cy_mode == ORC_CY_REF_FD) {
        /* core.h:663-781: divergence of S by the same one-sided rules, CY viscosity with
         * single precision powf, KS.rho still at its default of 1 */
        int64_t cxm = cidx(L, xs[0], y, z), cxp = cidx(L, xs[2], y, z);
        int64_t cym = cidx(L, x, ys[0], z), cyp = cidx(L, x, ys[2], z);
        int64_t czm = cidx(L, x, y, zs[0]), czp = cidx(L, x, y, zs[2]);
        double F1 = 0, F2 = 0, F3 = 0;
        if (is_fluid(lab)) {
            int lxm = L->map[cxm], lxp = L->map[cxp], lym = L->map[cym], lyp = L->map[cyp];
            int lzm = L->map[czm], lzp = L->map[czp];
            F1 += fd1(L, ORC_M_S11, cxm, c, cxp, lxm, lxp, 0.5);
            F2 += fd1(L, ORC_M_S12, cxm, c, cxp, lxm, lxp, 0.5);
            F3 += fd1(L, ORC_M_S13, cxm, c, cxp, lxm, lxp, 0.5);
            F1 += fd1(L, ORC_M_S12, cym, c, cyp, lym, lyp, 0.5);
            F2 += fd1(L, ORC_M_S22, cym, c, cyp, lym, lyp, 0.5);
            F3 += fd1(L, ORC_M_S32, cym, c, cyp, lym, lyp, 0.5);
            F1 += fd1(L, ORC_M_S13, czm, c, czp, lzm, lzp, 0.5);
            F2 += fd1(L, ORC_M_S32, czm, c, czp, lzm, lzp, 0.5);
            F3 += fd1(L, ORC_M_S33, czm, c, czp, lzm, lzp, 0.5);
        }
        double S11 = MACRO(L, ORC_M_S11, c), S12 = MACRO(L, ORC_M_S12, c), S13 = MACRO(L, ORC_M_S13, c);
        double S22 = MACRO(L, ORC_M_S22, c), S32 = MACRO(L, ORC_M_S32, c), S33 = MACRO(L, ORC_M_S33, c);
        double gamma = sqrt(2.0) * sqrt(S11 * S11 + S22 * S22 + S33 * S33 + 2.0 * (S12 * S12 + S13 * S13 + S32 * S32));
        /* the reference evaluates the law with single-precision powf; here each power is
         * taken in double and rounded once to float, i.e. the correctly rounded powf */
        float inner = (float)pow((double)(float)(gamma * d->cy_lambda), (double)(float)d->cy_a);
        float outer = (float)pow((double)(float)(1.0 + (double)inner), (double)(float)((d->cy_n - 1.0) / d->cy_a));
        double nuc = nu + (d->cy_nu0 - nu) * (double)outer;
        fx += 2.0 * (nuc - nu) * F1 * 1.0;
        fy += 2.0 * (nuc - nu) * F2 * 1.0;
        fz += 2.0 * (nuc - nu) * F3 * 1.0;
    }

    if (lab == ORC_FLUID || lab == ORC_PERIODIC) {
        pull(L, src, xs, ys, zs, f);
        double r[4];
        orc_density_velocity(f, fx, fy, fz, r);
        rho = r[0]; vx = r[1]; vy = r[2]; vz = r[3];
    }

    double S6[6] = {0, 0, 0, 0, 0, 0};
    switch (lab) {
    case ORC_WALL:
        if (d->halfway_bounce_back) {
            memcpy(f, &src[c * NQ], sizeof f);
        } else {
            pull_bounce_back(L, src, xs, ys, zs, f);
        }
        rho = 1.0; vx = vy = vz = 0.0;
        break;
    case ORC_INFLOW_LEFT:
    case ORC_INFLOW_RIGHT: {
        /* sim_tcpc.cu:242-261: density of the post-streaming state one cell inward */
        double fl[27], r[4];
        int lx[3];
        if (lab == ORC_INFLOW_LEFT) { lx[0] = x; lx[1] = xs[2]; lx[2] = xs[2] + 1; }
        else { lx[0] = xs[0] - 1; lx[1] = xs[0]; lx[2] = x; }
        pull(L, src, lx, ys, zs, fl);
        orc_density_velocity(fl, 0.0, 0.0, 0.0, r);
        int64_t area = lab == ORC_INFLOW_LEFT ? L->left_area : L->right_area;
        double flux = lab == ORC_INFLOW_LEFT ? L->ivc_flux : -L->svc_flux;
        vx = area > 0 ? flux / (double)area : 0.0;
        vy = 0.0; vz = 0.0;
        rho = r[0];
        orc_feq(d->equilibrium, rho, vx, vy, vz, f);
        break;
    }
    case ORC_OUTFLOW_FRONT:
    case ORC_OUTFLOW_BACK: {
        /* sim_tcpc.cu:262-273: velocity of the post-streaming state one cell inward */
        int ly[3];
        double r[4];
        if (lab == ORC_OUTFLOW_FRONT) { ly[0] = y; ly[1] = ys[2]; ly[2] = ys[2] + 1; }
        else { ly[0] = ys[0] - 1; ly[1] = ys[0]; ly[2] = y; }
        pull(L, src, xs, ly, zs, f);
        orc_density_velocity(f, fx, fy, fz, r);
        rho = 1.0; vx = r[1]; vy = r[2]; vz = r[3];
        orc_feq(d->equilibrium, rho, vx, vy, vz, f);
        break;
    }
    case ORC_INFLOW_EQ:
        /* lbm_bc.h:126-129 with a per-cell prescribed velocity */
        rho = L->rho_eq;
        vx = L->prof[c]; vy = L->prof[L->N + c]; vz = L->prof[2 * L->N + c];
        orc_feq(d->equilibrium, rho, vx, vy, vz, f);
        break;
    case ORC_OUTFLOW_RIGHT_EQ: {
        /* lbm_bc.h:147-152 */
        int lx[3];
        double r[4];
        lx[0] = xs[0] - 1; lx[1] = xs[0]; lx[2] = x;
        pull(L, src, lx, ys, zs, f);
        orc_density_velocity(f, fx, fy, fz, r);
        rho = 1.0; vx = r[1]; vy = r[2]; vz = r[3];
        orc_feq(d->equilibrium, rho, vx, vy, vz, f);
        break;
    }
    default: {
        double nuc = nu;
        if (d->cy_mode == ORC_CY_LOCAL_NEQ)
            nuc = orc_local_nu(f, rho, vx, vy, vz, nu, d->cy_nu0, d->cy_lambda, d->cy_a, d->cy_n, S6);
        orc_collide(d->collision, nuc, f, rho, vx, vy, vz, fx, fy, fz);
    }
    }
    memcpy(&dst[c * NQ], f, sizeof f);

    *MACROP(L, ORC_M_RHO, c) = rho;
    *MACROP(L, ORC_M_VX, c) = vx;
    *MACROP(L, ORC_M_VY, c) = vy;
    *MACROP(L, ORC_M_VZ, c) = vz;
    *MACROP(L, ORC_M_FX, c) = fx;
    *MACROP(L, ORC_M_FY, c) = fy;
    *MACROP(L, ORC_M_FZ, c) = fz;
    if (d->cy_mode == ORC_CY_LOCAL_NEQ) {
        *MACROP(L, ORC_M_S11, c) = S6[0]; *MACROP(L, ORC_M_S12, c) = S6[1]; *MACROP(L, ORC_M_S13, c) = S6[2];
        *MACROP(L, ORC_M_S22, c) = S6[3]; *MACROP(L, ORC_M_S32, c) = S6[4]; *MACROP(L, ORC_M_S33, c) = S6[5];
    }
    if (acc) {
        *MACROP(L, ORC_M_VM_PLUS_X, c) += (vx > 0) ? rho * vx : 0;
        *MACROP(L, ORC_M_VM_MINUS_X, c) += (vx < 0) ? rho * vx : 0;
        *MACROP(L, ORC_M_VM_Y, c) += rho * vy;
        *MACROP(L, ORC_M_VM_Z, c) += rho * vz;
        *MACROP(L, ORC_M_VM_XX, c) += rho * rho * vx * vx;
        *MACROP(L, ORC_M_VM_YY, c) += rho * rho * vy * vy;
        *MACROP(L, ORC_M_VM_ZZ, c) += rho * rho * vz * vz;
    }
}

void orc_step(orc_lattice* L, int accumulate_stats)
{
    const int X = L->d.nx, Y = L->d.ny, Z = L->d.nz;
    const double* src = L->df[L->cur];
    double* dst = L->df[1 - L->cur];
    if (L->d.cy_mode == ORC_CY_REF_FD) {
        /* the three phases of the multi-rank step, core.h:1169-1310 */
        phase_velocity(L, src);
        phase_stress(L);
    }
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < Z; ++z)
        for (int y = 0; y < Y; ++y)
            for (int x = 0; x < X; ++x) cell_step(L, src, dst, x, y, z, accumulate_stats);
    L->cur = 1 - L->cur;
    L->iterations++;
}

void orc_get_df(const orc_lattice* L, double* out)
{
    const double* a = L->df[L->cur];
    for (int64_t c = 0; c < L->N; ++c)
        for (int q = 0; q < NQ; ++q) out[(int64_t)q * L->N + c] = a[c * NQ + q];
}

void orc_set_df(orc_lattice* L, const double* in)
{
    double* a = L->df[L->cur];
    for (int64_t c = 0; c < L->N; ++c)
        for (int q = 0; q < NQ; ++q) a[c * NQ + q] = in[(int64_t)q * L->N + c];
}

void orc_get_macro(const orc_lattice* L, int field, double* out)
{
    memcpy(out, &L->macro[(int64_t)field * L->N], sizeof(double) * (size_t)L->N);
}

void orc_set_macro(orc_lattice* L, int field, const double* in)
{
    memcpy(&L->macro[(int64_t)field * L->N], in, sizeof(double) * (size_t)L->N);
}

/* StateTcpc::statReset, sim_tcpc.cu:665-682 */
void orc_stat_reset(orc_lattice* L)
{
    for (int fld = ORC_M_VM_PLUS_X; fld <= ORC_M_VM_ZZ; ++fld)
        memset(&L->macro[(int64_t)fld * L->N], 0, sizeof(double) * (size_t)L->N);
}

/* mass and the plane fluxes of postprocess/compute_flows.py:107-147 in lattice units,
 * inflow positive for the IVC/SVC planes and outflow positive for the outlets */
void orc_reduce(const orc_lattice* L, double out[5])
{
    double mass = 0, q3 = 0, q4 = 0, q5 = 0, q6 = 0;
    for (int64_t c = 0; c < L->N; ++c) {
        int lab = L->map[c];
        if (lab == ORC_FLUID || lab == ORC_PERIODIC) mass += MACRO(L, ORC_M_RHO, c);
        if (lab == ORC_INFLOW_LEFT) q3 += MACRO(L, ORC_M_VX, c);
        if (lab == ORC_INFLOW_RIGHT) q4 -= MACRO(L, ORC_M_VX, c);
        if (lab == ORC_OUTFLOW_FRONT) q5 -= MACRO(L, ORC_M_VY, c);
        if (lab == ORC_OUTFLOW_BACK) q6 += MACRO(L, ORC_M_VY, c);
    }
    out[0] = mass; out[1] = q3; out[2] = q4; out[3] = q5; out[4] = q6;
}

int64_t orc_iterations(const orc_lattice* L) { return L->iterations; }
