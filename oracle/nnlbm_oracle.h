/*
 * nnlbm_oracle.h -- FP64 CPU oracle for the fused D3Q27 stream + collide step of the
 * TCPC lattice-Boltzmann solver (buresjan/nonnewlbm).
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference algorithm,
 * used by tests/, __graft_entry__.smoke() and the cpu_baseline / reference legs of
 * bench.py as the checker.  The product path (nonnewlbm_b200/libnnlbm.so) never links,
 * loads or calls anything in this directory.
 *
 * Semantics follow the reference's two-lattice pull step (solver/lbm3d/core.h:578-800,
 * A-B buffers rotated per step, solver/lbm3d/lbm.hpp:392-418) with the TCPC policies of
 * solver/sim_tcpc/sim_tcpc.cu:187-418 and the generic inflow / outflow blocks of
 * solver/lbm3d/lbm_bc.h:126-152.  Every function in nnlbm_oracle.c cites the reference
 * lines it follows.
 *
 * Layouts used at this interface (all row-major, x fastest):
 *   cell c = x + nx*(y + ny*z)
 *   populations [27][nz][ny][nx]; direction q = 9*(cx+1) + 3*(cy+1) + (cz+1), which is
 *   the reference's direction enum (solver/lbm3d/defs.h:215-247, mmm=0 ... ppp=26).
 */
#ifndef NNLBM_ORACLE_H
#define NNLBM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* solver map labels: 0..6 are LBM_BC_Tcpc::GEO (sim_tcpc.cu:194-203); 7 and 8 are the
 * generic GEO_INFLOW and GEO_OUTFLOW_RIGHT_EQ blocks of lbm_bc.h:126-129,147-152 */
enum {
    ORC_FLUID = 0, ORC_WALL = 1, ORC_PERIODIC = 2, ORC_INFLOW_LEFT = 3, ORC_INFLOW_RIGHT = 4,
    ORC_OUTFLOW_FRONT = 5, ORC_OUTFLOW_BACK = 6, ORC_INFLOW_EQ = 7, ORC_OUTFLOW_RIGHT_EQ = 8
};

/* collision ids, in the order of the collision selector strings
 * CUM, KBC_N1..KBC_N4, KBC_C1..KBC_C4, MRT_LES, BGK */
enum {
    ORC_COL_CUM = 0, ORC_COL_KBC_N1 = 1, ORC_COL_KBC_N2, ORC_COL_KBC_N3, ORC_COL_KBC_N4,
    ORC_COL_KBC_C1 = 5, ORC_COL_KBC_C2, ORC_COL_KBC_C3, ORC_COL_KBC_C4,
    ORC_COL_MRT = 9, ORC_COL_BGK = 10
};

/* equilibria used by setEquilibrium (BC nodes) and by the initial condition */
enum {
    ORC_EQ_INV_CUM_REF = 0, /* LBM_EQ_INV_CUM exactly as shipped, incl. the rho^2 in feq_pmm */
    ORC_EQ_INV_CUM = 1,     /* the same factorised equilibrium with feq_pmm corrected */
    ORC_EQ_DEFAULT = 2,     /* LBM_EQ_DEFAULT second-order Maxwellian */
    ORC_EQ_ENTROPIC = 3     /* LBM_EQ_ENTROPIC */
};

enum { ORC_CY_NONE = 0, ORC_CY_REF_FD = 1, ORC_CY_LOCAL_NEQ = 2 };

/* macro fields (MacroTcpc enum, sim_tcpc.cu:328-335) */
enum {
    ORC_M_RHO = 0, ORC_M_VX, ORC_M_VY, ORC_M_VZ,
    ORC_M_VM_PLUS_X, ORC_M_VM_MINUS_X, ORC_M_VM_Y, ORC_M_VM_Z,
    ORC_M_VM_XX, ORC_M_VM_YY, ORC_M_VM_ZZ,
    ORC_M_FX, ORC_M_FY, ORC_M_FZ,
    ORC_M_S11, ORC_M_S12, ORC_M_S13, ORC_M_S22, ORC_M_S32, ORC_M_S33,
    ORC_M_N
};

typedef struct {
    int nx, ny, nz;
    int collision;
    int equilibrium;
    int cy_mode;
    int halfway_bounce_back; /* 0: wall nodes with full-way bounce-back (reference); 1: halfway:
                                every pull from a WALL cell takes the pulling centre's own
                                post-collision population of the opposite direction */
    double nu;               /* lattice viscosity (nu_inf when Carreau-Yasuda is on) */
    double cy_nu0, cy_lambda, cy_a, cy_n;
    double fx, fy, fz;       /* homogeneous body force */
} orc_desc;

typedef struct orc_lattice orc_lattice;

orc_lattice* orc_create(const orc_desc* d);
void orc_destroy(orc_lattice* L);
int orc_set_map(orc_lattice* L, const uint8_t* map);
int orc_get_map(const orc_lattice* L, uint8_t* map);
/* mask -> labels (sim_tcpc.cu:494-645 + lbm.hpp:144-155); counts =
 * {left_area, right_area, out_front, out_back, wall, fluid, vtk3, vtk4, vtk5, vtk6} */
int orc_setup_tcpc(orc_lattice* L, const int32_t* wall, int64_t counts[10]);
void orc_init_equilibrium(orc_lattice* L, double rho, double ux, double uy, double uz);
/* TCPC inflow data (LBM_Data_Tcpc, sim_tcpc.cu:288-309 and :657-663) plus the constant
 * density of the generic INFLOW_EQ cells */
void orc_set_inflow(orc_lattice* L, double ivc_flux, double svc_flux, double rho_left,
                    double rho_right, double rho_eq);
/* per-cell prescribed velocity of INFLOW_EQ cells, [3][N] (component-major) */
void orc_set_inflow_profile(orc_lattice* L, const double* u3);
void orc_step(orc_lattice* L, int accumulate_stats);
void orc_get_df(const orc_lattice* L, double* out);   /* [27][N] post-collision state */
void orc_set_df(orc_lattice* L, const double* in);
void orc_get_macro(const orc_lattice* L, int field, double* out); /* [N] */
void orc_set_macro(orc_lattice* L, int field, const double* in);
void orc_stat_reset(orc_lattice* L);
/* {mass over FLUID+PERIODIC, Q_ivc, Q_svc, Q_out5, Q_out6} in lattice units */
void orc_reduce(const orc_lattice* L, double out[5]);
int64_t orc_iterations(const orc_lattice* L);
void orc_set_threads(int n);

/* per-cell kernels, exposed for known-answer tests */
void orc_feq(int eq, double rho, double ux, double uy, double uz, double f[27]);
/* rho/u exactly as LBM_COMMON::computeDensityAndVelocity (lbm_common.h:16-39) */
void orc_density_velocity(const double* f, double fx, double fy, double fz, double out[4]);
/* one collision, in place; rho/u/force as the kernel would pass them */
void orc_collide(int col, double nu, double* f, double rho, double ux, double uy, double uz,
                 double fx, double fy, double fz);
/* Carreau-Yasuda local viscosity from the non-equilibrium second moments; returns nu,
 * writes S (S11,S12,S13,S22,S32,S33) */
double orc_local_nu(const double* f, double rho, double ux, double uy, double uz,
                    double nu_inf, double nu0, double lambda, double a, double n, double S[6]);

#ifdef __cplusplus
}
#endif
#endif
