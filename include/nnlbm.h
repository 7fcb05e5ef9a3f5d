/*
 * nnlbm.h -- C ABI of libnnlbm.so, the B200 (sm_100a) implementation of the fused D3Q27
 * stream + collide step of the TCPC lattice-Boltzmann solver (buresjan/nonnewlbm).
 *
 * Plain C: no exceptions cross the boundary, every call returns an nnlbm_status, sizes are
 * explicit and host buffers are caller-owned, C-contiguous and copied synchronously.  The
 * library owns every device buffer.  One context is driven by one host thread at a time.
 *
 * Each entry point states the reference interface it replaces.  In the reference the
 * step is reached through a process boundary (scripts/run_case.py:21-95 builds the
 * sim_tcpc argv, solver/sim_tcpc/sim_tcpc.cu:70-125 parses it) and, inside the process,
 * through the compile-time policy API LBM_TYPE / STREAMING / MACRO / LBM_DATA / LBM_BC
 * composed in sim_tcpc.cu:431-438 and dispatched by SimUpdate (solver/lbm3d/core.h:1025).
 *
 * Layouts at this boundary (x fastest everywhere):
 *   cell            c = x + nx*(y + ny*z)
 *   labels / masks  [nz][ny][nx]
 *   populations     [27][nz][ny][nx], direction q = 9*(cx+1) + 3*(cy+1) + (cz+1), i.e. the
 *                   reference direction enum mmm=0 ... ppp=26 (solver/lbm3d/defs.h:215-247);
 *                   values are the post-collision populations of the last completed step,
 *                   which is what the reference holds in df_out (core.h:798).
 */
#ifndef NNLBM_H
#define NNLBM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    NNLBM_OK = 0,
    NNLBM_ERR_ARG = -1,     /* invalid argument, label, size or state */
    NNLBM_ERR_CUDA = -2,    /* a CUDA runtime call failed */
    NNLBM_ERR_NAN = -3,     /* the device watchdog saw a non-finite or out-of-range density */
    NNLBM_ERR_TIMEOUT = -4, /* a bounded device wait gave up: the staged step form waited too
                               long (2 s) for its own bulk copies into shared memory; the
                               states of the context are then undefined */
    NNLBM_ERR_OOM = -5,     /* device allocation failed */
    NNLBM_ERR_AREA = -6     /* zero inlet or outlet area after the TCPC boundary setup */
} nnlbm_status;

/* storage type of the populations; arithmetic is FP32 for F32/F16/BF16 and FP64 for F64 */
enum { NNLBM_F64 = 0, NNLBM_F32 = 1, NNLBM_F16 = 2, NNLBM_BF16 = 3 };

/* collision selector; the names are the reference's id strings (lbm_col_*.h) */
enum {
    NNLBM_COL_CUM = 0,                                                    /* lbm_col_cum.h:11 */
    NNLBM_COL_KBC_N1 = 1, NNLBM_COL_KBC_N2, NNLBM_COL_KBC_N3, NNLBM_COL_KBC_N4, /* lbm_col_kbc_n.h */
    NNLBM_COL_KBC_C1 = 5, NNLBM_COL_KBC_C2, NNLBM_COL_KBC_C3, NNLBM_COL_KBC_C4, /* lbm_col_kbc_c.h */
    NNLBM_COL_MRT_LES = 9,                                                /* lbm_col_mrt.h:11 */
    NNLBM_COL_BGK = 10                                                    /* lbm_col_bgk.h:13 */
};

/* equilibrium used at boundary nodes and for the initial state */
enum {
    NNLBM_EQ_INV_CUM_REF = 0, /* LBM_EQ_INV_CUM as shipped (feq_pmm carries rho twice, lbm_eq_inv_cum.h:49) */
    NNLBM_EQ_INV_CUM = 1,     /* the same factorised equilibrium, corrected */
    NNLBM_EQ_DEFAULT = 2,     /* LBM_EQ_DEFAULT, lbm_eq.h:7-48 */
    NNLBM_EQ_ENTROPIC = 3     /* LBM_EQ_ENTROPIC, lbm_eq_entropic.h:141-176 */
};

/* Carreau-Yasuda coupling */
enum {
    NNLBM_CY_NONE = 0,     /* Newtonian collision viscosity (also the single-rank reference, whose strain field stays 0) */
    NNLBM_CY_REF_FD = 1,   /* the reference's multi-rank finite-difference force, core.h:273-800 and :1169-1310 */
    NNLBM_CY_LOCAL_NEQ = 2 /* local viscosity from the non-equilibrium second moments */
};

/* solver map labels: 0..6 are LBM_BC_Tcpc::GEO (sim_tcpc.cu:194-203); 7 and 8 are the
 * generic GEO_INFLOW and GEO_OUTFLOW_RIGHT_EQ blocks (solver/lbm3d/lbm_bc.h:126-152) */
enum {
    NNLBM_FLUID = 0, NNLBM_WALL = 1, NNLBM_PERIODIC = 2, NNLBM_INFLOW_LEFT = 3,
    NNLBM_INFLOW_RIGHT = 4, NNLBM_OUTFLOW_FRONT = 5, NNLBM_OUTFLOW_BACK = 6,
    NNLBM_INFLOW_EQ = 7, NNLBM_OUTFLOW_RIGHT_EQ = 8
};

/* macro fields for nnlbm_get_macro (MacroTcpc, sim_tcpc.cu:328-335; the mean/rms
 * accumulators are returned by nnlbm_get_stats) */
enum {
    NNLBM_M_RHO = 0, NNLBM_M_VX = 1, NNLBM_M_VY = 2, NNLBM_M_VZ = 3,
    NNLBM_M_FX = 4, NNLBM_M_FY = 5, NNLBM_M_FZ = 6,
    NNLBM_M_S11 = 7, NNLBM_M_S12 = 8, NNLBM_M_S13 = 9, NNLBM_M_S22 = 10, NNLBM_M_S32 = 11, NNLBM_M_S33 = 12,
    NNLBM_M_N = 13
};

/* per-step work flags (nnlbm_step_ex) */
enum {
    NNLBM_STEP_STATS = 1, /* accumulate the mean/rms sums (MacroTcpc::outputMacro, sim_tcpc.cu:347-353) */
    NNLBM_STEP_MACRO = 2, /* store rho, u, F and S of every cell */
    NNLBM_STEP_REDUCE = 4, /* FP64 mass and plane-flux sums (nnlbm_reduce) */
    NNLBM_STEP_ASYNC = 8,  /* enqueue the steps and return without waiting; the watchdog is
                              checked by the next nnlbm_sync or synchronous nnlbm_step */
    NNLBM_STEP_READBACK = 16 /* with NNLBM_STEP_ASYNC only: after the steps, also enqueue a copy of
                              the context's status block (step cursors, watchdog flags, the FP64
                              sums of NNLBM_STEP_REDUCE) into the next of NNLBM_READBACK_SLOTS
                              mapped pinned host slots, for nnlbm_readback.  A one-block kernel
                              in the context's stream writes the slot (NNLBM_READBACK_COPY=1 in
                              the environment at nnlbm_create: a device-to-host copy instead) */
};
#define NNLBM_READBACK_SLOTS 4

/* One lattice (case).  Physical inputs are already in lattice units; the unit conversions
 * of sim_tcpc.cu:795-814 live in the Python host layer. */
typedef struct {
    int32_t nx, ny, nz;
    int32_t dtype;       /* NNLBM_F64 / F32 / F16 / BF16 */
    int32_t collision;   /* NNLBM_COL_* */
    int32_t equilibrium; /* NNLBM_EQ_* */
    int32_t cy_mode;     /* NNLBM_CY_* */
    int32_t stats_f64;   /* 1: FP64 mean/rms accumulators, 0: FP32 (the reference's dreal) */
    double nu;           /* lattice viscosity; nu_inf when Carreau-Yasuda is on */
    double cy_nu0, cy_lambda, cy_a, cy_n; /* Carreau-Yasuda, lattice units */
    double fx, fy, fz;   /* homogeneous body force */
    double storage_scale; /* multiplier of the shifted populations f-w in F16/BF16 storage; 0 = default */
    int32_t bounce_back; /* NNLBM_BB_* */
    int32_t reserved;    /* 0 */
} nnlbm_case_desc;

/* wall treatment (nnlbm_case_desc.bounce_back) */
enum {
    NNLBM_BB_FULLWAY = 0, /* wall nodes: a wall cell returns the reversed populations it pulled, two steps
                             after they left (the reference's only wall, lbm_streaming.h:78-107) */
    NNLBM_BB_HALFWAY = 1  /* link-wise: a population that would come from a wall cell is the cell's own
                             post-collision population of the opposite direction of the previous
                             step, one step after it left; applies to every pull, the re-centred
                             stencils of the open planes included.  No reference counterpart. */
};

typedef struct nnlbm_ctx nnlbm_ctx;

/* Create a context of n_cases independent lattices on CUDA device `device`.
 * Replaces: State/LBM construction and device allocation (sim_tcpc.cu:808-810,
 * solver/lbm3d/lbm.hpp:308-372, core.h:1549). */
int nnlbm_create(const nnlbm_case_desc* desc, int n_cases, int device, nnlbm_ctx** out);

/* Replaces: the TNL host->device map copy after State::reset (core.h:1550,
 * solver/lbm3d/state.hpp:1857-1867).  map: [nz][ny][nx] solver labels. */
int nnlbm_set_map(nnlbm_ctx* ctx, int ic, const uint8_t* map);

/* Replaces: StateTcpc::setupBoundaries + LBM::projectWall (sim_tcpc.cu:494-645,
 * lbm.hpp:144-155).  wall: geometry cell array [nz][ny][nx] (0 fluid, 1 wall, 3..6 caps).
 * counts (10, may be NULL): left, right, outlet5, outlet6, wall, fluid, vtk3..vtk6.
 * Returns NNLBM_ERR_AREA where the reference sets `terminate` (sim_tcpc.cu:633-640). */
int nnlbm_setup_tcpc(nnlbm_ctx* ctx, int ic, const int32_t* wall, int64_t* counts);

/* The same boundary setup without a context or a device (host only): map_out [nz][ny][nx]
 * solver labels, wall_flags_out (may be NULL) the wall flags after the planes were opened
 * (LBM::getWall, read by the output's near-wall test, sim_tcpc.cu:709-714), counts as
 * above. */
int nnlbm_tcpc_labels(int32_t nx, int32_t ny, int32_t nz, const int32_t* wall, uint8_t* map_out,
                      uint8_t* wall_flags_out, int64_t* counts);

/* Replaces: resetLattice / setEqLat + LBMKernelInit (sim_tcpc.cu:647-655,
 * lbm.hpp:1-39, core.h:833-863). */
int nnlbm_init_equilibrium(nnlbm_ctx* ctx, int ic, double rho, double ux, double uy, double uz);

/* Replaces: updateKernelVelocities (sim_tcpc.cu:657-663) with LBM_Data_Tcpc
 * (sim_tcpc.cu:288-309): lattice-unit IVC/SVC fluxes (plug velocity = flux / area) and the
 * densities handed to the inflow planes; rho_eq is the density of NNLBM_INFLOW_EQ cells. */
int nnlbm_set_inflow(nnlbm_ctx* ctx, int ic, double ivc_flux, double svc_flux,
                     double rho_left, double rho_right, double rho_eq);

/* Per-cell velocity of the NNLBM_INFLOW_EQ cells, [n][3] in cell order; the LBM_DATA
 * inflow() hook of lbm_bc.h:127 (LBM_Data_ConstInflow, solver/lbm3d/lbm_data.h:352-367). */
int nnlbm_set_inflow_profile(nnlbm_ctx* ctx, int ic, const double* u, int64_t n);

/* Per-step inflow schedule for the next nnlbm_step call(s): rows of
 * {ivc_flux, svc_flux, profile_scale} (ramp, pulsation, noise).  n = 0 clears it. */
int nnlbm_set_schedule(nnlbm_ctx* ctx, int ic, const double* rows, int64_t n);

/* Advance every case by n_steps (CUDA-graph replayed).  Replaces the time loop of
 * execute (core.h:1566-1622) around SimUpdate (core.h:1025-1340).  flags: NNLBM_STEP_*,
 * applied to every step; NNLBM_STEP_MACRO and NNLBM_STEP_REDUCE apply to the last step. */
int nnlbm_step(nnlbm_ctx* ctx, int64_t n_steps, int flags);

/* Size of the one scratch array that nnlbm_step_noalloc uses on each device: the step
 * cursors of up to 64 launch groups (1 KiB) plus, per launch group, four values (rho, ux, uy,
 * uz) of the arithmetic type for each open-plane node that its own thread writes
 * (nnlbm_step_info's bc_cells bounds that count).  4 MiB holds 262,080 such nodes in FP32
 * arithmetic and 131,040 in FP64. */
#define NNLBM_NOALLOC_SCRATCH_BYTES (4u << 20)

/* nnlbm_step that allocates no device memory.  No counterpart in the reference (its
 * sim_tcpc allocates every buffer at start-up and owns the whole device).
 *
 * It is meant for callers that cannot allocate while they step: a host loop that shares
 * the GPU with work on other streams (cudaMalloc and cudaFree synchronise the device and
 * would stall that work), and a coupled solver that reserved its HBM budget up front and
 * must not meet an out-of-memory error in the middle of a run.
 *
 * Same kernels, arguments and results as nnlbm_step, run as plain launches (no CUDA
 * graph).  The per-call scratch of nnlbm_step (the step cursors and the gathered
 * open-plane node values) lives instead in one file-scope device array of
 * NNLBM_NOALLOC_SCRATCH_BYTES per device, which the library holds until the process exits.
 * nnlbm_create looks its address up (cudaGetSymbolAddress, with the device current) and loads
 * the code of every kernel the context can launch, so that neither happens, with the device
 * memory it takes, inside this call under CUDA's lazy module loading.  Every call shares the
 * array: the cursors are cleared at the start of each call (the node values are written
 * before they are read in every step and need no clearing), and calls that overlap in time,
 * from two contexts on one device or from two host threads, race on it.  With
 * NNLBM_STEP_ASYNC the call returns once the steps are enqueued and nnlbm_sync checks them,
 * as for nnlbm_step; the control rows are still copied from the host before it returns.
 *
 * It returns NNLBM_ERR_ARG, with a message, and launches nothing when a buffer would
 * have to be allocated first: a launch group whose work lists are not on the device yet
 * (call nnlbm_step or nnlbm_step_info once after nnlbm_set_map / nnlbm_setup_tcpc),
 * NNLBM_STEP_MACRO or NNLBM_STEP_STATS (or NNLBM_CY_REF_FD) before any nnlbm_step with
 * that flag, n_steps above the control rows in place (at least 1024), or more
 * open-plane nodes than the scratch array holds. */
int nnlbm_step_noalloc(nnlbm_ctx* ctx, int64_t n_steps, int flags);

/* Replaces: StateTcpc::statReset (sim_tcpc.cu:665-682). */
int nnlbm_stat_reset(nnlbm_ctx* ctx, int ic);

/* Macro field of the last step that had NNLBM_STEP_MACRO (before any such step: the
 * initial state of LBMKernelInit, core.h:833-863); out: [nz][ny][nx] doubles.
 * Replaces: LBM::copyMacroToHost (core.h:1334). */
int nnlbm_get_macro(nnlbm_ctx* ctx, int ic, int field, double* out);

/* Mean/rms sums: out [6][nz][ny][nx] = sum rho*ux, rho*uy, rho*uz, (rho*ux)^2, (rho*uy)^2,
 * (rho*uz)^2; *n_accumulated = steps summed since the last reset.  The reference keeps
 * rho*ux split by sign (sim_tcpc.cu:347-348) and only ever uses their sum (:724-725). */
int nnlbm_get_stats(nnlbm_ctx* ctx, int ic, double* out, int64_t* n_accumulated);

/* The VTK output fields of StateTcpc::outputData (sim_tcpc.cu:684-784), computed on the
 * device from the macro fields of the last step that had NNLBM_STEP_MACRO and the mean/rms
 * sums, in double, and stored as float (the type of the file's arrays).  Replaces the
 * per-cell outputData calls of State::writeVTK_3D_singlefile (state.hpp:782-851).
 * params[10] = {dx [m], dt [s], density [kg/m^3], lattice reference viscosity
 *               (dt/dx^2 * nu_inf), Carreau-Yasuda flag (0/1), lattice nu0, lattice lambda,
 *               a, n, steps summed in the mean/rms sums (at least 1 is used)}.
 * wall_flags: [nz][ny][nx] wall flags after the planes were opened (LBM::getWall, as returned
 * by nnlbm_tcpc_labels), read by the near-wall test of wss_proxy_pa; NULL = no walls.
 * out: [20][nz][ny][nx] floats in file order: velocity (3), mean_velocity (3), lbm_rho,
 * pressure_pa, gamma_dot, nu_phys_m2_s, mu_phys_pa_s, wss_proxy_pa, turbulence_intensity,
 * rms_velocity, strain_diag_1_s (3), strain_shear_1_s (3).  Allocates a device buffer of
 * 20 floats per cell for the call. */
int nnlbm_output_fields(nnlbm_ctx* ctx, int ic, const double* params, const uint8_t* wall_flags, float* out);

/* Canonical populations (see the layout note above).  Replaces: LBM::copyDFsToHost
 * (core.h:1584) and the df dumps of State::saveState (state.hpp:1552-1721). */
int nnlbm_export_df(nnlbm_ctx* ctx, int ic, double* out);
int nnlbm_import_df(nnlbm_ctx* ctx, int ic, const double* in);

/* Restore state saved by a checkpoint: the mean/rms sums in the layout of nnlbm_get_stats
 * with their step count, and every macro field ([NNLBM_M_N][nz][ny][nx], the order above;
 * CY_REF_FD steps read the previous step's velocity from it).  Replaces the hmacro reload of
 * State::loadState (state.hpp:1744-1756, saveAndLoadState :1552-1721). */
int nnlbm_import_stats(nnlbm_ctx* ctx, int ic, const double* in, int64_t n_accumulated);
int nnlbm_import_macro(nnlbm_ctx* ctx, int ic, const double* in);

/* FP64 sums of the last step that had NNLBM_STEP_REDUCE: {mass of FLUID+PERIODIC cells,
 * Q_ivc, Q_svc, Q_outlet5, Q_outlet6}, lattice units, inflow positive at 3/4 and outflow
 * positive at 5/6 (postprocess/compute_flows.py:107-147).  Right after a synchronous
 * nnlbm_step (or nnlbm_sync) the sums come from the host copy that call already made of the
 * context's status words, without another device transfer. */
int nnlbm_reduce(nnlbm_ctx* ctx, int ic, double* out5);

/* Time the launch shapes of the step kernel on copies of the current state and keep the
 * fastest: the block size, and for the single-precision cumulant, BGK and MRT whether a
 * thread steps two cells (packed FP32; plain or staged) or one.  The one- and two-cell
 * forms round differently, so contexts that must agree bitwise should share the form (the
 * default is two cells).
 * No reference counterpart (the reference takes --block-size, sim_tcpc.cu:118-119). */
int nnlbm_autotune(nnlbm_ctx* ctx);

/* nnlbm_autotune timing steps that carry `flags` (NNLBM_STEP_STATS, NNLBM_STEP_MACRO; the
 * others are ignored), for a caller that will step with them; the mean/rms sums and macro
 * fields are restored afterwards like the populations. */
int nnlbm_autotune_flags(nnlbm_ctx* ctx, int flags);

/* Set the step kernel's launch shape by hand for every launch group: `block` threads (64,
 * 128 or 256) and 1 or 2 cells a thread (2 applies to the single-precision cumulant, BGK
 * and MRT; the others step one).  2 | NNLBM_LAUNCH_STAGED selects the staged form of the
 * two-cell kernel: persistent warps that bring each pair of chunks into shared memory with
 * bulk copies while they collide the pair before (its block size is fixed at 128; its pairs
 * are bitwise those of the two-cell form).  Replaces --block-size (sim_tcpc.cu:118-119). */
#define NNLBM_LAUNCH_STAGED 16
int nnlbm_set_launch(nnlbm_ctx* ctx, int block, int cells_per_thread);

/* The launch shape case ic's launch group runs with now (after nnlbm_autotune or
 * nnlbm_set_launch): block size and cells a thread, as nnlbm_set_launch takes them. */
int nnlbm_get_launch(nnlbm_ctx* ctx, int ic, int* block, int* cells_per_thread);

/* Number of populations-kernel launches and bytes moved per step for case ic
 * (roofline bookkeeping). */
int nnlbm_step_info(nnlbm_ctx* ctx, int ic, int64_t* fluid_cells, int64_t* bc_cells,
                    int64_t* launches_per_step, double* bytes_per_step);

/* Run n_steps of case ic as individual launches with CUDA events around every kernel and
 * return the summed device milliseconds per kernel kind in ms[5] = {open-plane gather,
 * fused step, open-plane write, CY_REF_FD velocity, CY_REF_FD strain} and the launch counts
 * in launches[5].  The steps are real steps (the lattice advances).  No reference
 * counterpart (the reference logs wall-clock MLUPS, core.h:1440-1469). */
int nnlbm_profile_step(nnlbm_ctx* ctx, int ic, int64_t n_steps, int flags, double* ms, int64_t* launches);

/* Wait for every step enqueued on the context's stream and check the watchdog: returns
 * NNLBM_ERR_NAN if a density left (0.25, 4) or became non-finite.  The reference's step
 * loop synchronises the device after every SimUpdate (core.h:1197-1198, 1256-1257); with
 * NNLBM_STEP_ASYNC the caller chooses when. */
int nnlbm_sync(nnlbm_ctx* ctx);

/* Wait for the oldest status copy enqueued by NNLBM_STEP_READBACK, check its step cursors and
 * watchdog flags as nnlbm_sync does, and return its FP64 sums in the layout of nnlbm_reduce, 5
 * doubles per case in case order (`out` holds n_cases >= the context's cases).  Copies are
 * returned in the order the calls enqueued them; NNLBM_ERR_ARG when none is pending, and
 * nnlbm_step refuses NNLBM_STEP_READBACK while NNLBM_READBACK_SLOTS copies are pending.  A loop
 * that enqueues step k + 1 before it reads the sums of step k keeps the device busy while the
 * host waits for each copy.  No reference counterpart (the reference synchronises after every
 * step, core.h:1197-1198). */
int nnlbm_readback(nnlbm_ctx* ctx, double* out, int n_cases);

/* Raw CUDA stream (cudaStream_t) of the context, for callers that interleave their own work. */
void* nnlbm_stream(nnlbm_ctx* ctx);

/* Copy of the last error message; returns its full length. */
int nnlbm_last_error(nnlbm_ctx* ctx, char* buf, size_t n);

int nnlbm_destroy(nnlbm_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif
