// nnlbm_kernels.cuh -- storage traits, kernel arguments and the sm_100a kernels of one time
// step.
//
// Memory layout (HBM): one structure-of-arrays lattice per case, 27 direction arrays of
// nx*ny*nz elements each (x fastest), updated in place with the A-A pattern:
//   even step: cell x reads slot q at x (its incoming f_q) and writes its post-collision
//              f*_q to slot opp(q) at x;
//   odd step:  cell x reads slot opp(q) at x - c_q and writes f*_q to slot q at x + c_q.
// Each cell reads and writes the same 27 locations within a step, so the update is race
// free without a second lattice.  Indices that leave the box wrap around (periodic cells
// read across the faces; writes of face cells land where a periodic reader looks).
//
// Full-way bounce-back wall nodes (solver/lbm3d/lbm_streaming.h:78-107 used by
// solver/sim_tcpc/sim_tcpc.cu:235-241) need no work at all under A-A: their post-step
// value f*_q = incoming f_opp(q) already sits in the slot the neighbour reads next.
//
// Work decomposition: a packed list of 32-cell row chunks of colliding cells over all
// cases of a launch group (same storage type and collision), followed by warps of 32
// boundary nodes.  Three launch forms, picked by the host's autotuner: one warp per chunk
// (one cell a thread), one warp per two chunks (two cells a thread on the packed FP32 pipe,
// single-precision arithmetic only), and the staged form of the latter (persistent warps
// that bring their next pair into shared memory with tensor copies).  Per-case parameters
// live in a device array indexed by the chunk's case, and in parameter space for groups of
// up to 16 cases (case_args).
//
// Open-plane nodes (TCPC IVC/SVC inflow and outlets, generic GEO_OUTFLOW_RIGHT_EQ) pull a
// stencil re-centred one cell inward (sim_tcpc.cu:242-273, lbm_bc.h:147-152).  Where that
// inward cell collides and lies off every face, the stencil is the cell's own pull, so the
// cell's thread writes the node's equilibrium into the node's slots (serve_nodes).  For the
// other nodes k_bc_gather computes density / velocity from the pre-step state before the
// step kernel runs, and the node warps of the step kernel write each node's equilibrium
// into the node's own slots, which no other cell touches within the step.  GEO_INFLOW
// nodes take their prescribed velocity and need no gather.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "nnlbm_physics.cuh"

namespace nnlbm {

enum : int { L_FLUID = 0, L_WALL = 1, L_PERIODIC = 2, L_IN_L = 3, L_IN_R = 4, L_OUT_F = 5, L_OUT_B = 6,
             L_IN_EQ = 7, L_OUT_REQ = 8 };
// flag bit of the device label byte (the low four bits hold the label): a boundary node
// of the node list
enum : int { LF_SELF = 0x40, L_MASK = 0x0f };
enum : int { CY_NONE = 0, CY_REF_FD = 1, CY_LOCAL_NEQ = 2 };
enum : int { F_STATS = 1, F_MACRO = 2, F_REDUCE = 4 };
// macro field order of the context's macro array
enum : int { M_RHO = 0, M_VX, M_VY, M_VZ, M_FX, M_FY, M_FZ, M_S11, M_S12, M_S13, M_S22, M_S32, M_S33, M_N };

// ---------------------------------------------------------------------------------------
// storage: F64 holds f itself; F32/F16/BF16 hold the shifted value (f - w_q), times the
// per-lattice scale for the 16-bit types
// ---------------------------------------------------------------------------------------
template <int DT> struct Storage;
template <> struct Storage<0> {
    using T = double; using CT = double;
    __device__ static __forceinline__ CT from(T v, int, CT) { return v; }
    __device__ static __forceinline__ CT load(const T* p, int64_t i, int, CT) { return p[i]; }
    __device__ static __forceinline__ void store(T* p, int64_t i, int, CT v, CT) { p[i] = v; }
};
template <> struct Storage<1> {
    using T = float; using CT = float;
    __device__ static __forceinline__ CT from(T v, int q, CT) { return weight<float>(q) + v; }
    __device__ static __forceinline__ CT load(const T* p, int64_t i, int q, CT) { return weight<float>(q) + p[i]; }
    __device__ static __forceinline__ void store(T* p, int64_t i, int q, CT v, CT) { p[i] = v - weight<float>(q); }
};
template <> struct Storage<2> {
    using T = __half; using CT = float;
    __device__ static __forceinline__ CT from(T v, int q, CT isc) { return weight<float>(q) + __half2float(v) * isc; }
    __device__ static __forceinline__ CT load(const T* p, int64_t i, int q, CT isc) { return from(p[i], q, isc); }
    // (v - w) sc as one fused v sc - w sc (four distinct w sc per thread)
    __device__ static __forceinline__ void store(T* p, int64_t i, int q, CT v, CT sc) { p[i] = __float2half_rn(fmaf(v, sc, -(weight<float>(q) * sc))); }
};
template <> struct Storage<3> {
    using T = __nv_bfloat16; using CT = float;
    __device__ static __forceinline__ CT from(T v, int q, CT isc) { return weight<float>(q) + __bfloat162float(v) * isc; }
    __device__ static __forceinline__ CT load(const T* p, int64_t i, int q, CT isc) { return from(p[i], q, isc); }
    __device__ static __forceinline__ void store(T* p, int64_t i, int q, CT v, CT sc) { p[i] = __float2bfloat16_rn(fmaf(v, sc, -(weight<float>(q) * sc))); }
};

// per-step control row written by the host before each nnlbm_step call and indexed by a
// device cursor that the step kernel advances, so one captured graph replays any schedule
template <class CT>
struct StepCtl {
    int flags;
    int pad;
    CT u_left, u_right;   // plug velocities of the IVC / SVC planes (flux / area, SVC negative)
    CT rho_left, rho_right, rho_eq, prof_scale;
};

// everything a kernel needs to know about one case
template <class CT>
struct CaseArgs {
    void* df;                  // 27 direction arrays, qstride elements apart
    int64_t qstride;
    const uint8_t* label;      // [N] label | flag bits
    int nx, ny, nz, pad0;
    int64_t N;
    CT nu, nu0, lam, a, n;     // viscosity (nu_inf for CY) and Carreau-Yasuda parameters
    CT fx, fy, fz;             // homogeneous force
    CT scale, inv_scale;       // 16-bit storage scale
    int cy_mode, eq;
    CT* macro;                 // [M_N][N] or null
    void* stats;               // [6][N] (double or float) or null
    int stats_f64, pad1;
    const StepCtl<CT>* ctl;
    double* red;               // [kRedStripes][8]: stripes of {mass, Q_ivc, Q_svc, Q_out5, Q_out6}
    int* err;                  // watchdog flag
    // halfway bounce-back only (null otherwise): per cell, bit q set where cell x + c_q is a
    // WALL cell (neighbours wrap around the box like the A-A stores)
    const uint32_t* hw;
    // per-slot base addresses of a plain chunk's accesses, each the population array of one
    // slot already offset by the cell shift of the access, so that an address is one
    // shift-and-add of the cell index: slot q (even step, loads of slot q and stores of
    // slot opp(q)); slot q at +c_q (odd-step stores of direction q).  The odd-step load of
    // direction q, slot opp(q) at -c_q, is the store base of opp(q) (odd_ld), so the odd
    // step's 54 accesses use 27 base addresses, like the even step's
    const void* slot_even[27];
    const void* slot_odd_st[27];
    // the staged form's tensor maps of the population arrays (single-precision arithmetic
    // only): dims {qstride cells, 9, 3} over slot s = 9 * hi + lo, boxes of StageGeom::win
    // cells by {all 9 x all 3} (the even step's 27 slots of a chunk) and by {1 x all 3} (the
    // three slots of one (cy, cz) group in the odd step)
    CUtensorMap tm_even, tm_odd;
};

// the odd-step load base of direction q: slot opp(q) shifted by -c_q = +c_opp(q)
template <class CT>
__device__ __forceinline__ const void* odd_ld(const CaseArgs<CT>& a, int q)
{
    return a.slot_odd_st[26 - q];
}

// one 32-cell row chunk of the work list: the first cell, its row, the case and flags,
// and per lane (bit = lane) which cells collide and which of those are PERIODIC
struct alignas(16) Chunk {
    int c0, yz, cflags, pad0;
    unsigned fluid, periodic, pad1, pad2;
};
// per chunk (in a parallel array read only by serve_nodes): which lanes finish an open-plane
// node next to them, the node at x-1 (IN_L), at x+1 (IN_R, or OUT_REQ where the lane is in
// xreq too), at y-1 (OUT_F), at y+1 (OUT_B)
struct alignas(16) ChunkNodes {
    unsigned xneg, xpos, xreq, yneg, ypos, pad0, pad1, pad2;
};
// chunk flags (bits 16.. of cflags, the case index below).  CH_PLAIN: no neighbour of any
// colliding lane wraps around the box (the chunk is off the y/z faces and has no
// colliding cell at x = 0 or nx-1); CH_SRC: some lane finishes an open-plane node
enum : int { CH_CASE_MASK = 0xffff, CH_FLUID = 1 << 16, CH_FACE = 1 << 17, CH_PLAIN = 1 << 18, CH_SRC = 1 << 19,
             CH_HW = 1 << 20 };
// bits of a case's watchdog word: a density out of range (or not finite), a bounded wait of
// the staged step that gave up
enum : int { ERR_DENSITY = 1, ERR_STALL = 2 };
// CH_HW (halfway bounce-back): some colliding lane has a WALL neighbour; such chunks take the
// general path, whose odd step reads a population arriving from a wall from the cell's own
// slot q (where the previous, even, step left its f*_opp(q)) and stores a population leaving
// towards a wall into its own slot opp(q) (where the next, even, step reads it): each
// reflects one step after it left

// a launch group: cases sharing storage type and collision.  Up to kParamCases cases also
// travel in the kernel parameters (read through the constant cache, indexed by the
// chunk's case); larger groups read them from the device array.
constexpr int kParamCases = 16;
template <class CT>
struct GroupArgs {
    CaseArgs<CT> cp[kParamCases];  // copies of the first kParamCases cases in parameter space
    int n_cases, pad2;
    const CaseArgs<CT>* cases;
    const Chunk* chunks;
    const ChunkNodes* chunk_nodes;  // [n_chunks]
    int n_chunks, pad0;
    const int4* gather;        // {cell, case, node index, label} of the open-plane nodes
    int n_gather, n_nodes;
    const int2* nodes;         // [n_nodes] {cell, case} of every boundary node (open planes, INFLOW_EQ)
    const CT* bc_prof;         // [n_nodes][3] prescribed velocity (GEO_INFLOW nodes)
    CT* bc_buf;                // [n_nodes][4] gathered rho, ux, uy, uz
    // step cursors into every case's ctl, one per A-A parity: a step of parity p reads
    // cursor[p] and stores cursor[p] + 1 into cursor[1 - p], which no kernel of the step
    // reads, so no launch needs a grid-wide count
    int* cursor;
    // the staged form's wait on its bulk copies gives up after stage_wait_ns and reports
    // ERR_STALL; stage_pad (0 in a run) is added to the bytes each wait expects, so that a
    // test can make every wait run out with all copies complete
    long long stage_wait_ns;
    int stage_pad, pad3;
};

// where a kernel finds the arguments of case ci: the device array, the parameters indexed
// by the case, or, for a one-case group, the parameters' first entry at fixed offsets (read
// as constant operands, with no indexed constant loads)
enum : int { ARGS_GLOBAL = 0, ARGS_PARAM = 1, ARGS_ONE = 2 };
template <int ARGS, class CT>
__device__ __forceinline__ const CaseArgs<CT>& case_args(const GroupArgs<CT>& g, int ci)
{
    return ARGS == ARGS_ONE ? g.cp[0] : ARGS == ARGS_PARAM ? g.cp[ci] : g.cases[ci];
}
// the launch's choice for a group of n cases
__host__ __device__ constexpr int args_mode(int n_cases)
{
    return n_cases == 1 ? ARGS_ONE : n_cases <= kParamCases ? ARGS_PARAM : ARGS_GLOBAL;
}

// programmatic dependent launch (sm_90+): the open-plane gather lets the step kernel of the
// same step start at once; the step kernel waits for the gather's completion (and its
// memory) only before its first population store and before reading the gathered values.
// Without the launch attribute the wait returns at once.
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <int DT>
__device__ __forceinline__ typename Storage<DT>::T* qptr(const CaseArgs<typename Storage<DT>::CT>& a, int q)
{
    return (typename Storage<DT>::T*)a.df + (int64_t)q * a.qstride;
}

__device__ __forceinline__ int wrapc(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

// the FP64 reductions of a case land in kRedStripes stripes of 8 doubles (64 bytes apart),
// picked by warp or node index, so that thousands of warps do not serialise on one
// address in L2; the host adds the stripes up when it reads the sums
constexpr int kRedStripes = 32;
__device__ __forceinline__ double* red_stripe(double* red, int i) { return red + 8 * (i & (kRedStripes - 1)); }
__device__ __forceinline__ int global_warp() { return (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); }

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <class CT>
__device__ __forceinline__ void accumulate_stats(const CaseArgs<CT>& a, int c, CT rho, CT ux, CT uy, CT uz)
{
    // MacroTcpc::outputMacro (sim_tcpc.cu:347-353); the sign split of rho*ux is summed
    const CT jx = rho * ux, jy = rho * uy, jz = rho * uz;
    const int64_t N = a.N;
    // one contribution per cell and step: fire-and-forget reductions in L2 give the same
    // sums as a read-modify-write without exposing the read latency
    if (a.stats_f64) {
        double* s = (double*)a.stats;
        atomicAdd(s + c, (double)jx); atomicAdd(s + N + c, (double)jy); atomicAdd(s + 2 * N + c, (double)jz);
        atomicAdd(s + 3 * N + c, (double)jx * (double)jx); atomicAdd(s + 4 * N + c, (double)jy * (double)jy);
        atomicAdd(s + 5 * N + c, (double)jz * (double)jz);
    } else {
        float* s = (float*)a.stats;
        atomicAdd(s + c, (float)jx); atomicAdd(s + N + c, (float)jy); atomicAdd(s + 2 * N + c, (float)jz);
        atomicAdd(s + 3 * N + c, (float)(jx * jx)); atomicAdd(s + 4 * N + c, (float)(jy * jy));
        atomicAdd(s + 5 * N + c, (float)(jz * jz));
    }
}

template <class CT>
__device__ __forceinline__ void write_macro(const CaseArgs<CT>& a, int c, CT rho, CT ux, CT uy, CT uz, CT fx, CT fy, CT fz)
{
    CT* M = a.macro;
    const int64_t N = a.N;
    M[M_RHO * N + c] = rho; M[M_VX * N + c] = ux; M[M_VY * N + c] = uy; M[M_VZ * N + c] = uz;
    M[M_FX * N + c] = fx; M[M_FY * N + c] = fy; M[M_FZ * N + c] = fz;
}

// Carreau-Yasuda viscosity of the reference's finite-difference coupling (core.h:763-766),
// evaluated in single precision as the reference's powf does; in FP64 builds the power is
// taken in double and rounded once so that the value is the correctly rounded float
template <class CT>
__device__ __forceinline__ CT ref_cy_nu(CT nu, CT nu0, CT gam, CT lam, CT a, CT n);
template <>
__device__ __forceinline__ float ref_cy_nu<float>(float nu, float nu0, float gam, float lam, float a, float n)
{
    return nu + (nu0 - nu) * powf(1.0f + powf(gam * lam, a), (n - 1.0f) / a);
}
template <>
__device__ __forceinline__ double ref_cy_nu<double>(double nu, double nu0, double gam, double lam, double a, double n)
{
    const float inner = (float)pow((double)(float)(gam * lam), (double)(float)a);
    const float outer = (float)pow((double)(float)(1.0 + (double)inner), (double)(float)((n - 1.0) / a));
    return nu + (nu0 - nu) * (double)outer;
}

// write the equilibrium of an open-plane node into its own slots (A-A layout of this step)
template <int DT, bool ODD>
__device__ __forceinline__ void store_node_eq(const CaseArgs<typename Storage<DT>::CT>& a, int c, int x, int y, int z,
                                              typename Storage<DT>::CT rho, typename Storage<DT>::CT ux,
                                              typename Storage<DT>::CT uy, typename Storage<DT>::CT uz)
{
    using S = Storage<DT>;
    using CT = typename S::CT;
    CT f[27];
    equilibrium<CT>(a.eq, rho, ux, uy, uz, f);
    const int sy = a.nx, sz = a.nx * a.ny;
    if (!ODD) {
#pragma unroll
        for (int q = 0; q < 27; ++q) S::store(qptr<DT>(a, oppq(q)), c, q, f[q], a.scale);
    } else {
        // with halfway bounce-back a population headed into a wall stays in the node's slot opp(q)
        const uint32_t hwm = a.hw ? a.hw[c] : 0u;
#pragma unroll
        for (int q = 0; q < 27; ++q) {
            if ((hwm >> q) & 1u) S::store(qptr<DT>(a, oppq(q)), c, q, f[q], a.scale);
            else S::store(qptr<DT>(a, q), wrapc(x + cxq(q), a.nx) + sy * wrapc(y + cyq(q), a.ny) + sz * wrapc(z + czq(q), a.nz),
                          q, f[q], a.scale);
        }
    }
}

// macro / stats bookkeeping of an open-plane node; returns its contribution to the plane
// flux sums of postprocess/compute_flows.py:107-147 (inflow positive at 3/4)
template <class CT>
__device__ __forceinline__ double node_outputs(const CaseArgs<CT>& a, int flags, int lab, int c, CT rho, CT ux, CT uy, CT uz)
{
    if ((flags & F_MACRO) || a.cy_mode == CY_REF_FD) write_macro<CT>(a, c, rho, ux, uy, uz, a.fx, a.fy, a.fz);
    if (flags & F_STATS) accumulate_stats<CT>(a, c, rho, ux, uy, uz);
    return lab == L_IN_L ? (double)ux : lab == L_IN_R ? -(double)ux : lab == L_OUT_F ? -(double)uy : lab == L_OUT_B ? (double)uy : 0.0;
}

// Open-plane nodes finished by their inward neighbour.  A node's re-centred stencil
// (sim_tcpc.cu:242-273, lbm_bc.h:147-152) pulls the populations of the step around the cell
// one plane inward; where that cell collides and none of its neighbours wraps or is
// clamped, this is exactly the pull of that cell itself, and in the A-A layout every slot
// the stencil reads is read and overwritten by that cell alone within the step.  So the
// cell's own pre-collision density and velocity are the node's gathered values: after the
// chunk's cells have stored, the node's equilibrium goes into the node's slots (which no
// other cell touches within the step) with the node's outputs, and no separate gather, with
// its wait before the first store, is needed.  The chunk's lane masks say which nodes its
// lanes finish.  Where few lanes serve (an inlet row has one), the whole warp writes each
// node, lane q storing population q; where many serve (an outlet row), each lane writes its
// own.

// the chunks that serve nodes are few; their node code stays out of line unless the build
// asks otherwise
#ifndef NNLBM_SERVE_INLINE
#define NNLBM_SERVE_INLINE __noinline__
#endif

// the node of serving lane direction d (0: x-1, 1: x+1, 2: y-1, 3: y+1) and its label
__device__ __forceinline__ int served_label(int d, bool req)
{
    return d == 0 ? L_IN_L : d == 1 ? (req ? L_OUT_REQ : L_IN_R) : d == 2 ? L_OUT_F : L_OUT_B;
}

// density and velocity of a served node from its inward cell's (sim_tcpc.cu:242-273,
// lbm_bc.h:147-152): the inflow planes take the cell's density and the plug velocity, the
// outlets rho = 1 and the cell's velocity
template <class CT>
__device__ __forceinline__ void served_state(int lab, CT rho, CT ux, CT uy, CT uz, const StepCtl<CT>& ctl, CT& r, CT& u, CT& v,
                                             CT& w)
{
    if (lab == L_IN_L || lab == L_IN_R) {
        r = rho; u = lab == L_IN_L ? ctl.u_left : ctl.u_right; v = CT(0); w = CT(0);
    } else {
        r = CT(1); u = ux; v = uy; w = uz;
    }
}

// element offset, from the slot base of this step's store of population q, of node n at
// (xn, yn, zn): the cell itself in the even step; x + c_q wrapped around the box in the odd
// step, from a base already shifted by c_q (slot_odd_st)
__device__ __forceinline__ int node_wrap(int xn, int yn, int zn, int q, int nx, int ny, int nz)
{
    const int x = xn + cxq(q), y = yn + cyq(q), z = zn + czq(q);
    return (x < 0 ? nx : x >= nx ? -nx : 0) + nx * ((y < 0 ? ny : y >= ny ? -ny : 0) + ny * (z < 0 ? nz : z >= nz ? -nz : 0));
}

// the node's macro / stats / flux outputs (by one lane)
template <class CT>
__device__ __forceinline__ void served_outputs(const CaseArgs<CT>& a, int flags, int lab, int n, CT r, CT u, CT v, CT w)
{
    const double qn = node_outputs<CT>(a, flags, lab, n, r, u, v, w);
    if ((flags & F_REDUCE) && qn != 0.0) {
        const int slot = lab == L_IN_L ? 1 : lab == L_IN_R ? 2 : lab == L_OUT_F ? 3 : lab == L_OUT_B ? 4 : 0;
        if (slot) atomicAdd(red_stripe(a.red, n) + slot, qn);
    }
}

// called by the whole warp of a chunk with serving lanes (CH_SRC), after its stores; rho and
// u are each lane's pre-collision values
template <int DT, bool ODD>
__device__ NNLBM_SERVE_INLINE void serve_nodes(const CaseArgs<typename Storage<DT>::CT>* ap, const Chunk* chp,
                                               const ChunkNodes* cnp, int lane, typename Storage<DT>::CT rho,
                                               typename Storage<DT>::CT ux, typename Storage<DT>::CT uy,
                                               typename Storage<DT>::CT uz, int step, int flags)
{
    using S = Storage<DT>;
    using T = typename S::T;
    using CT = typename S::CT;
    const CaseArgs<CT>& a = *ap;
    // the records are read here rather than kept in registers through the collision
    const int c0 = chp->c0, yz = chp->yz;
    const unsigned xneg = cnp->xneg, xpos = cnp->xpos, xreq = cnp->xreq, yneg = cnp->yneg, ypos = cnp->ypos;
    const int y = yz & 0xffff, z = yz >> 16;
    const int sy = a.nx, x0 = c0 - y * sy - z * sy * a.ny;
    const StepCtl<CT>& ctl = a.ctl[step];
    const unsigned masks[4] = {xneg, xpos, yneg, ypos};
    const unsigned src = xneg | xpos | yneg | ypos;
    if (__popc(src) > 4) {
        // many serving lanes: each writes its own nodes
        const unsigned bit = 1u << lane;
        for (int d = 0; d < 4; ++d) {
            if (!(masks[d] & bit)) continue;
            const int lab = served_label(d, (xreq & bit) != 0);
            const int xn = x0 + lane - (d == 0) + (d == 1), yn = y - (d == 2) + (d == 3);
            const int n = c0 + lane + (d == 0 ? -1 : d == 1 ? 1 : d == 2 ? -sy : sy);
            CT r, u, v, w;
            served_state<CT>(lab, rho, ux, uy, uz, ctl, r, u, v, w);
            CT f[27];
            equilibrium<CT>(a.eq, r, u, v, w, f);
            const uint32_t hwm = (ODD && a.hw) ? a.hw[n] : 0u; // halfway: populations headed into a wall stay
#pragma unroll
            for (int q = 0; q < 27; ++q) {
                if (!ODD || ((hwm >> q) & 1u)) S::store((T*)a.slot_even[oppq(q)], n, q, f[q], a.scale);
                else S::store((T*)a.slot_odd_st[q], n + node_wrap(xn, yn, z, q, a.nx, a.ny, a.nz), q, f[q], a.scale);
            }
            served_outputs<CT>(a, flags, lab, n, r, u, v, w);
        }
        return;
    }
    // few serving lanes: the warp writes each node, lane q population q
    for (unsigned todo = src; todo; todo &= todo - 1) {
        const int s = __ffs(todo) - 1;
        const CT rs = __shfl_sync(0xffffffffu, rho, s), us = __shfl_sync(0xffffffffu, ux, s);
        const CT vs = __shfl_sync(0xffffffffu, uy, s), ws = __shfl_sync(0xffffffffu, uz, s);
        for (int d = 0; d < 4; ++d) {
            if (!((masks[d] >> s) & 1u)) continue;
            const int lab = served_label(d, ((xreq >> s) & 1u) != 0);
            const int xn = x0 + s - (d == 0) + (d == 1), yn = y - (d == 2) + (d == 3);
            const int n = c0 + s + (d == 0 ? -1 : d == 1 ? 1 : d == 2 ? -sy : sy);
            CT r, u, v, w;
            served_state<CT>(lab, rs, us, vs, ws, ctl, r, u, v, w);
            if (lane < 27) {
                const int q = lane;
                const CT fq = feq_one<CT>(a.eq, q, r, u, v, w);
                const bool stay = ODD && a.hw && ((a.hw[n] >> q) & 1u); // halfway: headed into a wall
                if (!ODD || stay) S::store((T*)a.slot_even[oppq(q)], n, q, fq, a.scale);
                else S::store((T*)a.slot_odd_st[q], n + node_wrap(xn, yn, z, q, a.nx, a.ny, a.nz), q, fq, a.scale);
            }
            if (lane == s) served_outputs<CT>(a, flags, lab, n, r, u, v, w);
        }
    }
}

// the finite-difference Carreau-Yasuda force of CY_REF_FD (core.h:663-781), kept out of
// line so that it takes no registers from the bulk path:
// divergence of the strain of the previous phase with one-sided differences next to
// non-FLUID cells, then 2 (nu(gamma) - nu) F rho with rho still at its default of 1
template <class CT>
__device__ __noinline__ void refd_force(const CaseArgs<CT>* ap, int c, int sy, int sz, CT* F)
{
    const CaseArgs<CT>& a = *ap;
    const CT* M = a.macro;
    const int64_t N = a.N;
    const int cn[6] = {c - 1, c + 1, c - sy, c + sy, c - sz, c + sz};
    bool fl[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) fl[k] = (a.label[cn[k]] & L_MASK) == L_FLUID;
    auto d1 = [&](int fld, int axis) -> CT {
        const bool m = fl[2 * axis], p = fl[2 * axis + 1];
        const CT* Fd = M + (int64_t)fld * N;
        if (!m) return p ? Fd[cn[2 * axis + 1]] - Fd[c] : CT(0);
        if (!p) return Fd[c] - Fd[cn[2 * axis]];
        return CT(0.5) * (Fd[cn[2 * axis + 1]] - Fd[cn[2 * axis]]);
    };
    const CT F1 = d1(M_S11, 0) + d1(M_S12, 1) + d1(M_S13, 2);
    const CT F2 = d1(M_S12, 0) + d1(M_S22, 1) + d1(M_S32, 2);
    const CT F3 = d1(M_S13, 0) + d1(M_S32, 1) + d1(M_S33, 2);
    const CT S11 = M[M_S11 * N + c], S12 = M[M_S12 * N + c], S13 = M[M_S13 * N + c];
    const CT S22 = M[M_S22 * N + c], S32 = M[M_S32 * N + c], S33 = M[M_S33 * N + c];
    const CT gam = dsqrt<CT>(CT(2)) * dsqrt<CT>(S11 * S11 + S22 * S22 + S33 * S33 + CT(2) * (S12 * S12 + S13 * S13 + S32 * S32));
    const CT nuc = ref_cy_nu<CT>(a.nu, a.nu0, gam, a.lam, a.a, a.n);
    F[0] += CT(2) * (nuc - a.nu) * F1;
    F[1] += CT(2) * (nuc - a.nu) * F2;
    F[2] += CT(2) * (nuc - a.nu) * F3;
}

// the step kernel of a (storage, collision) pairs its plain chunks when the arithmetic is
// single precision and the collision is the cumulant, BGK or MRT (KBC's moment sets need
// too many registers for two cells a thread).  The host pads each case's chunk list to
// an even length, so a pair never mixes two cases: a chunk meets the same partner, and
// the same arithmetic, whether its case runs alone or batched with others.
__host__ __device__ constexpr bool pairs_chunks(int dt, int col)
{
    return dt != 0 && (col == COL_CUM || col == COL_BGK || col == COL_MRT);
}

// register budget per thread of each step-kernel variant: FP64 arithmetic may use all
// 255; the paired form (two cells per thread) gets NNLBM_PAIR_REGS (two 256-thread blocks
// per SM); the one-cell form of a collision that can pair gets NNLBM_CHUNK_REGS_F32 with
// FP32 storage (80, the most that keeps three blocks: the step then spills almost nothing,
// which outweighs the lost warps) and
// NNLBM_CHUNK_REGS with FP16/BF16 storage (four blocks: the packed loads need fewer
// registers, and the extra warps hide the conversions); KBC, which never pairs, 128
#ifndef NNLBM_PAIR_REGS
#define NNLBM_PAIR_REGS 128
#endif
#ifndef NNLBM_KBC_REGS
#define NNLBM_KBC_REGS 128
#endif
#ifndef NNLBM_CHUNK_REGS
#define NNLBM_CHUNK_REGS 64
#endif
#ifndef NNLBM_CHUNK_REGS_F32
#define NNLBM_CHUNK_REGS_F32 80
#endif
// the one-cell cumulant runs packed columns (step_cell_cum_packed) with every
// single-precision storage type; with FP16/BF16 storage it gets NNLBM_CHUNK_REGS_CUM16
// registers (72: the packed pairs spill at 64, and 128-thread blocks keep 28 warps per SM)
#ifndef NNLBM_PACK_DT
#define NNLBM_PACK_DT(dt) ((dt) != 0)
#endif
#ifndef NNLBM_CHUNK_REGS_CUM16
#define NNLBM_CHUNK_REGS_CUM16 72
#endif
template <int DT, int COL, bool PAIR>
struct StepRegs {
    static constexpr int value = DT == 0                ? 255
                                 : !pairs_chunks(DT, COL) ? NNLBM_KBC_REGS
                                 : PAIR                   ? NNLBM_PAIR_REGS
                                 : DT == 1                ? NNLBM_CHUNK_REGS_F32
                                 : COL == COL_CUM         ? NNLBM_CHUNK_REGS_CUM16
                                                          : NNLBM_CHUNK_REGS;
};

// a 16-bit stored value as float, and a float rounded to the 16-bit storage type
template <int DT>
__device__ __forceinline__ float widen16(typename Storage<DT>::T v)
{
    if constexpr (DT == 2) return __half2float(v);
    else return __bfloat162float(v);
}
template <int DT>
__device__ __forceinline__ typename Storage<DT>::T narrow16(float v)
{
    if constexpr (DT == 2) return __float2half_rn(v);
    else return __float2bfloat16_rn(v);
}

// ---------------------------------------------------------------------------------------
// one 32-cell chunk of the fused step (solver/lbm3d/core.h:578-800), one warp, one cell per
// lane.  The populations go straight from HBM to registers, 27 coalesced row loads per
// warp, issued as soon as the chunk record is in (its lane masks say which lanes collide,
// so no label load sits in front of them).  On a plain chunk every address is the cell's
// pointer plus an offset made of the slot, row and plane strides only; the rare chunks on
// a face wrap their neighbour indices around the box.
// ---------------------------------------------------------------------------------------
template <int DT, int COL, bool ODD>
__device__ __forceinline__ void fluid_chunk(const CaseArgs<typename Storage<DT>::CT>& a, const CaseArgs<typename Storage<DT>::CT>* ap,
                                            const Chunk& ch, const Chunk* chp, const ChunkNodes* cnp, int step, int flags,
                                            int lane)
{
    using S = Storage<DT>;
    using T = typename S::T;
    using CT = typename S::CT;
    double mass = 0.0;
    const unsigned bit = 1u << lane;
    CT rho = CT(1), ux = CT(0), uy = CT(0), uz = CT(0);
    if (ch.fluid & bit) {
        const int c = ch.c0 + lane;
        const int64_t qs = a.qstride, sy = a.nx, sz = (int64_t)a.nx * a.ny;
        const bool plain = (ch.cflags & CH_PLAIN) != 0;
        // the wrapped neighbour cell x + sign c_q of a face chunk
        auto nbr = [&](int q, int sign) -> int64_t {
            const int y = ch.yz & 0xffff, z = ch.yz >> 16;
            const int x = ch.c0 - y * a.nx - z * a.nx * a.ny + lane;
            return (int64_t)wrapc(x + sign * cxq(q), a.nx) + sy * wrapc(y + sign * cyq(q), a.ny) +
                   sz * wrapc(z + sign * czq(q), a.nz) - c;
        };
        const T* pc = (const T*)a.df + c;
        // halfway bounce-back: which neighbours are walls (CH_HW chunks, odd step only)
        const uint32_t hwm = (ODD && (ch.cflags & CH_HW)) ? a.hw[c] : 0u;
        CT f[27];
        // PAIR16: 16-bit storage with BGK or MRT (measured +2 % each; the cumulant measured 3 %
        // slower): the
        // planes x = -1 and x = 0 scale and shift as packed pairs on the way in and out
        constexpr bool PAIR16 = DT >= 2 && (COL == COL_BGK || COL == COL_MRT);
        if constexpr (PAIR16) {
            if (!ODD || plain) {
                // slot q at c, or slot opp(q) at c - c_q
                auto src = [&](int q) { return (const T*)(ODD ? odd_ld(a, q) : a.slot_even[q]) + c; };
                const f2 isc2(a.inv_scale, a.inv_scale);
#pragma unroll
                for (int j = 0; j < 9; ++j) {
                    const f2 v = mad(f2(widen16<DT>(*src(j)), widen16<DT>(*src(9 + j))), isc2,
                                     f2(weight<float>(j), weight<float>(9 + j)));
                    f[j] = v.v.x;
                    f[9 + j] = v.v.y;
                }
#pragma unroll
                for (int q = 18; q < 27; ++q) f[q] = S::from(*src(q), q, a.inv_scale);
            }
        }
        if constexpr (PAIR16) {
            if (ODD && !plain) {
#pragma unroll
                for (int q = 0; q < 27; ++q)
                    f[q] = S::from(((hwm >> oppq(q)) & 1u) ? pc[q * qs] : pc[oppq(q) * qs + nbr(q, -1)], q, a.inv_scale);
            }
        } else if (!ODD) {
            // slot q at c
#pragma unroll
            for (int q = 0; q < 27; ++q) f[q] = S::from(((const T*)a.slot_even[q])[c], q, a.inv_scale);
        } else if (plain) {
            // slot opp(q) at c - c_q
#pragma unroll
            for (int q = 0; q < 27; ++q) f[q] = S::from(((const T*)odd_ld(a, q))[c], q, a.inv_scale);
        } else {
#pragma unroll
            for (int q = 0; q < 27; ++q)
                f[q] = S::from(((hwm >> oppq(q)) & 1u) ? pc[q * qs] : pc[oppq(q) * qs + nbr(q, -1)], q, a.inv_scale);
        }
        CT fx = a.fx, fy = a.fy, fz = a.fz;
        if (a.cy_mode == CY_REF_FD && !(ch.periodic & bit)) {
            CT F[3] = {fx, fy, fz};
            refd_force<CT>(ap, c, (int)sy, (int)sz, F);
            fx = F[0]; fy = F[1]; fz = F[2];
        }
        // one inlined collision for both viscosity models (the local Carreau-Yasuda law is
        // a runtime branch inside it)
        CT Sl[6];
        const CYParams<CT> cy = {a.nu, a.nu0, a.lam, a.a, a.n};
        step_cell<CT, COL, CT, NNLBM_PACK_DT(DT) ? DT : 0>(f, fx, fy, fz, a.nu, a.cy_mode == CY_LOCAL_NEQ ? &cy : nullptr, Sl, rho, ux, uy, uz);
        // the gather of this step reads the slots written below
        pdl_wait();
        T* ps = (T*)a.df + c;
        if constexpr (PAIR16) {
            if (!ODD || plain) {
                // slot opp(q) at c, or slot q at c + c_q
                auto dst = [&](int q) { return (T*)(ODD ? a.slot_odd_st[q] : a.slot_even[oppq(q)]) + c; };
                const f2 sc2(a.scale, a.scale);
#pragma unroll
                for (int j = 0; j < 9; ++j) {
                    const f2 v = mad(f2(f[j], f[9 + j]), sc2, f2(-(weight<float>(j) * a.scale), -(weight<float>(9 + j) * a.scale)));
                    *dst(j) = narrow16<DT>(v.v.x);
                    *dst(9 + j) = narrow16<DT>(v.v.y);
                }
#pragma unroll
                for (int q = 18; q < 27; ++q) S::store(dst(q), 0, q, f[q], a.scale);
            } else {
#pragma unroll
                for (int q = 0; q < 27; ++q)
                    S::store(ps, ((hwm >> q) & 1u) ? oppq(q) * qs : q * qs + nbr(q, 1), q, f[q], a.scale);
            }
        } else if (!ODD) {
            // slot opp(q) at c
#pragma unroll
            for (int q = 0; q < 27; ++q) S::store((T*)a.slot_even[oppq(q)], c, q, f[q], a.scale);
        } else if (plain) {
            // slot q at c + c_q
#pragma unroll
            for (int q = 0; q < 27; ++q) S::store((T*)a.slot_odd_st[q], c, q, f[q], a.scale);
        } else {
#pragma unroll
            for (int q = 0; q < 27; ++q) S::store(ps, ((hwm >> q) & 1u) ? oppq(q) * qs : q * qs + nbr(q, 1), q, f[q], a.scale);
        }
        if ((flags & F_MACRO) || a.cy_mode == CY_REF_FD) {
            write_macro<CT>(a, c, rho, ux, uy, uz, fx, fy, fz);
            if (a.cy_mode == CY_LOCAL_NEQ) {
#pragma unroll
                for (int k = 0; k < 6; ++k) a.macro[(int64_t)(M_S11 + k) * a.N + c] = Sl[k];
            }
        }
        if (flags & F_STATS) accumulate_stats<CT>(a, c, rho, ux, uy, uz);
        if (!(rho > CT(0.25) && rho < CT(4))) atomicOr(a.err, ERR_DENSITY);
        mass = (double)rho;
    }
    if (ch.cflags & CH_SRC) serve_nodes<DT, ODD>(ap, chp, cnp, lane, rho, ux, uy, uz, step, flags);
    if (flags & F_REDUCE) {
        const double s0 = warp_sum(mass);
        if (lane == 0 && s0 != 0.0) atomicAdd(red_stripe(a.red, global_warp()), s0);
    }
}

// ---------------------------------------------------------------------------------------
// two plain chunks of one case in one warp, one cell of each per lane, for the cumulant,
// BGK and MRT in single-precision arithmetic: the two cells' arithmetic runs as f2 on the packed
// FP32 pipe, so the pair issues about the FP32 instructions of one cell; loads, stores
// and the per-cell outputs stay per cell.  A lane whose cell in one chunk does not
// collide computes that half from the rest state and stores nothing for it.
// ---------------------------------------------------------------------------------------
// raw stored value <-> float of the single-precision storage types (no shift, no scale)
template <int DT> struct Cook;
template <> struct Cook<1> {
    __device__ static __forceinline__ float put(float v) { return v; }
    __device__ static __forceinline__ float get(float v) { return v; }
};
template <> struct Cook<2> {
    __device__ static __forceinline__ __half put(float v) { return __float2half_rn(v); }
    __device__ static __forceinline__ float get(__half v) { return __half2float(v); }
    __device__ static __forceinline__ unsigned short bits(__half v) { return __half_as_ushort(v); }
    __device__ static __forceinline__ float of_bits(unsigned short b) { return __half2float(__ushort_as_half(b)); }
};
template <> struct Cook<3> {
    __device__ static __forceinline__ __nv_bfloat16 put(float v) { return __float2bfloat16_rn(v); }
    __device__ static __forceinline__ float get(__nv_bfloat16 v) { return __bfloat162float(v); }
    __device__ static __forceinline__ unsigned short bits(__nv_bfloat16 v) { return __bfloat16_as_ushort(v); }
    __device__ static __forceinline__ float of_bits(unsigned short b) { return __bfloat162float(__ushort_as_bfloat16(b)); }
};

// predicated global loads (0 where `on` is false) and stores that stay one predicated
// instruction each: a branch around each would split the warp's batch of loads, and its
// stream of stores, into one piece per population
__device__ __forceinline__ float ld_if(const float* p, bool on)
{
    float v = 0.f;
    asm("{ .reg .pred q; setp.ne.b32 q, %2, 0; @q ld.global.f32 %0, [%1]; }" : "+f"(v) : "l"(p), "r"((int)on));
    return v;
}
__device__ __forceinline__ unsigned short ld_if(const unsigned short* p, bool on)
{
    unsigned short v = 0;
    asm("{ .reg .pred q; setp.ne.b32 q, %2, 0; @q ld.global.b16 %0, [%1]; }" : "+h"(v) : "l"(p), "r"((int)on));
    return v;
}
__device__ __forceinline__ void st_if(float* p, float v, bool on)
{
    asm volatile("{ .reg .pred q; setp.ne.b32 q, %2, 0; @q st.global.f32 [%0], %1; }" ::"l"(p), "f"(v), "r"((int)on)
                 : "memory");
}
__device__ __forceinline__ void st_if(float2* p, float2 v, bool on)
{
    asm volatile("{ .reg .pred q; setp.ne.b32 q, %3, 0; @q st.global.v2.f32 [%0], {%1, %2}; }" ::"l"(p), "f"(v.x),
                 "f"(v.y), "r"((int)on)
                 : "memory");
}
__device__ __forceinline__ void st_if(unsigned* p, unsigned v, bool on)
{
    asm volatile("{ .reg .pred q; setp.ne.b32 q, %2, 0; @q st.global.b32 [%0], %1; }" ::"l"(p), "r"(v), "r"((int)on)
                 : "memory");
}
__device__ __forceinline__ void st_if(unsigned short* p, unsigned short v, bool on)
{
    asm volatile("{ .reg .pred q; setp.ne.b32 q, %2, 0; @q st.global.b16 [%0], %1; }" ::"l"(p), "h"(v), "r"((int)on)
                 : "memory");
}

// one population of a pair half: load (the raw stored value as float, 0 where off) and store
template <int DT>
__device__ __forceinline__ float pair_get(const typename Storage<DT>::T* p, bool on)
{
    if constexpr (DT == 1) return ld_if(p, on);
    else return Cook<DT>::of_bits(ld_if((const unsigned short*)p, on));
}
template <int DT>
__device__ __forceinline__ void pair_put(typename Storage<DT>::T* p, float v, bool on)
{
    if constexpr (DT == 1) st_if(p, v, on);
    else st_if((unsigned short*)p, Cook<DT>::bits(Cook<DT>::put(v)), on);
}

// ---------------------------------------------------------------------------------------
// x-adjacent pairs: where a pair of chunks is one contiguous 64-cell row span whose cells
// all collide, lane l takes cells 2l and 2l+1, so that one 4-byte (FP16, BF16) or 8-byte
// (FP32) access moves a population of both and feeds the f2 pair with one conversion.
// ---------------------------------------------------------------------------------------
template <int DT> struct Pair2;
template <> struct Pair2<1> {
    __device__ static __forceinline__ f2 load(const float* e) { return f2(*(const float2*)e); }
    __device__ static __forceinline__ void store(float* e, f2 v) { *(float2*)e = v.v; }
};
template <> struct Pair2<2> {
    __device__ static __forceinline__ f2 of(unsigned w)
    {
        const __half2 h = *reinterpret_cast<const __half2*>(&w);
        return f2(__half22float2(h));
    }
    __device__ static __forceinline__ unsigned word(f2 v)
    {
        const __half2 h = __float22half2_rn(v.v);
        return *reinterpret_cast<const unsigned*>(&h);
    }
};
template <> struct Pair2<3> {
    __device__ static __forceinline__ f2 of(unsigned w)
    {
        const __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162*>(&w);
        return f2(__bfloat1622float2(h));
    }
    __device__ static __forceinline__ unsigned word(f2 v)
    {
        const __nv_bfloat162 h = __float22bfloat162_rn(v.v);
        return *reinterpret_cast<const unsigned*>(&h);
    }
};

// elements (e, e+1) of every lane, e = base + 2 lane.  The even step's pairs start at an even
// element and move as one 8-byte (FP32) or 4-byte (FP16, BF16) access.  The odd step's pairs
// are shifted by the neighbour offsets, whose parity depends on the box width, and move as
// their two elements (the warp's two accesses touch the same sectors): the access form is
// then fixed at compile time, no population waits behind a branch on its alignment, and the
// 27 loads issue as one batch
template <int DT, bool SPLIT>
__device__ __forceinline__ f2 load_adjacent(const typename Storage<DT>::T* e)
{
    if constexpr (DT == 1) {
        if constexpr (SPLIT) return f2(e[0], e[1]);
        else return Pair2<1>::load(e);
    } else {
        if constexpr (SPLIT) {
            const unsigned short* h = (const unsigned short*)e;
            return Pair2<DT>::of((unsigned)h[0] | ((unsigned)h[1] << 16));
        } else {
            return Pair2<DT>::of(*(const unsigned*)e);
        }
    }
}

template <int DT, bool SPLIT>
__device__ __forceinline__ void store_adjacent(typename Storage<DT>::T* e, f2 v)
{
    if constexpr (DT == 1) {
        if constexpr (SPLIT) {
            e[0] = v.v.x;
            e[1] = v.v.y;
        } else {
            Pair2<1>::store(e, v);
        }
    } else {
        const unsigned w = Pair2<DT>::word(v);
        if constexpr (SPLIT) {
            unsigned short* h = (unsigned short*)e;
            h[0] = (unsigned short)(w & 0xffffu);
            h[1] = (unsigned short)(w >> 16);
        } else {
            *(unsigned*)e = w;
        }
    }
}

// two chunks that are one contiguous 64-cell span of colliding cells with no node to serve
template <int DT>
__device__ __forceinline__ bool adjacent_span(const Chunk& ca, const Chunk& cb)
{
    return DT != 0 && (ca.fluid & cb.fluid) == 0xffffffffu && cb.c0 == ca.c0 + 32 && !(ca.c0 & 1) &&
           !((ca.cflags | cb.cflags) & CH_SRC);
}

template <int DT, bool ODD>
__device__ __forceinline__ void pair_load_adjacent(const CaseArgs<float>& a, int c0, int lane, f2* f)
{
    using T = typename Storage<DT>::T;
    const f2 isc(a.inv_scale);
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const void* p = ODD ? odd_ld(a, q) : a.slot_even[q];
        const f2 raw = load_adjacent<DT, ODD>((const T*)p + c0 + 2 * lane);
        const f2 w(weight<float>(q));
        f[q] = DT == 1 ? raw + w : mad(raw, isc, w);
    }
}

// the rest of a pair once its populations f (raw stored value + weight, or the rest state
// where the cell does not collide) are in registers: collision, stores, per-cell outputs.
// `adj`: an x-adjacent span (lane l holds cells c0 + 2l and c0 + 2l + 1)
template <int DT, int COL, bool ODD>
__device__ __forceinline__ void pair_finish(const CaseArgs<float>& a, const CaseArgs<float>* ap, const Chunk& ca,
                                            const Chunk& cb, const Chunk* cap, const ChunkNodes* cnp, f2* f, int step, int flags,
                                            int lane, bool adj)
{
    using T = typename Storage<DT>::T;
    const unsigned bit = 1u << lane;
    const bool fa = adj || (ca.fluid & bit) != 0, fb = adj || (cb.fluid & bit) != 0;
    double mass = 0.0;
    float r[2] = {1.f, 1.f}, u0[2] = {0.f, 0.f}, u1[2] = {0.f, 0.f}, u2[2] = {0.f, 0.f};
    if (fa || fb) {
        const int cA = adj ? ca.c0 + 2 * lane : ca.c0 + lane, cB = adj ? ca.c0 + 2 * lane + 1 : cb.c0 + lane;
        const f2 fx(a.fx), fy(a.fy), fz(a.fz);
        f2 rho, ux, uy, uz;
        f2 Sl[6];
        const CYParams<float> cy = {a.nu, a.nu0, a.lam, a.a, a.n};
        step_cell<f2, COL, float>(f, fx, fy, fz, f2(a.nu), a.cy_mode == CY_LOCAL_NEQ ? &cy : nullptr, Sl, rho, ux, uy, uz);
        // the gather of this step reads the slots written below
        pdl_wait();
        const f2 sc(a.scale);
#pragma unroll
        for (int q = 0; q < 27; ++q) {
            T* p = (T*)(ODD ? a.slot_odd_st[q] : a.slot_even[oppq(q)]);
            const f2 w(weight<float>(q));
            const f2 v = DT == 1 ? f[q] - w : mad(f[q], sc, -(w * sc));
            if (adj) {
                store_adjacent<DT, ODD>(p + cA, v);
            } else {
                pair_put<DT>(p + cA, v.v.x, fa);
                pair_put<DT>(p + cB, v.v.y, fb);
            }
        }
        r[0] = rho.v.x; r[1] = rho.v.y; u0[0] = ux.v.x; u0[1] = ux.v.y;
        u1[0] = uy.v.x; u1[1] = uy.v.y; u2[0] = uz.v.x; u2[1] = uz.v.y;
        const bool on[2] = {fa, fb};
        const int cc[2] = {cA, cB};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (!on[h]) continue;
            if (flags & F_MACRO) {
                write_macro<float>(a, cc[h], r[h], u0[h], u1[h], u2[h], a.fx, a.fy, a.fz);
                if (a.cy_mode == CY_LOCAL_NEQ) {
#pragma unroll
                    for (int k = 0; k < 6; ++k) a.macro[(int64_t)(M_S11 + k) * a.N + cc[h]] = h ? Sl[k].v.y : Sl[k].v.x;
                }
            }
            if (flags & F_STATS) accumulate_stats<float>(a, cc[h], r[h], u0[h], u1[h], u2[h]);
            if (!(r[h] > 0.25f && r[h] < 4.f)) atomicOr(a.err, ERR_DENSITY);
            mass += (double)r[h];
        }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        if ((h ? cb : ca).cflags & CH_SRC) serve_nodes<DT, ODD>(ap, cap + h, cnp + h, lane, r[h], u0[h], u1[h], u2[h], step, flags);
    }
    if (flags & F_REDUCE) {
        const double s0 = warp_sum(mass);
        if (lane == 0 && s0 != 0.0) atomicAdd(red_stripe(a.red, global_warp()), s0);
    }
}

// a pair's populations straight from HBM: the raw stored value + weight of each cell, or
// the rest state where the cell does not collide
template <int DT, bool ODD>
__device__ __forceinline__ void pair_load(const CaseArgs<float>& a, const Chunk& ca, const Chunk& cb, int lane, f2* f)
{
    using T = typename Storage<DT>::T;
    const unsigned bit = 1u << lane;
    const bool fa = (ca.fluid & bit) != 0, fb = (cb.fluid & bit) != 0;
    const int cA = ca.c0 + lane, cB = cb.c0 + lane;
    const f2 isc(a.inv_scale);
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const T* p = (const T*)(ODD ? odd_ld(a, q) : a.slot_even[q]);
        const f2 raw(pair_get<DT>(p + cA, fa), pair_get<DT>(p + cB, fb));
        const f2 w(weight<float>(q));
        f[q] = DT == 1 ? raw + w : mad(raw, isc, w);
    }
}

// two plain chunks of one case (no finite-difference force) collide as a pair
template <int ARGS>
__device__ __forceinline__ bool pairable(const GroupArgs<float>& g, const Chunk& ca, const Chunk& cb)
{
    const int ci = ca.cflags & CH_CASE_MASK;
    return ((ca.cflags & cb.cflags) & CH_PLAIN) && ci == (cb.cflags & CH_CASE_MASK) &&
           case_args<ARGS>(g, ci).cy_mode != CY_REF_FD;
}

// 32 boundary nodes (open-plane nodes and GEO_INFLOW nodes, one per lane): each writes
// the equilibrium of its gathered (rho, u) (or of its prescribed inflow) into its own
// slots, which no other cell reads or writes within the step, and adds its plane flux
template <int DT, bool ODD>
__device__ __noinline__ void node_batch(const int2* nodes, int n_nodes, const CaseArgs<typename Storage<DT>::CT>* cases,
                                        const typename Storage<DT>::CT* bc_prof, const typename Storage<DT>::CT* bc_buf, int k,
                                        int step, int flags)
{
    using CT = typename Storage<DT>::CT;
    pdl_wait(); // the gathered values
    if (k >= n_nodes) return;
    const int2 nd = nodes[k];
    const CaseArgs<CT>& a = cases[nd.y];
    const int c = nd.x;
    const int lab = a.label[c] & L_MASK;
    const int x = c % a.nx, y = (c / a.nx) % a.ny, z = c / (a.nx * a.ny);
    CT rho, ux, uy, uz;
    if (lab == L_IN_EQ) { // lbm_bc.h:126-129
        const StepCtl<CT>& ctl = a.ctl[step];
        rho = ctl.rho_eq;
        ux = bc_prof[3 * k] * ctl.prof_scale;
        uy = bc_prof[3 * k + 1] * ctl.prof_scale;
        uz = bc_prof[3 * k + 2] * ctl.prof_scale;
    } else {
        rho = bc_buf[4 * k]; ux = bc_buf[4 * k + 1]; uy = bc_buf[4 * k + 2]; uz = bc_buf[4 * k + 3];
    }
    store_node_eq<DT, ODD>(a, c, x, y, z, rho, ux, uy, uz);
    const double qn = node_outputs<CT>(a, flags, lab, c, rho, ux, uy, uz);
    if ((flags & F_REDUCE) && qn != 0.0) {
        const int slot = lab == L_IN_L ? 1 : lab == L_IN_R ? 2 : lab == L_OUT_F ? 3 : lab == L_OUT_B ? 4 : 0;
        if (slot) atomicAdd(red_stripe(a.red, k) + slot, qn);
    }
}

// the step kernel: one warp per chunk of the work list (per two chunks where the variant
// pairs them), then one warp per 32 boundary nodes.  Both write only the slots their own
// cells read, so they run side by side.
template <int DT, int COL, bool ODD, int ARGS, bool PAIR>
__global__ void __launch_bounds__(256) __maxnreg__((StepRegs<DT, COL, PAIR>::value))
    k_step(const __grid_constant__ GroupArgs<typename Storage<DT>::CT> g)
{
    using CT = typename Storage<DT>::CT;
    const int lane = threadIdx.x & 31;
    const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int step = g.cursor[ODD ? 1 : 0];
    if (blockIdx.x == 0 && threadIdx.x == 0) g.cursor[ODD ? 0 : 1] = step + 1;
    // the step's flags are the same for every case of the group
    const int flags = case_args<ARGS>(g, 0).ctl[step].flags;
    if constexpr (PAIR && pairs_chunks(DT, COL)) {
        // warp w takes chunks 2w and 2w + 1 (the host pads the list to an even length); a
        // pair that is not pairable (a face chunk, two cases, the finite-difference force)
        // is stepped chunk by chunk
        const int np = g.n_chunks >> 1;
        if (w < np) {
            const Chunk ca = g.chunks[2 * w], cb = g.chunks[2 * w + 1];
            const int ci = ca.cflags & CH_CASE_MASK;
            const CaseArgs<CT>& a = case_args<ARGS>(g, ci);
            if (pairable<ARGS>(g, ca, cb)) {
                f2 f[27];
                const bool adj = adjacent_span<DT>(ca, cb);
                if (adj) pair_load_adjacent<DT, ODD>(a, ca.c0, lane, f);
                else pair_load<DT, ODD>(a, ca, cb, lane, f);
                pair_finish<DT, COL, ODD>(a, g.cases + ci, ca, cb, g.chunks + 2 * w, g.chunk_nodes + 2 * w, f, step, flags, lane,
                                          adj);
            } else {
                fluid_chunk<DT, COL, ODD>(a, g.cases + ci, ca, g.chunks + 2 * w, g.chunk_nodes + 2 * w, step, flags, lane);
                if (cb.fluid) {
                    const int cj = cb.cflags & CH_CASE_MASK;
                    fluid_chunk<DT, COL, ODD>(case_args<ARGS>(g, cj), g.cases + cj, cb, g.chunks + 2 * w + 1,
                                              g.chunk_nodes + 2 * w + 1, step, flags, lane);
                }
            }
        } else {
            node_batch<DT, ODD>(g.nodes, g.n_nodes, g.cases, g.bc_prof, g.bc_buf, (w - np) * 32 + lane, step, flags);
        }
    } else {
        if (w < g.n_chunks) {
            const Chunk ch = g.chunks[w];
            const int ci = ch.cflags & CH_CASE_MASK;
            fluid_chunk<DT, COL, ODD>(case_args<ARGS>(g, ci), g.cases + ci, ch, g.chunks + w, g.chunk_nodes + w, step, flags, lane);
        } else {
            node_batch<DT, ODD>(g.nodes, g.n_nodes, g.cases, g.bc_prof, g.bc_buf, (w - g.n_chunks) * 32 + lane, step, flags);
        }
    }
}

// ---------------------------------------------------------------------------------------
// the staged paired form: persistent warps, each stepping pairs of chunks in turn, whose
// populations it has brought into shared memory with tensor copies (cp.async.bulk.tensor,
// completion counted in bytes on an mbarrier) while it collided the pair before.  Each
// warp owns two buffers and their barriers, so that no warp waits on another.  The loads
// leave the warp's critical path (the copy of pair k + 1 is in flight while pair k
// collides), and a population costs one or two shared-memory reads instead of a global load
// and its address arithmetic.  One lane issues the copies: per chunk, the even step's 27
// slots at the chunk's cells are one box; the odd step reads slot opp(q) at x - c_q, and the
// three directions of one (cy, cz) share a row and differ by one cell in x, so each of the
// nine (cy, cz) groups is one box a few cells wider than the chunk.  A box starts at the
// 16-byte boundary at or below its first cell; the reads index it from that offset.  A pair
// that is not pairable, and the boundary-node batches, take the unstaged paths.
// ---------------------------------------------------------------------------------------
template <int DT>
struct StageGeom {
    static constexpr int sz = (int)sizeof(typename Storage<DT>::T);
    static constexpr int align = 16 / sz;                        // cells per 16 bytes
    static constexpr int win = (32 + 2 + align - 1 + align - 1) / align * align; // box width: 40 (FP32), 48
    static constexpr int row = win * sz;                          // one slot's window: 160 or 96 bytes
    static constexpr int group = (3 * row + 127) / 128 * 128;     // an odd-step box, 128-byte aligned
    static constexpr int chunk = 9 * group;                       // a chunk's 27 windows (>= 27 rows)
    static constexpr int unit = 2 * chunk;                        // a pair
    static constexpr unsigned tx = 54u * row;                     // bytes the boxes of a pair bring
    static constexpr int warps = 4;                               // warps per block
    static constexpr int smem = warps * 2 * unit + 128;           // two buffers per warp, alignment slack
};
constexpr int kStagedThreads = 128;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
// the initialised barriers visible to the tensor-copy (async) proxy
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
// one box of a 3-d tensor map into shared memory (x: the cell coordinate, a multiple of
// 16 bytes; it may lie below zero or past the array, where the box reads zeros)
__device__ __forceinline__ void tensor_to_smem(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            smem_addr(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity)
{
    uint32_t ok;
    asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                 : "=r"(ok)
                 : "r"(smem_addr(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
// wait for the phase of `parity` to complete, for at most limit_ns (and at most 2^24 polls)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, long long limit_ns)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (int i = 0; i < (1 << 24); ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((long long)(global_ns() - t0) > limit_ns) break;
    }
    return false;
}

// the (cy, cz) of odd-step group lo (slot s = 9 hi + lo holds direction opp(s), whose
// c = (hi - 1, lo / 3 - 1, lo % 3 - 1) negated)
__device__ __forceinline__ int group_cy(int lo) { return 1 - lo / 3; }
__device__ __forceinline__ int group_cz(int lo) { return 1 - lo % 3; }
// the first cell of a chunk's window for odd-step group lo, before alignment: the source of
// its first cell for cx = +1
__device__ __forceinline__ int group_x0(const CaseArgs<float>& a, int c0, int lo)
{
    return c0 - group_cy(lo) * a.nx - group_cz(lo) * a.nx * a.ny - 1;
}

// one lane arms the barrier with the bytes of the pair and issues its boxes: one per chunk
// (even step) or nine per chunk (odd step)
template <int DT, bool ODD>
__device__ __forceinline__ void stage_pair(const CaseArgs<float>& a, int c0a, int c0b, int lane, char* buf, uint64_t* bar,
                                           int pad)
{
    using G = StageGeom<DT>;
    if (lane == 0) {
        mbar_expect_tx(bar, G::tx + (unsigned)pad);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int c0 = h ? c0b : c0a;
            char* d = buf + h * G::chunk;
            if (!ODD) {
                tensor_to_smem(d, &a.tm_even, c0 & ~(G::align - 1), 0, 0, bar);
            } else {
#pragma unroll
                for (int lo = 0; lo < 9; ++lo)
                    tensor_to_smem(d + lo * G::group, &a.tm_odd, group_x0(a, c0, lo) & ~(G::align - 1), lo, 0, bar);
            }
        }
    }
    __syncwarp();
}

// the shared-memory address of the value that cell c0 + j of a chunk reads for direction q:
// slot q at the cell (even step), slot s = opp(q) at x - c_q (odd step; s = 9 hi + lo with
// hi = 1 - cx, so the source lies hi cells into the group's window past the cell's own place)
template <int DT, bool ODD>
__device__ __forceinline__ const char* staged_elem(const CaseArgs<float>& a, const char* chunk_buf, int c0, int q, int j)
{
    using G = StageGeom<DT>;
    if (!ODD) return chunk_buf + q * G::row + ((c0 & (G::align - 1)) + j) * G::sz;
    const int s = 26 - q, hi = s / 9, lo = s % 9;
    const int r = group_x0(a, c0, lo) & (G::align - 1);
    return chunk_buf + lo * G::group + hi * G::row + (r + hi + j) * G::sz;
}

// a pair's populations from its staged windows: the raw stored value + weight of each cell,
// or the rest state where the cell does not collide
template <int DT, bool ODD>
__device__ __forceinline__ void staged_pair_load(const CaseArgs<float>& a, const Chunk& ca, const Chunk& cb, bool adj, int lane,
                                                 const char* buf, f2* f)
{
    using G = StageGeom<DT>;
    const f2 isc(a.inv_scale);
    if (adj) {
        // lane l: cells 2l, 2l + 1 of the 64-cell span, in chunk l / 16.  Both chunks have the
        // same window offsets (they are 32 cells apart); the even step's pairs are aligned
        const char* cbuf = buf + (lane >> 4) * G::chunk;
        const int j = (2 * lane) & 31;
#pragma unroll
        for (int q = 0; q < 27; ++q) {
            const char* e = staged_elem<DT, ODD>(a, cbuf, ca.c0, q, j);
            f2 raw;
            if constexpr (DT == 1) {
                raw = ODD ? f2(((const float*)e)[0], ((const float*)e)[1]) : f2(*(const float2*)e);
            } else {
                const unsigned w = ODD ? ((unsigned)((const unsigned short*)e)[0] | ((unsigned)((const unsigned short*)e)[1] << 16))
                                       : *(const unsigned*)e;
                raw = Pair2<DT>::of(w);
            }
            const f2 w(weight<float>(q));
            f[q] = DT == 1 ? raw + w : mad(raw, isc, w);
        }
    } else {
        const unsigned bit = 1u << lane;
        const bool fa = (ca.fluid & bit) != 0, fb = (cb.fluid & bit) != 0;
#pragma unroll
        for (int q = 0; q < 27; ++q) {
            const char* ea = staged_elem<DT, ODD>(a, buf, ca.c0, q, lane);
            const char* eb = staged_elem<DT, ODD>(a, buf + G::chunk, cb.c0, q, lane);
            float va, vb;
            if constexpr (DT == 1) {
                va = *(const float*)ea;
                vb = *(const float*)eb;
            } else {
                va = Cook<DT>::of_bits(*(const unsigned short*)ea);
                vb = Cook<DT>::of_bits(*(const unsigned short*)eb);
            }
            const f2 raw(fa ? va : 0.f, fb ? vb : 0.f);
            const f2 w(weight<float>(q));
            f[q] = DT == 1 ? raw + w : mad(raw, isc, w);
        }
    }
}

template <int DT, int COL, bool ODD, int ARGS>
__global__ void __launch_bounds__(kStagedThreads) __maxnreg__((StepRegs<DT, COL, true>::value))
    k_step_staged(const __grid_constant__ GroupArgs<float> g)
{
    using G = StageGeom<DT>;
    extern __shared__ __align__(128) char stage_smem[];
    __shared__ __align__(8) uint64_t bars[G::warps][2];
    // each warp's loop state between its pairs: the unit, and bits {0: this unit staged,
    // 1: the next unit staged, 2 + b: the phase to wait for on buffer b, 4: this unit's
    // buffer}.  It lives in shared memory across the collision, whose registers it would
    // otherwise hold
    __shared__ int loop_state[G::warps][2];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int step = g.cursor[ODD ? 1 : 0];
    if (blockIdx.x == 0 && threadIdx.x == 0) g.cursor[ODD ? 0 : 1] = step + 1;
    const int flags = case_args<ARGS>(g, 0).ctl[step].flags;
    uint64_t* bar = bars[wid];
    volatile int* ls = loop_state[wid];
    if (lane == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_init_fence();
    }
    __syncwarp();
    // unit u < np: the chunk pair (2u, 2u + 1); above: a batch of 32 boundary nodes
    auto n_units = [&]() { return (g.n_chunks >> 1) + (g.n_nodes + 31) / 32; };
    char* const smem0 = stage_smem + ((128u - (smem_addr(stage_smem) & 127u)) & 127u); // 128-byte aligned
    auto buffer = [&](int b) { return smem0 + (wid * 2 + b) * G::unit; };
    auto stage = [&](int u, int b) -> bool {
        if (u >= (g.n_chunks >> 1)) return false;
        const Chunk ca = g.chunks[2 * u], cb = g.chunks[2 * u + 1];
        if (!pairable<ARGS>(g, ca, cb)) return false;
        stage_pair<DT, ODD>(case_args<ARGS>(g, ca.cflags & CH_CASE_MASK), ca.c0, cb.c0, lane, buffer(b), &bar[b], g.stage_pad);
        return true;
    };
    {
        const int u = blockIdx.x * G::warps + wid;
        const bool st = u < n_units() && stage(u, 0);
        if (lane == 0) { ls[0] = u; ls[1] = st ? 1 : 0; }
        __syncwarp();
    }
    while (true) {
        const int u = ls[0];
        int state = ls[1];
        if (u >= n_units()) break;
        const int b = (state >> 4) & 1;
        const int un = u + gridDim.x * G::warps;
        // the next pair's rows travel while this one collides (its buffer was released by
        // the __syncwarp that ended the unit before)
        if (un < n_units() && stage(un, b ^ 1)) state |= 2;
        const int np = g.n_chunks >> 1;
        if (u < np) {
            const Chunk ca = g.chunks[2 * u], cb = g.chunks[2 * u + 1];
            const int ci = ca.cflags & CH_CASE_MASK;
            const CaseArgs<float>& a = case_args<ARGS>(g, ci);
            if (state & 1) {
                if (!mbar_wait(&bar[b], (state >> (2 + b)) & 1, g.stage_wait_ns)) {
                    if (lane == 0) atomicOr(a.err, ERR_STALL);
                    // the copies of the next pair are this warp's: let them land before it leaves
                    if (state & 2) mbar_wait(&bar[b ^ 1], (state >> (3 - b)) & 1, g.stage_wait_ns);
                    return;
                }
                state ^= 4 << b;
                // the loop state waits in shared memory while the pair collides
                if (lane == 0) ls[1] = state;
                f2 f[27];
                const bool adj = adjacent_span<DT>(ca, cb);
                staged_pair_load<DT, ODD>(a, ca, cb, adj, lane, buffer(b), f);
                pair_finish<DT, COL, ODD>(a, g.cases + ci, ca, cb, g.chunks + 2 * u, g.chunk_nodes + 2 * u, f, step, flags, lane,
                                          adj);
                __syncwarp();
                state = ls[1];
            } else {
                // inline like the two-cell kernel's, so that both round these chunks alike
                if (lane == 0) ls[1] = state;
                fluid_chunk<DT, COL, ODD>(a, g.cases + ci, ca, g.chunks + 2 * u, g.chunk_nodes + 2 * u, step, flags, lane);
                if (cb.fluid) {
                    const int cj = cb.cflags & CH_CASE_MASK;
                    fluid_chunk<DT, COL, ODD>(case_args<ARGS>(g, cj), g.cases + cj, cb, g.chunks + 2 * u + 1,
                                              g.chunk_nodes + 2 * u + 1, step, flags, lane);
                }
                __syncwarp();
                state = ls[1];
            }
        } else {
            node_batch<DT, ODD>(g.nodes, g.n_nodes, g.cases, g.bc_prof, g.bc_buf, (u - np) * 32 + lane, step, flags);
        }
        // next: the next unit in this unit's place, its buffer the other one
        state = ((state >> 1) & 1) | (state & (3 << 2)) | ((b ^ 1) << 4);
        __syncwarp();
        if (lane == 0) { ls[0] = u + gridDim.x * G::warps; ls[1] = state; }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------------------
// open-plane nodes: the re-centred stencil of each, before the step
// ---------------------------------------------------------------------------------------
// canonical post-collision population q of cell (x,y,z) of the previous step, in the A-A
// layout that step left behind
__device__ __forceinline__ int clamp_cell(int nx, int ny, int nz, int x, int y, int z)
{
    return min(max(x, 0), nx - 1) + nx * (min(max(y, 0), ny - 1) + ny * min(max(z, 0), nz - 1));
}

template <int DT, bool ODD>
__device__ __forceinline__ typename Storage<DT>::CT canon(const CaseArgs<typename Storage<DT>::CT>& a, int x, int y, int z, int q)
{
    using S = Storage<DT>;
    x = min(max(x, 0), a.nx - 1); y = min(max(y, 0), a.ny - 1); z = min(max(z, 0), a.nz - 1);
    const int sy = a.nx, sz = a.nx * a.ny;
    const int c = x + sy * y + sz * z;
    if (ODD) // the previous (even) step stored f*_q of x in slot opp(q) at x
        return S::load(qptr<DT>(a, oppq(q)), c, q, a.inv_scale);
    // the previous (odd) step, or the initial state, stored f*_q of x in slot q at x + c_q, or,
    // with halfway bounce-back towards a wall, in slot opp(q) at x
    if (a.hw && ((a.hw[c] >> q) & 1u)) return S::load(qptr<DT>(a, oppq(q)), c, q, a.inv_scale);
    return S::load(qptr<DT>(a, q), wrapc(x + cxq(q), a.nx) + sy * wrapc(y + cyq(q), a.ny) + sz * wrapc(z + czq(q), a.nz), q,
                   a.inv_scale);
}

// LBM_STREAMING::streaming with explicit (m, centre, p) triples (lbm_streaming.h:10-39); with
// halfway bounce-back a population that would come from a WALL cell is the centre's own
// post-collision population of the opposite direction
template <int DT, bool ODD>
__device__ __forceinline__ void pull_triples(const CaseArgs<typename Storage<DT>::CT>& a, const int* xs, const int* ys, const int* zs,
                                             typename Storage<DT>::CT* f)
{
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const int sx = xs[1 - cxq(q)], sy = ys[1 - cyq(q)], sz = zs[1 - czq(q)];
        if (a.hw && (a.label[clamp_cell(a.nx, a.ny, a.nz, sx, sy, sz)] & L_MASK) == L_WALL)
            f[q] = canon<DT, ODD>(a, xs[1], ys[1], zs[1], oppq(q));
        else
            f[q] = canon<DT, ODD>(a, sx, sy, sz, q);
    }
}

template <int DT, bool ODD, int ARGS>
__global__ void __launch_bounds__(64) k_bc_gather(const __grid_constant__ GroupArgs<typename Storage<DT>::CT> g)
{
    using CT = typename Storage<DT>::CT;
    pdl_launch_dependents();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.n_gather) return;
    // {cell, case, node index, label}: the stencil loads depend on nothing but this record
    // (and the case's arguments, from the parameters where the group is small)
    const int4 e = g.gather[t];
    const CaseArgs<CT>& a = case_args<ARGS>(g, e.y);
    const StepCtl<CT>& ctl = a.ctl[g.cursor[ODD ? 1 : 0]];
    const int c = e.x, k = e.z;
    const int lab = e.w;
    const int x = c % a.nx, y = (c / a.nx) % a.ny, z = c / (a.nx * a.ny);
    // clamped neighbours of a non-periodic cell (core.h:651-661)
    const int xm = max(x - 1, 0), xp = min(x + 1, a.nx - 1), ym = max(y - 1, 0), yp = min(y + 1, a.ny - 1);
    const int zm = max(z - 1, 0), zp = min(z + 1, a.nz - 1);
    int xs[3] = {xm, x, xp}, ys[3] = {ym, y, yp}, zs[3] = {zm, z, zp};
    CT f[27];
    CT rho = 1, ux = 0, uy = 0, uz = 0;
    switch (lab) {
    case L_IN_L: // sim_tcpc.cu:242-251
    case L_IN_R: // sim_tcpc.cu:252-261
        if (lab == L_IN_L) { xs[0] = x; xs[1] = xp; xs[2] = xp + 1; }
        else { xs[0] = xm - 1; xs[1] = xm; xs[2] = x; }
        pull_triples<DT, ODD>(a, xs, ys, zs, f);
        rho = density<CT>(f);
        ux = lab == L_IN_L ? ctl.u_left : ctl.u_right;
        break;
    case L_OUT_F: // sim_tcpc.cu:262-267
    case L_OUT_B: // sim_tcpc.cu:268-273
        if (lab == L_OUT_F) { ys[0] = y; ys[1] = yp; ys[2] = yp + 1; }
        else { ys[0] = ym - 1; ys[1] = ym; ys[2] = y; }
        pull_triples<DT, ODD>(a, xs, ys, zs, f);
        density_velocity<CT>(f, a.fx, a.fy, a.fz, rho, ux, uy, uz);
        rho = CT(1);
        break;
    case L_OUT_REQ: // lbm_bc.h:147-152
        xs[0] = xm - 1; xs[1] = xm; xs[2] = x;
        pull_triples<DT, ODD>(a, xs, ys, zs, f);
        density_velocity<CT>(f, a.fx, a.fy, a.fz, rho, ux, uy, uz);
        rho = CT(1);
        break;
    default:
        break;
    }
    g.bc_buf[4 * k] = rho; g.bc_buf[4 * k + 1] = ux; g.bc_buf[4 * k + 2] = uy; g.bc_buf[4 * k + 3] = uz;
}

// ---------------------------------------------------------------------------------------
// NNLBM_CY_REF_FD phases 1 and 2 (core.h:1176-1258): velocity of the post-streaming state
// of every FLUID cell with the force of the previous step, then the finite-difference
// strain from it.  Non-FLUID values are never read by the strain stencil.
// ---------------------------------------------------------------------------------------
template <int DT, bool ODD>
__global__ void __launch_bounds__(256) k_refd_velocity(const __grid_constant__ GroupArgs<typename Storage<DT>::CT> g)
{
    using CT = typename Storage<DT>::CT;
    const int lane = threadIdx.x & 31;
    const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (warp >= g.n_chunks) return;
    const Chunk& ch = g.chunks[warp];
    const CaseArgs<CT>& a = g.cases[ch.cflags & CH_CASE_MASK];
    if (a.cy_mode != CY_REF_FD) return;
    const int y = ch.yz & 0xffff, z = ch.yz >> 16;
    const int x = ch.c0 - y * a.nx - z * a.nx * a.ny + lane;
    const int c = ch.c0 + lane;
    if (x >= a.nx || (a.label[c] & L_MASK) != L_FLUID) return;
    const int xs[3] = {x - 1, x, x + 1}, ys[3] = {y - 1, y, y + 1}, zs[3] = {z - 1, z, z + 1};
    CT f[27];
    pull_triples<DT, ODD>(a, xs, ys, zs, f);
    CT* M = a.macro;
    const int64_t N = a.N;
    CT rho, ux, uy, uz;
    density_velocity<CT>(f, M[M_FX * N + c], M[M_FY * N + c], M[M_FZ * N + c], rho, ux, uy, uz);
    M[M_RHO * N + c] = rho; M[M_VX * N + c] = ux; M[M_VY * N + c] = uy; M[M_VZ * N + c] = uz;
}

template <class CT>
__global__ void __launch_bounds__(256) k_refd_stress(const __grid_constant__ GroupArgs<CT> g)
{
    const int lane = threadIdx.x & 31;
    const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (warp >= g.n_chunks) return;
    const Chunk& ch = g.chunks[warp];
    const CaseArgs<CT>& a = g.cases[ch.cflags & CH_CASE_MASK];
    if (a.cy_mode != CY_REF_FD) return;
    const int sy = a.nx, sz = a.nx * a.ny;
    const int y = ch.yz & 0xffff, z = ch.yz >> 16;
    const int x = ch.c0 - y * sy - z * sz + lane;
    const int c = ch.c0 + lane;
    if (x >= a.nx || (a.label[c] & L_MASK) != L_FLUID) return;
    CT* M = a.macro;
    const int64_t N = a.N;
    const int cn[6] = {c - 1, c + 1, c - sy, c + sy, c - sz, c + sz};
    bool fl[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) fl[k] = (a.label[cn[k]] & L_MASK) == L_FLUID;
    auto d1 = [&](int fld, int axis) -> CT {
        const bool m = fl[2 * axis], p = fl[2 * axis + 1];
        const CT* F = M + (int64_t)fld * N;
        if (!m) return p ? F[cn[2 * axis + 1]] - F[c] : CT(0);
        if (!p) return F[c] - F[cn[2 * axis]];
        return CT(0.5) * (F[cn[2 * axis + 1]] - F[cn[2 * axis]]);
    };
    // core.h:489-573: S12 = (du_y/dx + du_x/dy)/2 etc.
    const CT S11 = d1(M_VX, 0), S22 = d1(M_VY, 1), S33 = d1(M_VZ, 2);
    const CT S12 = CT(0.5) * d1(M_VY, 0) + CT(0.5) * d1(M_VX, 1);
    const CT S13 = CT(0.5) * d1(M_VZ, 0) + CT(0.5) * d1(M_VX, 2);
    const CT S32 = CT(0.5) * d1(M_VZ, 1) + CT(0.5) * d1(M_VY, 2);
    M[M_S11 * N + c] = S11; M[M_S12 * N + c] = S12; M[M_S13 * N + c] = S13;
    M[M_S22 * N + c] = S22; M[M_S32 * N + c] = S32; M[M_S33 * N + c] = S33;
}

// ---------------------------------------------------------------------------------------
// VTK output fields (StateTcpc::outputData, sim_tcpc.cu:684-784), per cell in double like the
// reference's host code and stored as float, the type of the file's arrays
// ---------------------------------------------------------------------------------------
// physical scales of one output call (sim_tcpc.cu:716-745): lattice -> physical velocity,
// the physical density, the lattice reference viscosity and the Carreau-Yasuda law
struct OutputParams {
    double dx, dt, density, nu_lbm;
    double cy, nu0, lambda, a, n;  // cy != 0: Carreau-Yasuda material
    double diff;                   // steps summed in the mean/rms sums, at least 1
};
// fields in file order, 20 values a cell: velocity (3), mean_velocity (3), lbm_rho,
// pressure_pa, gamma_dot, nu_phys_m2_s, mu_phys_pa_s, wss_proxy_pa, turbulence_intensity,
// rms_velocity, strain_diag_1_s (3), strain_shear_1_s (3)
constexpr int kOutputValues = 20;

template <class CT>
__global__ void __launch_bounds__(256) k_output_fields(const CaseArgs<CT> a, const OutputParams p, const uint8_t* wall,
                                                       float* out)
{
    const int64_t N = a.N;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < N; c += (int64_t)gridDim.x * blockDim.x) {
        const CT* M = a.macro;
        const double v2p = p.dx / p.dt;
        const double vx = (double)M[M_VX * N + c] * v2p, vy = (double)M[M_VY * N + c] * v2p, vz = (double)M[M_VZ * N + c] * v2p;
        double s[6] = {0, 0, 0, 0, 0, 0};
        if (a.stats) {
            for (int k = 0; k < 6; ++k)
                s[k] = a.stats_f64 ? ((const double*)a.stats)[k * N + c] : (double)((const float*)a.stats)[k * N + c];
        }
        const double mx = s[0] * v2p / p.diff, my = s[1] * v2p / p.diff, mz = s[2] * v2p / p.diff;
        const double rx = fabs(s[3] * v2p * v2p / p.diff - mx * mx), ry = fabs(s[4] * v2p * v2p / p.diff - my * my);
        const double rz = fabs(s[5] * v2p * v2p / p.diff - mz * mz);
        const double rms = sqrt(rx * rx + ry * ry + rz * rz);
        const double meanv = sqrt(mx * mx + my * my + mz * mz);
        const double turb = fabs(meanv) <= 1e-10 ? 0.0 : rms / fabs(meanv);
        const double rho = (double)M[M_RHO * N + c];
        const double pressure = (rho - 1.0) * p.density * (v2p * v2p / 3.0);
        const double S11 = M[M_S11 * N + c], S12 = M[M_S12 * N + c], S13 = M[M_S13 * N + c];
        const double S22 = M[M_S22 * N + c], S32 = M[M_S32 * N + c], S33 = M[M_S33 * N + c];
        const double gl = sqrt(2.0) * sqrt(S11 * S11 + S22 * S22 + S33 * S33 + 2.0 * (S12 * S12 + S13 * S13 + S32 * S32));
        const double gdot = gl / p.dt;
        const double nul = p.cy != 0.0 ? p.nu_lbm + (p.nu0 - p.nu_lbm) * pow(1.0 + pow(gl * p.lambda, p.a), (p.n - 1.0) / p.a)
                                       : p.nu_lbm;
        const double nup = nul * p.dx * p.dx / p.dt;
        const double mup = nup * p.density;
        // nearWall (sim_tcpc.cu:709-714): a wall among the six neighbours inside the box
        const int x = (int)(c % a.nx), y = (int)((c / a.nx) % a.ny), z = (int)(c / ((int64_t)a.nx * a.ny));
        const int64_t sy = a.nx, sz = (int64_t)a.nx * a.ny;
        const bool near = (x > 0 && wall[c - 1]) || (x < a.nx - 1 && wall[c + 1]) || (y > 0 && wall[c - sy]) ||
                          (y < a.ny - 1 && wall[c + sy]) || (z > 0 && wall[c - sz]) || (z < a.nz - 1 && wall[c + sz]);
        const double v[kOutputValues] = {vx, vy, vz, mx, my, mz, rho, pressure, gdot, nup, mup, near ? mup * gdot : 0.0,
                                         turb, rms, S11 / p.dt, S22 / p.dt, S33 / p.dt, S12 / p.dt, S13 / p.dt, S32 / p.dt};
#pragma unroll
        for (int k = 0; k < kOutputValues; ++k) out[k * N + c] = (float)v[k];
    }
}

// ---------------------------------------------------------------------------------------
// host-side dispatch: one function per (storage, collision) instantiated in its own
// translation unit
// ---------------------------------------------------------------------------------------
using GroupLauncher = void (*)(bool odd, dim3 grid, dim3 block, cudaStream_t s, const void* group_args);
// the step kernel's launch forms: one cell a thread, two (the paired form), and the paired
// form with staged loads (k_step_staged, persistent warps, StageGeom shared memory)
enum : int { FORM_ONE = 0, FORM_PAIRED = 1, FORM_STAGED = 2 };
// the step kernel's launcher: `after_gather` launches it as a programmatic dependent of the
// gather kernel just enqueued on the stream
using StepLauncher = void (*)(bool odd, bool after_gather, int form, dim3 grid, dim3 block, cudaStream_t s,
                              const void* group_args);
// resident blocks per SM of the staged form (0 where the variant has no staged form)
using StagedOccupancy = int (*)();

// the kernel of one step variant
template <int DT, int COL, bool ODD, int ARGS, int FORM>
constexpr auto step_kernel()
{
    if constexpr (FORM == FORM_STAGED) return &k_step_staged<DT, COL, ODD, ARGS>;
    else return &k_step<DT, COL, ODD, ARGS, FORM == FORM_PAIRED>;
}
template <int DT, int FORM>
constexpr size_t step_smem()
{
    if constexpr (FORM == FORM_STAGED) return (size_t)StageGeom<DT>::smem;
    else return 0;
}

// the work list stays in L2 between steps where it is small (a sparse geometry's list is
// read at the head of every warp's dependent chain; a dense box's streams once per step)
#ifndef NNLBM_PERSIST_CHUNKS
#define NNLBM_PERSIST_CHUNKS 1
#endif
constexpr size_t kPersistChunkBytes = size_t(16) << 20;

// launch of one step-kernel variant
template <int DT, int COL, bool ODD, int ARGS, int FORM>
void launch_step_variant(bool after_gather, dim3 grid, dim3 block, cudaStream_t s, const GroupArgs<typename Storage<DT>::CT>& g)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = step_smem<DT, FORM>();
    cfg.stream = s;
    cudaLaunchAttribute attr[2];
    int n = 0;
    if (after_gather) {
        attr[n].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[n].val.programmaticStreamSerializationAllowed = 1;
        ++n;
    }
    const size_t chunk_bytes = (size_t)g.n_chunks * sizeof(Chunk);
    if (NNLBM_PERSIST_CHUNKS && chunk_bytes > 0 && chunk_bytes <= kPersistChunkBytes) {
        attr[n].id = cudaLaunchAttributeAccessPolicyWindow;
        attr[n].val.accessPolicyWindow.base_ptr = (void*)g.chunks;
        attr[n].val.accessPolicyWindow.num_bytes = chunk_bytes;
        attr[n].val.accessPolicyWindow.hitRatio = 1.0f;
        attr[n].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        attr[n].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
        ++n;
    }
    cfg.attrs = attr;
    cfg.numAttrs = n;
    cudaLaunchKernelEx(&cfg, step_kernel<DT, COL, ODD, ARGS, FORM>(), g);
}

template <int DT, int COL, int FORM>
void launch_step_form(bool odd, bool after_gather, dim3 grid, dim3 block, cudaStream_t s, const GroupArgs<typename Storage<DT>::CT>& g)
{
    switch (args_mode(g.n_cases)) {
    case ARGS_ONE:
        if (odd) launch_step_variant<DT, COL, true, ARGS_ONE, FORM>(after_gather, grid, block, s, g);
        else launch_step_variant<DT, COL, false, ARGS_ONE, FORM>(after_gather, grid, block, s, g);
        break;
    case ARGS_PARAM:
        if (odd) launch_step_variant<DT, COL, true, ARGS_PARAM, FORM>(after_gather, grid, block, s, g);
        else launch_step_variant<DT, COL, false, ARGS_PARAM, FORM>(after_gather, grid, block, s, g);
        break;
    default:
        if (odd) launch_step_variant<DT, COL, true, ARGS_GLOBAL, FORM>(after_gather, grid, block, s, g);
        else launch_step_variant<DT, COL, false, ARGS_GLOBAL, FORM>(after_gather, grid, block, s, g);
    }
}

// `form`: FORM_PAIRED and FORM_STAGED apply where the collision pairs (pairs_chunks); the
// others step one cell a thread
template <int DT, int COL>
void launch_step(bool odd, bool after_gather, int form, dim3 grid, dim3 block, cudaStream_t s, const void* args)
{
    using CT = typename Storage<DT>::CT;
    const GroupArgs<CT>& g = *(const GroupArgs<CT>*)args;
    if constexpr (pairs_chunks(DT, COL)) {
        if (form == FORM_PAIRED) {
            launch_step_form<DT, COL, FORM_PAIRED>(odd, after_gather, grid, block, s, g);
            return;
        }
        if (form == FORM_STAGED) {
            launch_step_form<DT, COL, FORM_STAGED>(odd, after_gather, grid, block, s, g);
            return;
        }
    }
    launch_step_form<DT, COL, FORM_ONE>(odd, after_gather, grid, block, s, g);
}

StepLauncher step_launcher(int dtype, int collision);
StagedOccupancy staged_occupancy(int dtype, int collision);

// Every variant of the step kernel of a (storage, collision) resolved now.  Under CUDA's lazy
// module loading the runtime loads a kernel's code at its first launch, which allocates device
// memory then; a context loads its kernels when it is created instead.  The staged form is
// also allowed its shared memory here.
template <int DT, int COL, bool ODD, int ARGS>
cudaError_t load_step_variant()
{
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, (const void*)k_step<DT, COL, ODD, ARGS, false>);
    if constexpr (pairs_chunks(DT, COL)) {
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, (const void*)k_step<DT, COL, ODD, ARGS, true>);
        const void* k = (const void*)k_step_staged<DT, COL, ODD, ARGS>;
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, StageGeom<DT>::smem);
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k);
    }
    return e;
}
template <int DT, int COL>
cudaError_t load_step()
{
    const cudaError_t e[6] = {load_step_variant<DT, COL, false, ARGS_ONE>(), load_step_variant<DT, COL, true, ARGS_ONE>(),
                              load_step_variant<DT, COL, false, ARGS_PARAM>(), load_step_variant<DT, COL, true, ARGS_PARAM>(),
                              load_step_variant<DT, COL, false, ARGS_GLOBAL>(), load_step_variant<DT, COL, true, ARGS_GLOBAL>()};
    for (cudaError_t x : e)
        if (x != cudaSuccess) return x;
    return cudaSuccess;
}
// resident blocks per SM of the staged form (the fewest over its variants), 0 without one
template <int DT, int COL>
int staged_blocks()
{
    if constexpr (pairs_chunks(DT, COL)) {
        int best = 1 << 30;
        const void* ks[6] = {(const void*)k_step_staged<DT, COL, false, ARGS_ONE>, (const void*)k_step_staged<DT, COL, true, ARGS_ONE>,
                             (const void*)k_step_staged<DT, COL, false, ARGS_PARAM>, (const void*)k_step_staged<DT, COL, true, ARGS_PARAM>,
                             (const void*)k_step_staged<DT, COL, false, ARGS_GLOBAL>, (const void*)k_step_staged<DT, COL, true, ARGS_GLOBAL>};
        for (const void* k : ks) {
            int n = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, kStagedThreads, StageGeom<DT>::smem) != cudaSuccess) return 0;
            best = n < best ? n : best;
        }
        return best;
    } else {
        return 0;
    }
}

} // namespace nnlbm
