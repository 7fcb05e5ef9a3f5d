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
// Work decomposition: a packed list of 32-cell row chunks (one warp each) that contain a
// cell with work, over all cases of a launch group (same storage type and collision).
// Per-case parameters live in a device array indexed by the chunk's case.
//
// Open-plane nodes (TCPC IVC/SVC inflow and outlets, generic GEO_OUTFLOW_RIGHT_EQ) pull a
// stencil re-centred one cell inward (sim_tcpc.cu:242-273, lbm_bc.h:147-152).  Those
// populations are exactly the ones the inward neighbour pulls for itself, so when that
// neighbour is a FLUID/PERIODIC cell with the same tangential stencil ("source") its own
// thread computes the node's density / velocity and writes the node's equilibrium into
// the node's slots (which no other cell touches within the step).  The remaining nodes
// (corners, CY_REF_FD outlets) are gathered by k_bc_gather before the step kernel and
// written by their own thread; GEO_INFLOW nodes need no gather at all.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>

#include "nnlbm_physics.cuh"

namespace nnlbm {

enum : int { L_FLUID = 0, L_WALL = 1, L_PERIODIC = 2, L_IN_L = 3, L_IN_R = 4, L_OUT_F = 5, L_OUT_B = 6,
             L_IN_EQ = 7, L_OUT_REQ = 8 };
// flag bits of the device label byte (the low four bits hold the label)
enum : int { LF_SOURCE = 0x80, LF_SELF = 0x40, LF_FUSED = 0x20, L_MASK = 0x0f };
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
    __device__ static __forceinline__ CT load(const T* p, int i, int, CT) { return p[i]; }
    __device__ static __forceinline__ void store(T* p, int i, int, CT v, CT) { p[i] = v; }
};
template <> struct Storage<1> {
    using T = float; using CT = float;
    __device__ static __forceinline__ CT from(T v, int q, CT) { return weight<float>(q) + v; }
    __device__ static __forceinline__ CT load(const T* p, int i, int q, CT) { return weight<float>(q) + p[i]; }
    __device__ static __forceinline__ void store(T* p, int i, int q, CT v, CT) { p[i] = v - weight<float>(q); }
};
template <> struct Storage<2> {
    using T = __half; using CT = float;
    __device__ static __forceinline__ CT from(T v, int q, CT isc) { return weight<float>(q) + __half2float(v) * isc; }
    __device__ static __forceinline__ CT load(const T* p, int i, int q, CT isc) { return from(p[i], q, isc); }
    __device__ static __forceinline__ void store(T* p, int i, int q, CT v, CT sc) { p[i] = __float2half_rn((v - weight<float>(q)) * sc); }
};
template <> struct Storage<3> {
    using T = __nv_bfloat16; using CT = float;
    __device__ static __forceinline__ CT from(T v, int q, CT isc) { return weight<float>(q) + __bfloat162float(v) * isc; }
    __device__ static __forceinline__ CT load(const T* p, int i, int q, CT isc) { return from(p[i], q, isc); }
    __device__ static __forceinline__ void store(T* p, int i, int q, CT v, CT sc) { p[i] = __float2bfloat16_rn((v - weight<float>(q)) * sc); }
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
    double* red;               // [5] mass, Q_ivc, Q_svc, Q_out5, Q_out6
    int* err;                  // watchdog flag
};

// a launch group: cases sharing storage type and collision
template <class CT>
struct GroupArgs {
    CaseArgs<CT> c0;           // copy of case 0 in parameter space (single-case groups)
    int n_cases, pad2;
    const CaseArgs<CT>* cases;
    const int4* chunks;        // {first cell, y | z << 16, case, first self-node index}
    int n_chunks, pad0;
    const int4* gather;        // {cell, case, self-node index, 0} of the gathered nodes
    int n_gather, pad1;
    const CT* bc_prof;         // [n_self][3] prescribed velocity (GEO_INFLOW nodes)
    CT* bc_buf;                // [n_self][4] gathered rho, ux, uy, uz
    int* cursor;               // step cursor into every case's ctl
    int* done;                 // block counter of the step kernel
};

template <int DT>
__device__ __forceinline__ typename Storage<DT>::T* qptr(const CaseArgs<typename Storage<DT>::CT>& a, int q)
{
    return (typename Storage<DT>::T*)a.df + (int64_t)q * a.qstride;
}

__device__ __forceinline__ int wrapc(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

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
#pragma unroll
        for (int q = 0; q < 27; ++q)
            S::store(qptr<DT>(a, q), wrapc(x + cxq(q), a.nx) + sy * wrapc(y + cyq(q), a.ny) + sz * wrapc(z + czq(q), a.nz), q, f[q],
                     a.scale);
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

// rare paths of the step kernel are kept out of line so that they do not take registers
// from the bulk path: the equilibrium of an open-plane node with its bookkeeping ...
template <int DT, bool ODD>
__device__ __noinline__ double finish_node(const CaseArgs<typename Storage<DT>::CT>& a, int flags, int lab, int c, int x, int y,
                                           int z, typename Storage<DT>::CT rho, typename Storage<DT>::CT ux,
                                           typename Storage<DT>::CT uy, typename Storage<DT>::CT uz)
{
    store_node_eq<DT, ODD>(a, c, x, y, z, rho, ux, uy, uz);
    return node_outputs<typename Storage<DT>::CT>(a, flags, lab, c, rho, ux, uy, uz);
}

// ... and the finite-difference Carreau-Yasuda force of CY_REF_FD (core.h:663-781):
// divergence of the strain of the previous phase with one-sided differences next to
// non-FLUID cells, then 2 (nu(gamma) - nu) F rho with rho still at its default of 1
template <class CT>
__device__ __noinline__ void refd_force(const CaseArgs<CT>& a, int c, int sy, int sz, CT* F)
{
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

// minimum resident blocks of 256 threads: the register budget of each variant (FP64
// arithmetic and the KBC family need more live values than the cumulant in FP32)
#ifndef NNLBM_STEP_MINB
#define NNLBM_STEP_MINB 2
#endif
template <int DT, int COL>
struct StepOccupancy {
    static constexpr int value = DT == 0 ? 1 : ((COL >= COL_KBC_N1 && COL <= COL_KBC_C4) ? 2 : NNLBM_STEP_MINB);
};

// ---------------------------------------------------------------------------------------
// shared-memory staging of a chunk with TMA bulk copies (cp.async.bulk global -> shared,
// completion counted in bytes on an mbarrier); no cluster, no multicast
// ---------------------------------------------------------------------------------------
// chunk record flags (bits 16.. of the case word)
enum : int { CH_CASE_MASK = 0xffff, CH_FLUID = 1 << 16, CH_FACE = 1 << 17 };

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// one bounded probe of the phase; the hint caps the suspension at 20 microseconds
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done)
                 : "r"(bar), "r"(parity), "r"(20000u)
                 : "memory");
    return done != 0;
}

// wait for a phase with an iteration limit (about two seconds); false when it ran out
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (int it = 0; it < 100000; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// `bytes` (a multiple of 16) from 16-byte aligned global memory into shared memory
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// one pipeline stage of a warp: the 27 population rows of its chunk, each copied from the
// 16-byte boundary at or below the row's first element (so a row spans 32 elements plus
// up to 16 bytes of slack), and the chunk's label row likewise
template <int DT>
struct Stage {
    static constexpr int S = (int)sizeof(typename Storage<DT>::T);
    static constexpr int RB = 32 * S + 16;
    static constexpr int LB = 48;
    static constexpr int BYTES = 27 * RB + LB;
};
// per warp: two mbarriers (16 B) and a ring of its next 32 chunk records (512 B), then
// the two stages; up to 8 warps per block
constexpr int kRing = 32;
constexpr int kStepSmemHead = 8 * (16 + kRing * 16);
template <int DT>
constexpr int step_smem_bytes(int warps_per_block) { return kStepSmemHead + warps_per_block * 2 * Stage<DT>::BYTES; }

// start the copies of chunk `rec` into stage `stg`; returns the bytes the stage's
// mbarrier expects (0: the chunk loads directly from global memory)
template <int DT, bool ODD, bool SINGLE>
__device__ __forceinline__ uint32_t issue_chunk(const GroupArgs<typename Storage<DT>::CT>& g, int4 rec, unsigned char* stg,
                                                uint32_t bar, int lane)
{
    using G = Stage<DT>;
    using CT = typename Storage<DT>::CT;
    // an odd step of a chunk on a y/z face pulls across the face (wrapped rows)
    if (ODD && (rec.z & CH_FACE)) return 0;
    const CaseArgs<CT>& a = SINGLE ? g.c0 : g.cases[rec.z & CH_CASE_MASK];
    const bool fluid = (rec.z & CH_FLUID) != 0;
    const uint32_t bytes = fluid ? (uint32_t)(27 * G::RB + G::LB) : (uint32_t)G::LB;
    if (lane == 0) mbar_arrive_expect_tx(bar, bytes);
    __syncwarp();
    const int c0 = rec.x;
    if (lane < 27) {
        if (fluid) {
            const int q = lane;
            // even: slot q at the chunk's cells; odd: slot opp(q) at the cells - c_q
            const int slot = ODD ? oppq(q) : q;
            const int cs = ODD ? c0 - (cxq(q) + a.nx * cyq(q) + a.nx * a.ny * czq(q)) : c0;
            const int64_t off = ((int64_t)slot * a.qstride + cs) * G::S;
            bulk_g2s(smem_u32(stg) + q * G::RB, (const char*)a.df + (off & ~(int64_t)15), G::RB, bar);
        }
    } else if (lane == 27) {
        bulk_g2s(smem_u32(stg) + 27 * G::RB, a.label + (c0 & ~15), G::LB, bar);
    }
    return bytes;
}

// ---------------------------------------------------------------------------------------
// one 32-cell chunk of the fused step (solver/lbm3d/core.h:578-800): FLUID / PERIODIC
// cells collide, source cells also finish their fused open-plane neighbours,
// self-handled nodes write their equilibrium.  `stg` is the chunk's staged rows, or null
// when the chunk loads directly from global memory.
// ---------------------------------------------------------------------------------------
template <int DT, int COL, bool ODD, bool SINGLE>
__device__ __forceinline__ void process_chunk(const GroupArgs<typename Storage<DT>::CT>& g, int4 ch, const unsigned char* stg,
                                              int step, int lane)
{
    using S = Storage<DT>;
    using T = typename S::T;
    using CT = typename S::CT;
    using G = Stage<DT>;
    const CaseArgs<CT>& a = SINGLE ? g.c0 : g.cases[ch.z & CH_CASE_MASK];
    const int y = ch.y & 0xffff, z = ch.y >> 16;
    const int sy = a.nx, sz = a.nx * a.ny;
    const int x0 = ch.x - y * sy - z * sz;
    const int x = x0 + lane;
    const bool inb = x < a.nx;
    const int c = ch.x + lane;
    const int raw = !inb ? (int)L_WALL : stg ? (int)stg[27 * G::RB + (ch.x & 15) + lane] : (int)a.label[c];
    const int lab = raw & L_MASK;
    const bool fluid = lab == L_FLUID || lab == L_PERIODIC;
    const bool self = (raw & LF_SELF) != 0;
    const unsigned selfmask = __ballot_sync(0xffffffffu, self);
    const int flags = a.ctl[step].flags;
    double mass = 0.0, q3 = 0.0, q4 = 0.0, q5 = 0.0, q6 = 0.0;
    if (fluid) {
        const bool xin = x > 0 && x < a.nx - 1;
        // odd steps: index corrections of the wrapped neighbours (zero inside the box);
        // w*m apply to a neighbour at coordinate - 1, w*p to one at coordinate + 1
        const int wxm = x == 0 ? a.nx : 0, wxp = x == a.nx - 1 ? -a.nx : 0;
        const int wym = y == 0 ? sz : 0, wyp = y == a.ny - 1 ? -sz : 0;
        const int wzm = z == 0 ? (int)a.N : 0, wzp = z == a.nz - 1 ? -(int)a.N : 0;
        auto nbr = [&](int q, int sign) -> int { // cell at x + sign c_q
            const int dx = sign * cxq(q), dy = sign * cyq(q), dz = sign * czq(q);
            return c + dx + sy * dy + sz * dz + (dx < 0 ? wxm : dx > 0 ? wxp : 0) + (dy < 0 ? wym : dy > 0 ? wyp : 0) +
                   (dz < 0 ? wzm : dz > 0 ? wzp : 0);
        };
        CT f[27];
        if (!ODD) {
            // even steps always have the chunk staged: the element of this lane sits
            // (first element mod 16) bytes into its row, plus lane * element size
            const unsigned char* p = stg + lane * G::S + (((unsigned)ch.x * (unsigned)G::S) & 15u);
#pragma unroll
            for (int q = 0; q < 27; ++q) f[q] = S::from(*(const T*)(p + q * G::RB), q, a.inv_scale);
        } else if (stg && xin) {
            const unsigned char* p = stg + lane * G::S;
            const unsigned c0b = (unsigned)ch.x * (unsigned)G::S;
            const unsigned syb = (unsigned)sy * (unsigned)G::S, szb = (unsigned)sz * (unsigned)G::S;
#pragma unroll
            for (int q = 0; q < 27; ++q) {
                const unsigned d = (c0b - (unsigned)(cxq(q) * G::S) - (unsigned)cyq(q) * syb - (unsigned)czq(q) * szb) & 15u;
                f[q] = S::from(*(const T*)(p + q * G::RB + d), q, a.inv_scale);
            }
        } else {
#pragma unroll
            for (int q = 0; q < 27; ++q) f[q] = S::load(qptr<DT>(a, oppq(q)), nbr(q, -1), q, a.inv_scale);
        }
        CT fx = a.fx, fy = a.fy, fz = a.fz;
        if (a.cy_mode == CY_REF_FD && lab == L_FLUID) {
            CT F[3] = {fx, fy, fz};
            refd_force<CT>(a, c, sy, sz, F);
            fx = F[0]; fy = F[1]; fz = F[2];
        }
        CT rho, ux, uy, uz;
        density_velocity<CT>(f, fx, fy, fz, rho, ux, uy, uz);
        if (raw & LF_SOURCE) {
            // fused open-plane neighbours: their re-centred stencil is this cell's own pull
            const StepCtl<CT>& ctl = a.ctl[step];
            const int nbc[4] = {c - 1, c + 1, c - sy, c + sy};
            const bool inside[4] = {x > 0, x < a.nx - 1, y > 0, y < a.ny - 1};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (!inside[k]) continue;
                const int nr = a.label[nbc[k]];
                const int nl = nr & L_MASK;
                const bool ok = (nr & LF_FUSED) && (k == 0 ? nl == L_IN_L : k == 1 ? (nl == L_IN_R || nl == L_OUT_REQ)
                                                                           : k == 2 ? nl == L_OUT_F : nl == L_OUT_B);
                if (!ok) continue;
                const int bx = x + (k == 0 ? -1 : k == 1 ? 1 : 0), by = y + (k == 2 ? -1 : k == 3 ? 1 : 0);
                CT brho, bux = 0, buy = 0, buz = 0;
                if (nl == L_IN_L || nl == L_IN_R) { // sim_tcpc.cu:242-261
                    brho = rho;
                    bux = nl == L_IN_L ? ctl.u_left : ctl.u_right;
                } else { // sim_tcpc.cu:262-273, lbm_bc.h:147-152
                    brho = CT(1); bux = ux; buy = uy; buz = uz;
                }
                const double qn = finish_node<DT, ODD>(a, flags, nl, nbc[k], bx, by, z, brho, bux, buy, buz);
                if (nl == L_IN_L) q3 += qn;
                else if (nl == L_IN_R) q4 += qn;
                else if (nl == L_OUT_F) q5 += qn;
                else if (nl == L_OUT_B) q6 += qn;
            }
        }
        // one inlined collision for both viscosity models (the local Carreau-Yasuda law is
        // a runtime branch inside it)
        CT Sl[6];
        const CYParams<CT> cy = {a.nu, a.nu0, a.lam, a.a, a.n};
        collide<CT, COL>(f, rho, ux, uy, uz, fx, fy, fz, a.nu, a.cy_mode == CY_LOCAL_NEQ ? &cy : nullptr, Sl);
        // one running pointer over the direction arrays keeps the 27 store addresses out
        // of the register file
        const int64_t qs = a.qstride;
        if (!ODD) {
            T* p = (T*)a.df + (c + 26 * qs);
#pragma unroll
            for (int q = 0; q < 27; ++q, p -= qs) S::store(p, 0, q, f[q], a.scale);
        } else {
            T* p = (T*)a.df;
#pragma unroll
            for (int q = 0; q < 27; ++q, p += qs) S::store(p, nbr(q, 1), q, f[q], a.scale);
        }
        if ((flags & F_MACRO) || a.cy_mode == CY_REF_FD) {
            write_macro<CT>(a, c, rho, ux, uy, uz, fx, fy, fz);
            if (a.cy_mode == CY_LOCAL_NEQ) {
#pragma unroll
                for (int k = 0; k < 6; ++k) a.macro[(int64_t)(M_S11 + k) * a.N + c] = Sl[k];
            }
        }
        if (flags & F_STATS) accumulate_stats<CT>(a, c, rho, ux, uy, uz);
        if (!(rho > CT(0.25) && rho < CT(4))) atomicOr(a.err, 1);
        mass = (double)rho;
    } else if (self) {
        // GEO_INFLOW nodes (lbm_bc.h:126-129) and gathered open-plane nodes
        const int k = ch.w + __popc(selfmask & ((1u << lane) - 1u));
        CT rho, ux, uy, uz;
        if (lab == L_IN_EQ) {
            const StepCtl<CT>& ctl = a.ctl[step];
            rho = ctl.rho_eq;
            ux = g.bc_prof[3 * k] * ctl.prof_scale;
            uy = g.bc_prof[3 * k + 1] * ctl.prof_scale;
            uz = g.bc_prof[3 * k + 2] * ctl.prof_scale;
        } else {
            rho = g.bc_buf[4 * k]; ux = g.bc_buf[4 * k + 1]; uy = g.bc_buf[4 * k + 2]; uz = g.bc_buf[4 * k + 3];
        }
        const double qn = finish_node<DT, ODD>(a, flags, lab, c, x, y, z, rho, ux, uy, uz);
        if (lab == L_IN_L) q3 = qn;
        else if (lab == L_IN_R) q4 = qn;
        else if (lab == L_OUT_F) q5 = qn;
        else if (lab == L_OUT_B) q6 = qn;
    }
    if (flags & F_REDUCE) {
        const double s0 = warp_sum(mass), s1 = warp_sum(q3), s2 = warp_sum(q4), s3 = warp_sum(q5), s4 = warp_sum(q6);
        if (lane == 0) {
            if (s0 != 0.0) atomicAdd(a.red, s0);
            if (s1 != 0.0) atomicAdd(a.red + 1, s1);
            if (s2 != 0.0) atomicAdd(a.red + 2, s2);
            if (s3 != 0.0) atomicAdd(a.red + 3, s3);
            if (s4 != 0.0) atomicAdd(a.red + 4, s4);
        }
    }
}

// ---------------------------------------------------------------------------------------
// the step kernel: persistent warps walk the chunk list with a stride of all warps of the
// grid; each warp stages its next chunk in shared memory (two stages) while it computes
// the current one.  The last block to finish advances the step cursor.
// ---------------------------------------------------------------------------------------
template <int DT, int COL, bool ODD, bool SINGLE>
__global__ void __launch_bounds__(256, StepOccupancy<DT, COL>::value)
    k_step(const __grid_constant__ GroupArgs<typename Storage<DT>::CT> g)
{
    using G = Stage<DT>;
    extern __shared__ __align__(128) unsigned char smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    const uint32_t bar0 = smem_u32(smem) + 16 * wib;
    int4* const ring = (int4*)(smem + 8 * 16) + wib * kRing;
    unsigned char* const stg0 = smem + kStepSmemHead + wib * 2 * G::BYTES;
    if (lane == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar0 + 8, 1);
        fence_mbar_init();
    }
    const int n = g.n_chunks;
    const int W = (int)gridDim.x * wpb;
    const int step = *g.cursor;
    const int i0 = (int)blockIdx.x * wpb + wib;
    // the records of this warp's chunks k = 0..31 (chunk i0 + k W), refilled every 32
    {
        const int i = i0 + lane * W;
        if (i < n) ring[lane] = g.chunks[i];
    }
    __syncwarp();
    uint32_t bytes_cur = i0 < n ? issue_chunk<DT, ODD, SINGLE>(g, ring[0], stg0, bar0, lane) : 0u, bytes_nxt = 0;
    uint32_t parity = 0; // bit s: phase parity of stage s
    int s = 0, k = 0;
    bool ok = true;
    for (int i = i0; i < n; i += W, ++k, s ^= 1) {
        const int4 cur = ring[k & (kRing - 1)];
        if (((k + 1) & (kRing - 1)) == 0) {
            // refill the ring with the records of chunks k+1 .. k+32
            __syncwarp();
            const int j = i + (lane + 1) * W;
            if (j < n) ring[lane] = g.chunks[j];
            __syncwarp();
        }
        // stage the next chunk while this one computes
        bytes_nxt = i + W < n ? issue_chunk<DT, ODD, SINGLE>(g, ring[(k + 1) & (kRing - 1)], stg0 + (s ^ 1) * G::BYTES,
                                                             bar0 + 8 * (s ^ 1), lane)
                              : 0u;
        if (bytes_cur) {
            ok = __all_sync(0xffffffffu, mbar_wait(bar0 + 8 * s, (parity >> s) & 1u));
            if (!ok) {
                // a staged chunk never arrived: flag it, let the copies in flight land, stop
                if (lane == 0) atomicOr(SINGLE ? g.c0.err : g.cases[cur.z & CH_CASE_MASK].err, 2);
                mbar_wait(bar0 + 8 * s, (parity >> s) & 1u);
                if (bytes_nxt) mbar_wait(bar0 + 8 * (s ^ 1), (parity >> (s ^ 1)) & 1u);
                break;
            }
            parity ^= 1u << s;
        }
        process_chunk<DT, COL, ODD, SINGLE>(g, cur, bytes_cur ? stg0 + s * G::BYTES : nullptr, step, lane);
        // all reads of this stage are done before the next copy into it
        fence_proxy_async_smem();
        __syncwarp();
        bytes_cur = bytes_nxt;
    }
    // the last block to finish advances the step cursor (every block has read it above)
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(g.done, 1) == (int)gridDim.x - 1) {
            *g.done = 0;
            *g.cursor = step + 1;
            __threadfence();
        }
    }
}

// ---------------------------------------------------------------------------------------
// gathered open-plane nodes (the ones without a source neighbour)
// ---------------------------------------------------------------------------------------
// canonical post-collision population q of cell (x,y,z) of the previous step, in the A-A
// layout that step left behind
template <int DT, bool ODD>
__device__ __forceinline__ typename Storage<DT>::CT canon(const CaseArgs<typename Storage<DT>::CT>& a, int x, int y, int z, int q)
{
    using S = Storage<DT>;
    x = min(max(x, 0), a.nx - 1); y = min(max(y, 0), a.ny - 1); z = min(max(z, 0), a.nz - 1);
    const int sy = a.nx, sz = a.nx * a.ny;
    if (ODD) // the previous (even) step stored f*_q of x in slot opp(q) at x
        return S::load(qptr<DT>(a, oppq(q)), x + sy * y + sz * z, q, a.inv_scale);
    // the previous (odd) step, or the initial state, stored f*_q of x in slot q at x + c_q
    return S::load(qptr<DT>(a, q), wrapc(x + cxq(q), a.nx) + sy * wrapc(y + cyq(q), a.ny) + sz * wrapc(z + czq(q), a.nz), q,
                   a.inv_scale);
}

// LBM_STREAMING::streaming with explicit (m, centre, p) triples (lbm_streaming.h:10-39)
template <int DT, bool ODD>
__device__ __forceinline__ void pull_triples(const CaseArgs<typename Storage<DT>::CT>& a, const int* xs, const int* ys, const int* zs,
                                             typename Storage<DT>::CT* f)
{
#pragma unroll
    for (int q = 0; q < 27; ++q) f[q] = canon<DT, ODD>(a, xs[1 - cxq(q)], ys[1 - cyq(q)], zs[1 - czq(q)], q);
}

template <int DT, bool ODD>
__global__ void __launch_bounds__(128) k_bc_gather(const __grid_constant__ GroupArgs<typename Storage<DT>::CT> g)
{
    using CT = typename Storage<DT>::CT;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.n_gather) return;
    const int4 e = g.gather[t];
    const CaseArgs<CT>& a = g.cases[e.y];
    const StepCtl<CT>& ctl = a.ctl[*g.cursor];
    const int c = e.x, k = e.z;
    const int lab = a.label[c] & L_MASK;
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
    const int4 ch = g.chunks[warp];
    const CaseArgs<CT>& a = g.cases[ch.z & CH_CASE_MASK];
    if (a.cy_mode != CY_REF_FD) return;
    const int y = ch.y & 0xffff, z = ch.y >> 16;
    const int x = ch.x - y * a.nx - z * a.nx * a.ny + lane;
    const int c = ch.x + lane;
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
    const int4 ch = g.chunks[warp];
    const CaseArgs<CT>& a = g.cases[ch.z & CH_CASE_MASK];
    if (a.cy_mode != CY_REF_FD) return;
    const int sy = a.nx, sz = a.nx * a.ny;
    const int y = ch.y & 0xffff, z = ch.y >> 16;
    const int x = ch.x - y * sy - z * sz + lane;
    const int c = ch.x + lane;
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
// host-side dispatch: one function per (storage, collision) instantiated in its own
// translation unit
// ---------------------------------------------------------------------------------------
using GroupLauncher = void (*)(bool odd, dim3 grid, dim3 block, cudaStream_t s, const void* group_args);

// launch of one step-kernel variant: the dynamic shared memory is opted in once per
// device, and the grid is capped at the blocks that are resident at once (persistent)
template <int DT, int COL, bool ODD, bool SINGLE>
void launch_step_variant(dim3 grid, dim3 block, cudaStream_t s, const GroupArgs<typename Storage<DT>::CT>& g)
{
    auto kern = k_step<DT, COL, ODD, SINGLE>;
    const int smem = step_smem_bytes<DT>((int)block.x / 32);
    static std::atomic<unsigned long long> attr_set{0};
    static std::atomic<int> resident[9] = {};  // per block size / 32
    static std::atomic<int> sm_count{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(attr_set.load() & bit)) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, step_smem_bytes<DT>(8));
        attr_set.fetch_or(bit);
    }
    const int wpb = (int)block.x / 32;
    if (wpb < 1 || wpb > 8) return;
    if (!resident[wpb].load()) {
        int nb = 0, sms = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, (int)block.x, smem);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        sm_count.store(std::max(sms, 1));
        resident[wpb].store(std::max(nb, 1));
    }
    const unsigned cap = (unsigned)(resident[wpb].load() * sm_count.load());
    const dim3 gr(std::max(1u, std::min(grid.x, cap)));
    kern<<<gr, block, smem, s>>>(g);
}

template <int DT, int COL>
void launch_step(bool odd, dim3 grid, dim3 block, cudaStream_t s, const void* args)
{
    using CT = typename Storage<DT>::CT;
    const GroupArgs<CT>& g = *(const GroupArgs<CT>*)args;
    if (g.n_cases == 1) {
        if (odd) launch_step_variant<DT, COL, true, true>(grid, block, s, g);
        else launch_step_variant<DT, COL, false, true>(grid, block, s, g);
    } else {
        if (odd) launch_step_variant<DT, COL, true, false>(grid, block, s, g);
        else launch_step_variant<DT, COL, false, false>(grid, block, s, g);
    }
}

GroupLauncher step_launcher(int dtype, int collision);

} // namespace nnlbm
