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
// The open-plane nodes (TCPC inflow/outflow, generic GEO_INFLOW / GEO_OUTFLOW_RIGHT_EQ) pull
// a re-centred stencil from a neighbour (sim_tcpc.cu:242-273, lbm_bc.h:126-152).  Those
// reads touch slots that the neighbour overwrites in the same step, so one step is three
// launches: k_bc_gather (the re-centred moments of every boundary node, before anything is
// written), k_step (FLUID and PERIODIC cells), k_bc_write (equilibria of the boundary
// nodes into their own slots).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "nnlbm_physics.cuh"

namespace nnlbm {

enum : int { L_FLUID = 0, L_WALL = 1, L_PERIODIC = 2, L_IN_L = 3, L_IN_R = 4, L_OUT_F = 5, L_OUT_B = 6,
             L_IN_EQ = 7, L_OUT_REQ = 8 };
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
    __device__ static __forceinline__ CT load(const T* p, int i, int, CT) { return p[i]; }
    __device__ static __forceinline__ void store(T* p, int i, int, CT v, CT) { p[i] = v; }
};
template <> struct Storage<1> {
    using T = float; using CT = float;
    __device__ static __forceinline__ CT load(const T* p, int i, int q, CT) { return weight<float>(q) + p[i]; }
    __device__ static __forceinline__ void store(T* p, int i, int q, CT v, CT) { p[i] = v - weight<float>(q); }
};
template <> struct Storage<2> {
    using T = __half; using CT = float;
    __device__ static __forceinline__ CT load(const T* p, int i, int q, CT isc) { return weight<float>(q) + __half2float(p[i]) * isc; }
    __device__ static __forceinline__ void store(T* p, int i, int q, CT v, CT sc) { p[i] = __float2half_rn((v - weight<float>(q)) * sc); }
};
template <> struct Storage<3> {
    using T = __nv_bfloat16; using CT = float;
    __device__ static __forceinline__ CT load(const T* p, int i, int q, CT isc) { return weight<float>(q) + __bfloat162float(p[i]) * isc; }
    __device__ static __forceinline__ void store(T* p, int i, int q, CT v, CT sc) { p[i] = __float2bfloat16_rn((v - weight<float>(q)) * sc); }
};

// per-step control word written by the host before each nnlbm_step call and indexed by a
// device cursor that k_bc_write advances, so a captured graph replays any schedule
template <class CT>
struct StepCtl {
    int flags;
    int pad;
    CT u_left, u_right;   // plug velocities of the IVC / SVC planes (flux / area, SVC negative)
    CT rho_left, rho_right, rho_eq, prof_scale;
};

template <class CT>
struct KArgs {
    void* dfq[27];             // per-direction base pointers
    const uint8_t* label;      // [N]
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
    int* cursor;
    int* done;                 // block counter of k_bc_write
    double* red;               // [5] mass, Q_ivc, Q_svc, Q_out5, Q_out6
    int* err;                  // watchdog flag
    const int32_t* bc_cell;    // [n_bc] cell index of every open-plane node
    const CT* bc_prof;         // [n_bc][3] prescribed velocity (INFLOW_EQ nodes)
    CT* bc_buf;                // [n_bc][4] rho, ux, uy, uz of the current step
    int n_bc, pad2;
};

__device__ __forceinline__ int wrapc(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

template <class CT>
__device__ __forceinline__ void warp_add_double(double v, double* dst)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x + blockDim.x * threadIdx.y) % 32 == 0 && v != 0.0) atomicAdd(dst, v);
}

template <class CT>
__device__ __forceinline__ void accumulate_stats(const KArgs<CT>& a, int64_t c, CT rho, CT ux, CT uy, CT uz)
{
    // MacroTcpc::outputMacro (sim_tcpc.cu:347-353); the sign split of rho*ux is summed
    const CT jx = rho * ux, jy = rho * uy, jz = rho * uz;
    if (a.stats_f64) {
        double* s = (double*)a.stats;
        s[c] += (double)jx; s[a.N + c] += (double)jy; s[2 * a.N + c] += (double)jz;
        s[3 * a.N + c] += (double)jx * (double)jx; s[4 * a.N + c] += (double)jy * (double)jy;
        s[5 * a.N + c] += (double)jz * (double)jz;
    } else {
        float* s = (float*)a.stats;
        s[c] += (float)jx; s[a.N + c] += (float)jy; s[2 * a.N + c] += (float)jz;
        s[3 * a.N + c] += (float)(jx * jx); s[4 * a.N + c] += (float)(jy * jy); s[5 * a.N + c] += (float)(jz * jz);
    }
}

// ---------------------------------------------------------------------------------------
// the fused step for FLUID and PERIODIC cells (solver/lbm3d/core.h:578-800)
// ---------------------------------------------------------------------------------------
// minimum resident blocks of 256 threads: the register budget of each variant (FP64
// arithmetic and the KBC family need more live values than the cumulant in FP32)
template <int DT, int COL>
struct StepOccupancy {
    static constexpr int value = DT == 0 ? 1 : ((COL >= COL_KBC_N1 && COL <= COL_KBC_C4) ? 2 : 3);
};

template <int DT, int COL, bool ODD>
__global__ void __launch_bounds__(256, StepOccupancy<DT, COL>::value) k_step(const KArgs<typename Storage<DT>::CT> a)
{
    using S = Storage<DT>;
    using CT = typename S::CT;
    using T = typename S::T;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    const bool inb = x < a.nx && y < a.ny;
    // cell indices fit in 32 bits (nnlbm_create rejects lattices of 2^31 cells or more)
    const int sy = a.nx, sz = a.nx * a.ny;
    const int c = inb ? x + sy * y + sz * z : 0;
    const int lab = inb ? (int)a.label[c] : 255;
    const bool active = lab == L_FLUID || lab == L_PERIODIC;
    const int flags = a.ctl[*a.cursor].flags;
    double mass = 0.0;
    if (active) {
        const bool interior = x > 0 && x < a.nx - 1 && y > 0 && y < a.ny - 1 && z > 0 && z < a.nz - 1;
        CT f[27];
        if (!ODD) {
#pragma unroll
            for (int q = 0; q < 27; ++q) f[q] = S::load((const T*)a.dfq[q], c, q, a.inv_scale);
        } else {
#pragma unroll
            for (int q = 0; q < 27; ++q) {
                const int nb = interior ? c - (cxq(q) + sy * cyq(q) + sz * czq(q))
                                        : wrapc(x - cxq(q), a.nx) + sy * wrapc(y - cyq(q), a.ny) + sz * wrapc(z - czq(q), a.nz);
                f[q] = S::load((const T*)a.dfq[oppq(q)], nb, q, a.inv_scale);
            }
        }
        CT fx = a.fx, fy = a.fy, fz = a.fz;
        if (a.cy_mode == CY_REF_FD && lab == L_FLUID) {
            // core.h:663-781: divergence of the finite-difference strain of the previous
            // phase with one-sided differences next to non-FLUID cells, then the CY force
            // 2 (nu(gamma) - nu) F rho with rho still at its default of 1
            const CT* M = a.macro;
            const int64_t N = a.N;
            const int cn[6] = {c - 1, c + 1, c - sy, c + sy, c - sz, c + sz};
            bool fl[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) fl[k] = a.label[cn[k]] == L_FLUID;
            auto d1 = [&](int fld, int axis) -> CT {
                const bool m = fl[2 * axis], p = fl[2 * axis + 1];
                const CT* F = M + (int64_t)fld * N;
                if (!m) return p ? F[cn[2 * axis + 1]] - F[c] : CT(0);
                if (!p) return F[c] - F[cn[2 * axis]];
                return CT(0.5) * (F[cn[2 * axis + 1]] - F[cn[2 * axis]]);
            };
            const CT F1 = d1(M_S11, 0) + d1(M_S12, 1) + d1(M_S13, 2);
            const CT F2 = d1(M_S12, 0) + d1(M_S22, 1) + d1(M_S32, 2);
            const CT F3 = d1(M_S13, 0) + d1(M_S32, 1) + d1(M_S33, 2);
            const CT S11 = M[M_S11 * N + c], S12 = M[M_S12 * N + c], S13 = M[M_S13 * N + c];
            const CT S22 = M[M_S22 * N + c], S32 = M[M_S32 * N + c], S33 = M[M_S33 * N + c];
            const CT gam = dsqrt<CT>(CT(2)) * dsqrt<CT>(S11 * S11 + S22 * S22 + S33 * S33 + CT(2) * (S12 * S12 + S13 * S13 + S32 * S32));
            // single precision powf as in the reference
            const CT nuc = a.nu + (a.nu0 - a.nu) * (CT)powf((float)(CT(1) + (CT)powf((float)(gam * a.lam), (float)a.a)),
                                                           (float)((a.n - CT(1)) / a.a));
            fx += CT(2) * (nuc - a.nu) * F1;
            fy += CT(2) * (nuc - a.nu) * F2;
            fz += CT(2) * (nuc - a.nu) * F3;
        }
        CT rho, ux, uy, uz;
        density_velocity<CT>(f, fx, fy, fz, rho, ux, uy, uz);
        CT nu = a.nu;
        CT Sl[6];
        if (a.cy_mode == CY_LOCAL_NEQ) nu = local_nu<CT>(f, rho, ux, uy, uz, a.nu, a.nu0, a.lam, a.a, a.n, Sl);
        collide<CT, COL>(f, rho, ux, uy, uz, fx, fy, fz, nu);
        if (!ODD) {
#pragma unroll
            for (int q = 0; q < 27; ++q) S::store((T*)a.dfq[oppq(q)], c, q, f[q], a.scale);
        } else {
#pragma unroll
            for (int q = 0; q < 27; ++q) {
                const int nb = interior ? c + (cxq(q) + sy * cyq(q) + sz * czq(q))
                                        : wrapc(x + cxq(q), a.nx) + sy * wrapc(y + cyq(q), a.ny) + sz * wrapc(z + czq(q), a.nz);
                S::store((T*)a.dfq[q], nb, q, f[q], a.scale);
            }
        }
        if ((flags & F_MACRO) || a.cy_mode == CY_REF_FD) {
            CT* M = a.macro;
            const int64_t N = a.N;
            M[M_RHO * N + c] = rho; M[M_VX * N + c] = ux; M[M_VY * N + c] = uy; M[M_VZ * N + c] = uz;
            M[M_FX * N + c] = fx; M[M_FY * N + c] = fy; M[M_FZ * N + c] = fz;
            if (a.cy_mode == CY_LOCAL_NEQ) {
#pragma unroll
                for (int k = 0; k < 6; ++k) M[(M_S11 + k) * N + c] = Sl[k];
            }
        }
        if (flags & F_STATS) accumulate_stats<CT>(a, c, rho, ux, uy, uz);
        if (!(rho > CT(0.25) && rho < CT(4))) atomicOr(a.err, 1);
        mass = (double)rho;
    }
    if (flags & F_REDUCE) warp_add_double<CT>(mass, a.red);
}

// ---------------------------------------------------------------------------------------
// open-plane nodes
// ---------------------------------------------------------------------------------------
// canonical post-collision population q of cell (x,y,z) of the previous step, in the A-A
// layout that step left behind
template <int DT, bool ODD>
__device__ __forceinline__ typename Storage<DT>::CT canon(const KArgs<typename Storage<DT>::CT>& a, int x, int y, int z, int q)
{
    using S = Storage<DT>;
    using T = typename S::T;
    x = min(max(x, 0), a.nx - 1); y = min(max(y, 0), a.ny - 1); z = min(max(z, 0), a.nz - 1);
    const int sy = a.nx, sz = a.nx * a.ny;
    if (ODD) // the previous (even) step stored f*_q of x in slot opp(q) at x
        return S::load((const T*)a.dfq[oppq(q)], x + sy * y + sz * z, q, a.inv_scale);
    // the previous (odd) step, or the initial state, stored f*_q of x in slot q at x + c_q
    return S::load((const T*)a.dfq[q], wrapc(x + cxq(q), a.nx) + sy * wrapc(y + cyq(q), a.ny) + sz * wrapc(z + czq(q), a.nz), q,
                   a.inv_scale);
}

// LBM_STREAMING::streaming with explicit (m, centre, p) triples (lbm_streaming.h:10-39)
template <int DT, bool ODD>
__device__ __forceinline__ void pull_triples(const KArgs<typename Storage<DT>::CT>& a, const int* xs, const int* ys, const int* zs,
                                             typename Storage<DT>::CT* f)
{
#pragma unroll
    for (int q = 0; q < 27; ++q) f[q] = canon<DT, ODD>(a, xs[1 - cxq(q)], ys[1 - cyq(q)], zs[1 - czq(q)], q);
}

template <int DT, bool ODD>
__global__ void __launch_bounds__(128) k_bc_gather(const KArgs<typename Storage<DT>::CT> a)
{
    using CT = typename Storage<DT>::CT;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const StepCtl<CT> ctl = a.ctl[*a.cursor];
    if (k == 0 && (ctl.flags & F_REDUCE)) {
        for (int i = 0; i < 5; ++i) a.red[i] = 0.0;
    }
    if (k >= a.n_bc) return;
    const int c = a.bc_cell[k];
    const int lab = a.label[c];
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
    case L_IN_EQ: // lbm_bc.h:126-129
        rho = ctl.rho_eq;
        ux = a.bc_prof[3 * k] * ctl.prof_scale;
        uy = a.bc_prof[3 * k + 1] * ctl.prof_scale;
        uz = a.bc_prof[3 * k + 2] * ctl.prof_scale;
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
    a.bc_buf[4 * k] = rho; a.bc_buf[4 * k + 1] = ux; a.bc_buf[4 * k + 2] = uy; a.bc_buf[4 * k + 3] = uz;
}

template <int DT, bool ODD>
__global__ void __launch_bounds__(128) k_bc_write(const KArgs<typename Storage<DT>::CT> a)
{
    using S = Storage<DT>;
    using CT = typename S::CT;
    using T = typename S::T;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int cur = *a.cursor;
    const StepCtl<CT> ctl = a.ctl[cur];
    double q3 = 0, q4 = 0, q5 = 0, q6 = 0;
    if (k < a.n_bc) {
        const int c = a.bc_cell[k];
        const int lab = a.label[c];
        const int x = c % a.nx, y = (c / a.nx) % a.ny, z = c / (a.nx * a.ny);
        const CT rho = a.bc_buf[4 * k], ux = a.bc_buf[4 * k + 1], uy = a.bc_buf[4 * k + 2], uz = a.bc_buf[4 * k + 3];
        CT f[27];
        equilibrium<CT>(a.eq, rho, ux, uy, uz, f);
        const int sy = a.nx, sz = a.nx * a.ny;
        if (!ODD) {
#pragma unroll
            for (int q = 0; q < 27; ++q) S::store((T*)a.dfq[oppq(q)], c, q, f[q], a.scale);
        } else {
#pragma unroll
            for (int q = 0; q < 27; ++q)
                S::store((T*)a.dfq[q], wrapc(x + cxq(q), a.nx) + sy * wrapc(y + cyq(q), a.ny) + sz * wrapc(z + czq(q), a.nz), q, f[q],
                         a.scale);
        }
        if (ctl.flags & F_MACRO || a.cy_mode == CY_REF_FD) {
            CT* M = a.macro;
            const int64_t N = a.N;
            M[M_RHO * N + c] = rho; M[M_VX * N + c] = ux; M[M_VY * N + c] = uy; M[M_VZ * N + c] = uz;
            M[M_FX * N + c] = a.fx; M[M_FY * N + c] = a.fy; M[M_FZ * N + c] = a.fz;
        }
        if (ctl.flags & F_STATS) accumulate_stats<CT>(a, c, rho, ux, uy, uz);
        if (ctl.flags & F_REDUCE) {
            if (lab == L_IN_L) q3 = (double)ux;
            if (lab == L_IN_R) q4 = -(double)ux;
            if (lab == L_OUT_F) q5 = -(double)uy;
            if (lab == L_OUT_B) q6 = (double)uy;
        }
    }
    if (ctl.flags & F_REDUCE) {
        warp_add_double<CT>(q3, a.red + 1);
        warp_add_double<CT>(q4, a.red + 2);
        warp_add_double<CT>(q5, a.red + 3);
        warp_add_double<CT>(q6, a.red + 4);
    }
    // the last block to finish advances the step cursor (every block has read it above)
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const int prev = atomicAdd(a.done, 1);
        if (prev == (int)gridDim.x - 1) {
            *a.done = 0;
            *a.cursor = cur + 1;
            __threadfence();
        }
    }
}

// ---------------------------------------------------------------------------------------
// NNLBM_CY_REF_FD phases 1 and 2 (core.h:1176-1258): velocity of the post-streaming state
// of every FLUID cell with the force of the previous step, then the finite-difference
// strain from it.  Non-FLUID values are never read by the strain stencil.
// ---------------------------------------------------------------------------------------
template <int DT, bool ODD>
__global__ void __launch_bounds__(256) k_refd_velocity(const KArgs<typename Storage<DT>::CT> a)
{
    using CT = typename Storage<DT>::CT;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const int64_t c = (int64_t)x + (int64_t)a.nx * ((int64_t)y + (int64_t)a.ny * z);
    if (a.label[c] != L_FLUID) return;
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
__global__ void __launch_bounds__(256) k_refd_stress(const KArgs<CT> a)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const int64_t sy = a.nx, sz = (int64_t)a.nx * a.ny;
    const int64_t c = (int64_t)x + sy * y + sz * z;
    if (a.label[c] != L_FLUID) return;
    CT* M = a.macro;
    const int64_t N = a.N;
    const int64_t cn[6] = {c - 1, c + 1, c - sy, c + sy, c - sz, c + sz};
    bool fl[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) fl[k] = a.label[cn[k]] == L_FLUID;
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
using StepLauncher = void (*)(bool odd, dim3 grid, dim3 block, cudaStream_t s, const void* args);

template <int DT, int COL>
void launch_step(bool odd, dim3 grid, dim3 block, cudaStream_t s, const void* args)
{
    using CT = typename Storage<DT>::CT;
    const KArgs<CT>& a = *(const KArgs<CT>*)args;
    if (odd) k_step<DT, COL, true><<<grid, block, 0, s>>>(a);
    else k_step<DT, COL, false><<<grid, block, 0, s>>>(a);
}

StepLauncher step_launcher(int dtype, int collision);

} // namespace nnlbm
