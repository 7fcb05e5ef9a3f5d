// nnlbm_bc_inst.cu -- the open-plane gather, the CY_REF_FD phase kernels and the
// initial-state fills for one storage type (NNLBM_DT).
#include "nnlbm_kernels.cuh"

#ifndef NNLBM_DT
#error "NNLBM_DT must be defined"
#endif

#define NNLBM_CAT2(a, b) a##b
#define NNLBM_CAT(a, b) NNLBM_CAT2(a, b)

namespace nnlbm {

// every slot q of every cell <- feq_q(rho, u): a uniform state is valid in either A-A layout.
// With halfway bounce-back the layout an odd step leaves (the one written here) keeps a
// non-wall cell's population opp(q) in its own slot q where x - c_q is a wall.
template <int DT>
__global__ void k_fill_eq(const CaseArgs<typename Storage<DT>::CT> a, typename Storage<DT>::CT rho, typename Storage<DT>::CT ux,
                          typename Storage<DT>::CT uy, typename Storage<DT>::CT uz)
{
    using S = Storage<DT>;
    using CT = typename S::CT;
    CT f[27];
    equilibrium<CT>(a.eq, rho, ux, uy, uz, f);
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < a.N; c += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t m = (a.hw && (a.label[c] & L_MASK) != L_WALL) ? a.hw[c] : 0u;
#pragma unroll
        for (int q = 0; q < 27; ++q) S::store(qptr<DT>(a, q), (int)c, q, ((m >> oppq(q)) & 1u) ? f[oppq(q)] : f[q], a.scale);
    }
}

// initial macro state (LBMKernelInit, core.h:833-863): rho/u from f at FLUID and PERIODIC
// cells, rho = 1 and u = 0 elsewhere, F = the homogeneous force, S = 0
template <int DT>
__global__ void k_init_macro(const CaseArgs<typename Storage<DT>::CT> a, typename Storage<DT>::CT rho0, typename Storage<DT>::CT ux0,
                             typename Storage<DT>::CT uy0, typename Storage<DT>::CT uz0)
{
    using CT = typename Storage<DT>::CT;
    CT f[27];
    equilibrium<CT>(a.eq, rho0, ux0, uy0, uz0, f);
    CT r, u, v, w;
    density_velocity<CT>(f, a.fx, a.fy, a.fz, r, u, v, w);
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < a.N; c += (int64_t)gridDim.x * blockDim.x) {
        const int lab = a.label[c] & L_MASK;
        const bool fl = lab == L_FLUID || lab == L_PERIODIC;
        CT* M = a.macro;
        M[M_RHO * a.N + c] = fl ? r : CT(1);
        M[M_VX * a.N + c] = fl ? u : CT(0);
        M[M_VY * a.N + c] = fl ? v : CT(0);
        M[M_VZ * a.N + c] = fl ? w : CT(0);
        M[M_FX * a.N + c] = a.fx; M[M_FY * a.N + c] = a.fy; M[M_FZ * a.N + c] = a.fz;
        for (int k = M_S11; k <= M_S33; ++k) M[k * a.N + c] = CT(0);
    }
}

void NNLBM_CAT(launch_bc_gather_, NNLBM_DT)(bool odd, dim3 grid, dim3 block, cudaStream_t s, const void* args)
{
    using CT = typename Storage<NNLBM_DT>::CT;
    const GroupArgs<CT>& g = *(const GroupArgs<CT>*)args;
    switch (args_mode(g.n_cases)) {
    case ARGS_ONE:
        if (odd) k_bc_gather<NNLBM_DT, true, ARGS_ONE><<<grid, block, 0, s>>>(g);
        else k_bc_gather<NNLBM_DT, false, ARGS_ONE><<<grid, block, 0, s>>>(g);
        break;
    case ARGS_PARAM:
        if (odd) k_bc_gather<NNLBM_DT, true, ARGS_PARAM><<<grid, block, 0, s>>>(g);
        else k_bc_gather<NNLBM_DT, false, ARGS_PARAM><<<grid, block, 0, s>>>(g);
        break;
    default:
        if (odd) k_bc_gather<NNLBM_DT, true, ARGS_GLOBAL><<<grid, block, 0, s>>>(g);
        else k_bc_gather<NNLBM_DT, false, ARGS_GLOBAL><<<grid, block, 0, s>>>(g);
    }
}

void NNLBM_CAT(launch_refd_velocity_, NNLBM_DT)(bool odd, dim3 grid, dim3 block, cudaStream_t s, const void* args)
{
    using CT = typename Storage<NNLBM_DT>::CT;
    const GroupArgs<CT>& g = *(const GroupArgs<CT>*)args;
    if (odd) k_refd_velocity<NNLBM_DT, true><<<grid, block, 0, s>>>(g);
    else k_refd_velocity<NNLBM_DT, false><<<grid, block, 0, s>>>(g);
}

void NNLBM_CAT(launch_refd_stress_, NNLBM_DT)(bool, dim3 grid, dim3 block, cudaStream_t s, const void* args)
{
    using CT = typename Storage<NNLBM_DT>::CT;
    k_refd_stress<CT><<<grid, block, 0, s>>>(*(const GroupArgs<CT>*)args);
}

void NNLBM_CAT(launch_fill_eq_, NNLBM_DT)(const void* args, double rho, double ux, double uy, double uz, cudaStream_t s)
{
    using CT = typename Storage<NNLBM_DT>::CT;
    k_fill_eq<NNLBM_DT><<<148 * 8, 256, 0, s>>>(*(const CaseArgs<CT>*)args, (CT)rho, (CT)ux, (CT)uy, (CT)uz);
}

void NNLBM_CAT(launch_init_macro_, NNLBM_DT)(const void* args, double rho, double ux, double uy, double uz, cudaStream_t s)
{
    using CT = typename Storage<NNLBM_DT>::CT;
    k_init_macro<NNLBM_DT><<<148 * 8, 256, 0, s>>>(*(const CaseArgs<CT>*)args, (CT)rho, (CT)ux, (CT)uy, (CT)uz);
}

void NNLBM_CAT(launch_output_fields_, NNLBM_DT)(const void* args, const OutputParams& p, const uint8_t* wall, float* out,
                                              cudaStream_t s)
{
    using CT = typename Storage<NNLBM_DT>::CT;
    k_output_fields<CT><<<148 * 8, 256, 0, s>>>(*(const CaseArgs<CT>*)args, p, wall, out);
}

// every kernel of this translation unit resolved now (see load_step in nnlbm_kernels.cuh)
cudaError_t NNLBM_CAT(load_bc_, NNLBM_DT)()
{
    using CT = typename Storage<NNLBM_DT>::CT;
    const void* fns[] = {(const void*)k_bc_gather<NNLBM_DT, false, ARGS_ONE>, (const void*)k_bc_gather<NNLBM_DT, true, ARGS_ONE>,
                         (const void*)k_bc_gather<NNLBM_DT, false, ARGS_PARAM>, (const void*)k_bc_gather<NNLBM_DT, true, ARGS_PARAM>,
                         (const void*)k_bc_gather<NNLBM_DT, false, ARGS_GLOBAL>, (const void*)k_bc_gather<NNLBM_DT, true, ARGS_GLOBAL>,
                         (const void*)k_refd_velocity<NNLBM_DT, false>, (const void*)k_refd_velocity<NNLBM_DT, true>,
                         (const void*)k_refd_stress<CT>, (const void*)k_fill_eq<NNLBM_DT>, (const void*)k_init_macro<NNLBM_DT>,
                         (const void*)k_output_fields<CT>};
    cudaFuncAttributes fa;
    for (const void* f : fns) {
        const cudaError_t e = cudaFuncGetAttributes(&fa, f);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

} // namespace nnlbm
