// nnlbm_step_inst.cu -- explicit instantiation of the step kernel for one storage type
// (NNLBM_DT) and one collision (NNLBM_COL).  The build compiles this file once per pair so
// that the 44 kernels compile in parallel and FP64 units can use IEEE-exact flags.
#include "nnlbm_kernels.cuh"

#ifndef NNLBM_DT
#error "NNLBM_DT must be defined"
#endif
#ifndef NNLBM_COL
#error "NNLBM_COL must be defined"
#endif

#define NNLBM_CAT2(a, b, c) a##b##_##c
#define NNLBM_CAT(a, b, c) NNLBM_CAT2(a, b, c)

namespace nnlbm {
void NNLBM_CAT(launch_step_, NNLBM_DT, NNLBM_COL)(bool odd, bool after_gather, int form, dim3 grid, dim3 block,
                                                cudaStream_t s, const void* args)
{
    launch_step<NNLBM_DT, NNLBM_COL>(odd, after_gather, form, grid, block, s, args);
}

cudaError_t NNLBM_CAT(load_step_, NNLBM_DT, NNLBM_COL)() { return load_step<NNLBM_DT, NNLBM_COL>(); }

int NNLBM_CAT(staged_blocks_, NNLBM_DT, NNLBM_COL)() { return staged_blocks<NNLBM_DT, NNLBM_COL>(); }
} // namespace nnlbm
