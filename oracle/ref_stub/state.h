// Stand-in for solver/lbm3d/state.h when solver/lbm3d/core.h is compiled on the host by
// oracle/ref_shim.cpp (test infrastructure only).  The real header brings the State class,
// VTK output, checkpoints and the MPI communicator.  core.h's driver templates (SimUpdate,
// AfterSimUpdate, execute) are never instantiated by the shim, but the names they use
// outside their template parameters must exist: the counter and sparse-solver enums and
// the communicator calls, declared here as no-ops.
#pragma once

enum { ws_computeCPU, ws_computeCPU_TNL, ws_computeGPU_TNL, ws_computeHybrid_TNL, ws_computeHybrid_TNL_zerocopy,
       ws_computeGPU_CUSPARSE, ws_computeHybrid_CUSPARSE };
enum { PRINT, VTK1D, VTK2D, VTK3D, VTK3DCUT, PROBE1, PROBE2, PROBE3, STAT_RESET, STAT2_RESET, SAVESTATE, MAX_COUNTER };
enum { MPI_LOR };

struct TNLMPI {
    template <typename... A> static void Allreduce(A&&...) {}
    template <typename... A> static void Bcast(A&&...) {}
    template <typename... A> static void Barrier(A&&...) {}
    static constexpr int AllGroup = 0;
};
