// nnlbm_capi.cu -- the C ABI of libnnlbm.so (declared in include/nnlbm.h): contexts, device
// buffers, the TCPC boundary setup, the packed work lists, the per-step launch sequence of
// each launch group and its CUDA graphs.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/nnlbm.h"
#include "nnlbm_kernels.cuh"

namespace nnlbm {
#define NNLBM_DECL_STEP(DT, COL)                                                                  \
    void launch_step_##DT##_##COL(bool, bool, int, dim3, dim3, cudaStream_t, const void*); \
    cudaError_t load_step_##DT##_##COL();                                                  \
    int staged_blocks_##DT##_##COL();
#define NNLBM_DECL_STEP_DT(DT)                                                                                        \
    NNLBM_DECL_STEP(DT, 0) NNLBM_DECL_STEP(DT, 1) NNLBM_DECL_STEP(DT, 2) NNLBM_DECL_STEP(DT, 3) NNLBM_DECL_STEP(DT, 4) \
    NNLBM_DECL_STEP(DT, 5) NNLBM_DECL_STEP(DT, 6) NNLBM_DECL_STEP(DT, 7) NNLBM_DECL_STEP(DT, 8) NNLBM_DECL_STEP(DT, 9) \
    NNLBM_DECL_STEP(DT, 10)
NNLBM_DECL_STEP_DT(0) NNLBM_DECL_STEP_DT(1) NNLBM_DECL_STEP_DT(2) NNLBM_DECL_STEP_DT(3)
#define NNLBM_DECL_AUX(DT)                                                                \
    void launch_bc_gather_##DT(bool, dim3, dim3, cudaStream_t, const void*);             \
    void launch_refd_velocity_##DT(bool, dim3, dim3, cudaStream_t, const void*);         \
    void launch_refd_stress_##DT(bool, dim3, dim3, cudaStream_t, const void*);           \
    void launch_fill_eq_##DT(const void*, double, double, double, double, cudaStream_t); \
    void launch_init_macro_##DT(const void*, double, double, double, double, cudaStream_t); \
    void launch_output_fields_##DT(const void*, const OutputParams&, const uint8_t*, float*, cudaStream_t); \
    cudaError_t load_bc_##DT();
NNLBM_DECL_AUX(0) NNLBM_DECL_AUX(1) NNLBM_DECL_AUX(2) NNLBM_DECL_AUX(3)

// the loaders of every kernel a launch group of (storage, collision) can launch
static cudaError_t load_group_kernels(int dt, int col)
{
#define NNLBM_LROW(DT)                                                                                            \
    {load_step_##DT##_0, load_step_##DT##_1, load_step_##DT##_2, load_step_##DT##_3, load_step_##DT##_4,         \
     load_step_##DT##_5, load_step_##DT##_6, load_step_##DT##_7, load_step_##DT##_8, load_step_##DT##_9,         \
     load_step_##DT##_10}
    static cudaError_t (*const step[4][11])() = {NNLBM_LROW(0), NNLBM_LROW(1), NNLBM_LROW(2), NNLBM_LROW(3)};
    static cudaError_t (*const bc[4])() = {load_bc_0, load_bc_1, load_bc_2, load_bc_3};
    const cudaError_t e = step[dt][col]();
    return e != cudaSuccess ? e : bc[dt]();
}

StepLauncher step_launcher(int dt, int col)
{
#define NNLBM_ROW(DT)                                                                                     \
    {launch_step_##DT##_0, launch_step_##DT##_1, launch_step_##DT##_2, launch_step_##DT##_3,             \
     launch_step_##DT##_4, launch_step_##DT##_5, launch_step_##DT##_6, launch_step_##DT##_7,             \
     launch_step_##DT##_8, launch_step_##DT##_9, launch_step_##DT##_10}
    static const StepLauncher table[4][11] = {NNLBM_ROW(0), NNLBM_ROW(1), NNLBM_ROW(2), NNLBM_ROW(3)};
    return table[dt][col];
}

StagedOccupancy staged_occupancy(int dt, int col)
{
#define NNLBM_OROW(DT)                                                                                    \
    {staged_blocks_##DT##_0, staged_blocks_##DT##_1, staged_blocks_##DT##_2, staged_blocks_##DT##_3,     \
     staged_blocks_##DT##_4, staged_blocks_##DT##_5, staged_blocks_##DT##_6, staged_blocks_##DT##_7,     \
     staged_blocks_##DT##_8, staged_blocks_##DT##_9, staged_blocks_##DT##_10}
    static const StagedOccupancy table[4][11] = {NNLBM_OROW(0), NNLBM_OROW(1), NNLBM_OROW(2), NNLBM_OROW(3)};
    return table[dt][col];
}

struct AuxLaunchers {
    GroupLauncher gather, refd_velocity, refd_stress;
    void (*fill_eq)(const void*, double, double, double, double, cudaStream_t);
    void (*init_macro)(const void*, double, double, double, double, cudaStream_t);
    void (*output_fields)(const void*, const OutputParams&, const uint8_t*, float*, cudaStream_t);
};
static const AuxLaunchers& aux_launchers(int dt)
{
#define NNLBM_AUXROW(DT)                                                                                   \
    {launch_bc_gather_##DT, launch_refd_velocity_##DT, launch_refd_stress_##DT, launch_fill_eq_##DT,     \
     launch_init_macro_##DT, launch_output_fields_##DT}
    static const AuxLaunchers t[4] = {NNLBM_AUXROW(0), NNLBM_AUXROW(1), NNLBM_AUXROW(2), NNLBM_AUXROW(3)};
    return t[dt];
}
} // namespace nnlbm

using namespace nnlbm;

namespace {

const int kStorageBytes[4] = {8, 4, 2, 2};
const int kChunk = 32;
// which open-plane node a cell finishes (per cell while the work list is built)
enum : uint8_t { kServeXneg = 1, kServeXpos = 2, kServeXreq = 4, kServeYneg = 8, kServeYpos = 16 };
// slack around the populations and after the labels: every kernel reads only cells of the
// box, so nothing is read here; the slack keeps each allocation's start and end away from
// the first and last 32-cell row
const size_t kDfPad = 512;
const size_t kLabelPad = 64;

// storage for the kernel arguments of either arithmetic type, aligned like the structures
// they stand for
template <size_t N>
struct alignas(64) ArgBytes {
    unsigned char bytes[N];
    void* data() { return bytes; }
    const void* data() const { return bytes; }
};
constexpr size_t kCaseArgsBytes = std::max(sizeof(CaseArgs<double>), sizeof(CaseArgs<float>));
constexpr size_t kGroupArgsBytes = std::max(sizeof(GroupArgs<double>), sizeof(GroupArgs<float>));

struct Case {
    nnlbm_case_desc d{};
    int64_t N = 0;
    int ct_bytes = 4;        // arithmetic type size (8 for F64 storage)
    double scale = 1.0;      // 16-bit storage scale
    int group = 0;
    // device buffers
    void* df_base = nullptr; // allocation holding df with kDfPad bytes on either side
    void* df = nullptr;      // 27 direction arrays
    size_t q_stride = 0;     // elements between direction arrays
    uint8_t* d_label = nullptr;
    void* d_macro = nullptr;
    void* d_stats = nullptr;
    void* d_ctl = nullptr;
    int64_t ctl_cap = 0;
    double* d_red = nullptr;         // in the context's status block
    int* d_err = nullptr;            // in the context's status block
    uint32_t* d_hw = nullptr;        // halfway bounce-back: wall-neighbour bits per cell
    std::vector<uint32_t> hw;        // its host copy (empty with full-way bounce-back)
    // host state
    std::vector<uint8_t> label;      // plain solver labels
    std::vector<uint8_t> dlabel;     // labels with the work flags of the device copy
    std::vector<Chunk> chunks;       // work list (case index 0)
    bool stage_maps = false;         // the staged form's tensor maps are in args
    std::vector<ChunkNodes> chunk_nodes; // the open-plane nodes each chunk serves
    std::vector<int32_t> self_cell;  // cells handled by their own thread, in cell order
    std::vector<int32_t> gather_self;// self indices of the gathered nodes
    std::vector<double> self_prof;   // [n_self][3] prescribed velocity of INFLOW_EQ nodes
    int64_t n_fluid = 0, n_bc = 0, left_area = 0, right_area = 0, n_inflow_eq = 0;
    double ivc_flux = 0, svc_flux = 0, rho_left = 1, rho_right = 1, rho_eq = 1;
    std::vector<double> sched;       // rows of {ivc_flux, svc_flux, profile_scale}
    mutable std::vector<char> ctl_dev; // copy of the leading control rows on the device (empty: unknown)
    std::vector<char> ctl_buf;       // the rows of the current call, built on the host
    // pinned staging of the rows for their copies to the device: a ring of kCtlSlots buffers,
    // each reused once the copy recorded by its event has run, so that asynchronous calls can
    // run several steps ahead of the device
    static constexpr int kCtlSlots = 4;
    char* h_ctl[kCtlSlots] = {};
    size_t h_ctl_bytes[kCtlSlots] = {};
    cudaEvent_t ctl_done[kCtlSlots] = {};
    int ctl_slot = 0;
    int64_t parity = 0;              // steps done since the layout was last reset, mod 2
    int64_t iterations = 0;
    int64_t n_stats = 0;
    bool has_map = false, has_state = false;
    double init[4] = {1.0, 0.0, 0.0, 0.0}; // rho, u of the last initial equilibrium
    ArgBytes<kCaseArgsBytes> args{}; // CaseArgs<CT>
};

struct Group {
    int dtype = 1, collision = 0;
    std::vector<int> cases;          // context case indices
    bool dirty = true;
    void* d_cases = nullptr;         // CaseArgs<CT>[n]
    Chunk* d_chunks = nullptr;
    ChunkNodes* d_chunk_nodes = nullptr;
    int n_chunks = 0;
    int4* d_gather = nullptr;
    int2* d_nodes = nullptr;
    int n_gather = 0;
    void* d_bc_prof = nullptr;
    void* d_bc_buf = nullptr;
    int64_t n_self = 0;
    int* d_ints = nullptr;           // the two step cursors (one per A-A parity), in the status block
    bool any_refd = false;
    int block = 256;
    bool paired = false;             // two cells a thread (set where the collision can pair)
    bool staged = false;             // the paired form with staged loads (k_step_staged)
    int staged_max_blocks = 0;       // resident blocks of k_step_staged on the device (0: no staged form)
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    uint64_t graph_gen = ~0ull, gen = 0;
    ArgBytes<kGroupArgsBytes> args{}; // GroupArgs<CT>
};

} // namespace

// every word the host reads back after a step, in one device block (and one pinned host
// mirror) so that a synchronous step costs one small copy: per launch group 4 ints (the
// two step cursors), per case kRedStripes x 8 doubles (the striped reductions) and 2 ints
// (the watchdog flag).  The cursors and the sums lead, so that one memset clears what a
// step call restarts.
constexpr size_t kRedBytes = (size_t)kRedStripes * 8 * sizeof(double);
struct StatusLayout {
    size_t cur, red, err, bytes;
    explicit StatusLayout(size_t n_slots)
        : cur(0), red(16 * n_slots), err(red + kRedBytes * n_slots), bytes(err + 8 * n_slots) {}
};

struct nnlbm_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<Case> cases;
    std::vector<Group> groups;
    std::string err;
    char* d_status = nullptr;        // StatusLayout(cases.size()) on the device
    char* h_status = nullptr;        // its pinned host mirror
    bool status_fresh = false;       // the mirror holds the block as the last step left it
    int sm_count = 0;
    // copies of the status block enqueued by NNLBM_STEP_READBACK, oldest first: pinned slots,
    // the event after each copy, and what its check needs (the steps of the call, each group's
    // A-A parity after them)
    struct Readback {
        char* h = nullptr;
        unsigned long long* d = nullptr;  // the slot's device address (mapped pinned memory)
        cudaEvent_t done = nullptr;
        int64_t n = 0;
        std::vector<int> parity;
    };
    Readback rb[NNLBM_READBACK_SLOTS];
    int rb_head = 0, rb_count = 0;
    bool rb_copy = false;  // NNLBM_READBACK_COPY=1: a device-to-host copy instead of k_publish_status
    bool prologue_copy = false;  // NNLBM_PROLOGUE_COPY=1: copy and memsets instead of k_step_prologue
    // a status range that the next k_step_prologue clears (left by nnlbm_step for its first launch)
    unsigned long long* zero_next = nullptr;
    int zero_next_words = 0;
    // the staged step's bounded waits (GroupArgs::stage_wait_ns, stage_pad)
    long long stage_wait_ns = 2000000000LL;
    int stage_pad = 0;
};

namespace {

int set_err(nnlbm_ctx* ctx, int code, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (ctx) ctx->err = buf;
    return code;
}

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return set_err(ctx, e_ == cudaErrorMemoryAllocation ? NNLBM_ERR_OOM : NNLBM_ERR_CUDA, \
                           "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

// cuTensorMapEncodeTiled through the runtime's driver entry point (the library links only
// the CUDA runtime); null where the driver does not offer it
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*,
                                 const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encode_tiled()
{
    static EncodeTiled fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (EncodeTiled) nullptr;
        }
        return (EncodeTiled)p;
    }();
    return fn;
}

// the staged form's two tensor maps of a single-precision-arithmetic case (CaseArgs::tm_even,
// tm_odd); false if they cannot be made (the case then never steps staged)
template <int DT>
bool encode_stage_maps(const Case& c, CUtensorMap* even, CUtensorMap* odd)
{
    using G = StageGeom<DT>;
    const EncodeTiled enc = encode_tiled();
    if (!enc) return false;
    const CUtensorMapDataType type = DT == 1 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_UINT16;
    const cuuint64_t dims[3] = {(cuuint64_t)c.q_stride, 9, 3};
    const cuuint64_t strides[2] = {(cuuint64_t)c.q_stride * G::sz, (cuuint64_t)9 * c.q_stride * G::sz};
    const cuuint32_t box_even[3] = {(cuuint32_t)G::win, 9, 3}, box_odd[3] = {(cuuint32_t)G::win, 1, 3}, one[3] = {1, 1, 1};
    return enc(even, type, 3, c.df, dims, strides, box_even, one, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS &&
           enc(odd, type, 3, c.df, dims, strides, box_odd, one, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <class CT>
void fill_case_args(Case& c, CaseArgs<CT>& a)
{
    memset(&a, 0, sizeof a);
    a.df = c.df;
    a.qstride = (int64_t)c.q_stride;
    a.label = c.d_label;
    a.nx = c.d.nx; a.ny = c.d.ny; a.nz = c.d.nz;
    a.N = c.N;
    a.nu = (CT)c.d.nu; a.nu0 = (CT)c.d.cy_nu0; a.lam = (CT)c.d.cy_lambda; a.a = (CT)c.d.cy_a; a.n = (CT)c.d.cy_n;
    a.fx = (CT)c.d.fx; a.fy = (CT)c.d.fy; a.fz = (CT)c.d.fz;
    a.scale = (CT)c.scale; a.inv_scale = (CT)(1.0 / c.scale);
    a.cy_mode = c.d.cy_mode; a.eq = c.d.equilibrium;
    a.macro = (CT*)c.d_macro;
    a.stats = c.d_stats; a.stats_f64 = c.d.stats_f64;
    a.ctl = (const StepCtl<CT>*)c.d_ctl;
    a.red = c.d_red;
    a.err = c.d_err;
    a.hw = c.d_hw;
    // slot bases (integer arithmetic: a shifted base may point before the array; the cell
    // index of every plain access brings it back inside)
    const uintptr_t base = (uintptr_t)c.df;
    const int64_t S = kStorageBytes[c.d.dtype], qs = (int64_t)c.q_stride, sy = c.d.nx, sz = (int64_t)c.d.nx * c.d.ny;
    for (int q = 0; q < 27; ++q) {
        const int64_t sh = cxq(q) + cyq(q) * sy + czq(q) * sz;
        a.slot_even[q] = (const void*)(base + (uintptr_t)(q * qs * S));
        a.slot_odd_st[q] = (const void*)(base + (uintptr_t)((q * qs + sh) * S));
    }
    c.stage_maps = false;
    if (c.df && c.d.dtype == NNLBM_F32) c.stage_maps = encode_stage_maps<1>(c, &a.tm_even, &a.tm_odd);
    if (c.df && c.d.dtype == NNLBM_F16) c.stage_maps = encode_stage_maps<2>(c, &a.tm_even, &a.tm_odd);
    if (c.df && c.d.dtype == NNLBM_BF16) c.stage_maps = encode_stage_maps<3>(c, &a.tm_even, &a.tm_odd);
}

void rebuild_case_args(nnlbm_ctx* ctx, Case& c)
{
    if (c.ct_bytes == 8) {
        fill_case_args<double>(c, *(CaseArgs<double>*)c.args.data());
    } else {
        fill_case_args<float>(c, *(CaseArgs<float>*)c.args.data());
    }
    ctx->groups[c.group].dirty = true;
}

int check_case(nnlbm_ctx* ctx, int ic)
{
    if (!ctx) return NNLBM_ERR_ARG;
    if (ic < 0 || ic >= (int)ctx->cases.size()) return set_err(ctx, NNLBM_ERR_ARG, "case index %d out of range", ic);
    return NNLBM_OK;
}

int ensure_macro(nnlbm_ctx* ctx, Case& c)
{
    if (c.d_macro) return NNLBM_OK;
    CK(cudaMalloc(&c.d_macro, (size_t)M_N * c.N * c.ct_bytes));
    rebuild_case_args(ctx, c);
    aux_launchers(c.d.dtype).init_macro(c.args.data(), c.init[0], c.init[1], c.init[2], c.init[3], ctx->stream);
    CK(cudaGetLastError());
    return NNLBM_OK;
}

int ensure_stats(nnlbm_ctx* ctx, Case& c)
{
    if (c.d_stats) return NNLBM_OK;
    const size_t bytes = (size_t)6 * c.N * (c.d.stats_f64 ? 8 : 4);
    CK(cudaMalloc(&c.d_stats, bytes));
    CK(cudaMemsetAsync(c.d_stats, 0, bytes, ctx->stream));
    c.n_stats = 0;
    rebuild_case_args(ctx, c);
    return NNLBM_OK;
}

int ensure_ctl(nnlbm_ctx* ctx, Case& c, int64_t n)
{
    if (c.ctl_cap >= n && c.d_ctl) return NNLBM_OK;
    c.ctl_dev.clear();
    int64_t cap = std::max<int64_t>(n, 1024);
    if (c.d_ctl) cudaFree(c.d_ctl);
    c.d_ctl = nullptr;
    const size_t row = c.ct_bytes == 8 ? sizeof(StepCtl<double>) : sizeof(StepCtl<float>);
    CK(cudaMalloc(&c.d_ctl, cap * row));
    c.ctl_cap = cap;
    rebuild_case_args(ctx, c);
    return NNLBM_OK;
}

template <class CT>
void fill_ctl(const Case& c, std::vector<char>& buf, int64_t n, int flags)
{
    buf.resize(n * sizeof(StepCtl<CT>));
    StepCtl<CT>* r = (StepCtl<CT>*)buf.data();
    const int64_t ns = (int64_t)c.sched.size() / 3;
    for (int64_t k = 0; k < n; ++k) {
        double ivc = c.ivc_flux, svc = c.svc_flux, ps = 1.0;
        if (ns > 0) {
            const int64_t t = std::min(k, ns - 1);
            ivc = c.sched[3 * t]; svc = c.sched[3 * t + 1]; ps = c.sched[3 * t + 2];
        }
        int f = flags & NNLBM_STEP_STATS;
        if (k == n - 1) f |= flags & (NNLBM_STEP_MACRO | NNLBM_STEP_REDUCE);
        r[k].flags = f;
        r[k].pad = 0;
        // LBM_Data_Tcpc::inflowCondition{Left,Right} (sim_tcpc.cu:295-309) with
        // inflow_right = -svc_flux (sim_tcpc.cu:660), divided in the arithmetic type
        r[k].u_left = c.left_area > 0 ? (CT)ivc / (CT)c.left_area : CT(0);
        r[k].u_right = c.right_area > 0 ? (CT)(-svc) / (CT)c.right_area : CT(0);
        r[k].rho_left = (CT)c.rho_left; r[k].rho_right = (CT)c.rho_right; r[k].rho_eq = (CT)c.rho_eq;
        r[k].prof_scale = (CT)ps;
    }
}

template <class CT>
int upload_group(nnlbm_ctx* ctx, Group& g)
{
    // per-case argument array and the concatenated work lists of the group
    std::vector<CaseArgs<CT>> ca;
    std::vector<Chunk> chunks;
    std::vector<ChunkNodes> chunk_nodes;
    std::vector<int4> gather;
    std::vector<int2> nodes;
    std::vector<CT> prof;
    int64_t self_off = 0;
    g.any_refd = false;
    for (size_t j = 0; j < g.cases.size(); ++j) {
        const Case& c = ctx->cases[g.cases[j]];
        ca.push_back(*(const CaseArgs<CT>*)c.args.data());
        g.any_refd |= c.d.cy_mode == NNLBM_CY_REF_FD;
        for (Chunk ch : c.chunks) {
            ch.cflags = (int)j | (ch.cflags & ~CH_CASE_MASK);
            chunks.push_back(ch);
        }
        chunk_nodes.insert(chunk_nodes.end(), c.chunk_nodes.begin(), c.chunk_nodes.end());
        // a paired step kernel takes chunks two by two: an odd count gets an empty chunk
        // (no colliding lane), so that no pair mixes two cases and the list length is even
        if (pairs_chunks(g.dtype, g.collision) && (c.chunks.size() & 1)) {
            Chunk none = chunks.back();
            none.fluid = 0;
            none.periodic = 0;
            none.cflags &= ~CH_SRC;
            chunks.push_back(none);
            chunk_nodes.push_back(ChunkNodes{});
        }
        for (int32_t k : c.gather_self)
            gather.push_back(make_int4(c.self_cell[k], (int)j, (int)(self_off + k), (int)c.label[c.self_cell[k]]));
        for (int32_t cell : c.self_cell) nodes.push_back(make_int2(cell, (int)j));
        for (double v : c.self_prof) prof.push_back((CT)v);
        self_off += (int64_t)c.self_cell.size();
    }
    if (g.d_cases) cudaFree(g.d_cases);
    if (g.d_chunks) cudaFree(g.d_chunks);
    if (g.d_chunk_nodes) cudaFree(g.d_chunk_nodes);
    if (g.d_gather) cudaFree(g.d_gather);
    if (g.d_nodes) cudaFree(g.d_nodes);
    g.d_nodes = nullptr;
    if (g.d_bc_prof) cudaFree(g.d_bc_prof);
    if (g.d_bc_buf) cudaFree(g.d_bc_buf);
    g.d_cases = nullptr; g.d_chunks = nullptr; g.d_chunk_nodes = nullptr; g.d_gather = nullptr; g.d_bc_prof = nullptr; g.d_bc_buf = nullptr;
    CK(cudaMalloc(&g.d_cases, std::max<size_t>(ca.size(), 1) * sizeof(CaseArgs<CT>)));
    CK(cudaMemcpy(g.d_cases, ca.data(), ca.size() * sizeof(CaseArgs<CT>), cudaMemcpyHostToDevice));
    CK(cudaMalloc((void**)&g.d_chunks, std::max<size_t>(chunks.size(), 1) * sizeof(Chunk)));
    if (!chunks.empty()) CK(cudaMemcpy(g.d_chunks, chunks.data(), chunks.size() * sizeof(Chunk), cudaMemcpyHostToDevice));
    CK(cudaMalloc((void**)&g.d_chunk_nodes, std::max<size_t>(chunk_nodes.size(), 1) * sizeof(ChunkNodes)));
    if (!chunk_nodes.empty())
        CK(cudaMemcpy(g.d_chunk_nodes, chunk_nodes.data(), chunk_nodes.size() * sizeof(ChunkNodes), cudaMemcpyHostToDevice));
    CK(cudaMalloc((void**)&g.d_nodes, std::max<size_t>(nodes.size(), 1) * sizeof(int2)));
    if (!nodes.empty()) CK(cudaMemcpy(g.d_nodes, nodes.data(), nodes.size() * sizeof(int2), cudaMemcpyHostToDevice));
    CK(cudaMalloc((void**)&g.d_gather, std::max<size_t>(gather.size(), 1) * sizeof(int4)));
    if (!gather.empty()) CK(cudaMemcpy(g.d_gather, gather.data(), gather.size() * sizeof(int4), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&g.d_bc_prof, std::max<size_t>(prof.size(), 1) * sizeof(CT)));
    if (!prof.empty()) CK(cudaMemcpy(g.d_bc_prof, prof.data(), prof.size() * sizeof(CT), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&g.d_bc_buf, std::max<int64_t>(self_off, 1) * 4 * sizeof(CT)));
    CK(cudaMemset(g.d_bc_buf, 0, std::max<int64_t>(self_off, 1) * 4 * sizeof(CT)));
    g.n_chunks = (int)chunks.size();
    g.n_gather = (int)gather.size();
    // room in L2 for the work lists the step launches mark persisting (the limit is this
    // process's; it is raised, never lowered, and capped by the device)
    {
        size_t want = 0;
        for (const Group& h : ctx->groups) {
            const size_t b = (size_t)(&h == &g ? chunks.size() : h.n_chunks) * sizeof(Chunk);
            if (b <= kPersistChunkBytes) want += b;
        }
        int max_persist = 0;
        size_t cur = 0;
        if (want > 0 && cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, ctx->device) == cudaSuccess &&
            cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize) == cudaSuccess && cur < want && max_persist > 0)
            cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, std::min(want, (size_t)max_persist));
        cudaGetLastError();
    }
    g.n_self = self_off;
    GroupArgs<CT>& ga = *(GroupArgs<CT>*)g.args.data();
    memset(&ga, 0, sizeof ga);
    for (size_t j = 0; j < ca.size() && j < (size_t)kParamCases; ++j) ga.cp[j] = ca[j];
    ga.n_cases = (int)ca.size();
    ga.cases = (const CaseArgs<CT>*)g.d_cases;
    ga.chunks = g.d_chunks;
    ga.chunk_nodes = g.d_chunk_nodes;
    ga.n_chunks = g.n_chunks;
    ga.gather = g.d_gather;
    ga.n_gather = g.n_gather;
    ga.nodes = g.d_nodes;
    ga.n_nodes = (int)g.n_self;
    ga.bc_prof = (const CT*)g.d_bc_prof;
    ga.bc_buf = (CT*)g.d_bc_buf;
    ga.cursor = g.d_ints;
    ga.stage_wait_ns = ctx->stage_wait_ns;
    ga.stage_pad = ctx->stage_pad;
    g.dirty = false;
    g.gen++;
    return NNLBM_OK;
}

int prepare_group(nnlbm_ctx* ctx, Group& g)
{
    if (!g.dirty) return NNLBM_OK;
    return g.dtype == NNLBM_F64 ? upload_group<double>(ctx, g) : upload_group<float>(ctx, g);
}

// warps of one step launch: one per chunk (per two chunks where the step pairs them),
// then one per 32 boundary nodes
int step_warps(const Group& g)
{
    const int cw = g.paired ? g.n_chunks / 2 : g.n_chunks;
    return std::max(cw + (int)((g.n_self + 31) / 32), 1);
}

// whether a group can step in the staged form: its collision pairs, the kernel fits on the
// device, and every case has its tensor maps
bool can_stage(const nnlbm_ctx* ctx, const Group& g)
{
    if (!pairs_chunks(g.dtype, g.collision) || g.staged_max_blocks <= 0) return false;
    for (int ic : g.cases)
        if (!ctx->cases[ic].stage_maps) return false;
    return true;
}

// the step kernel's launch: the staged form runs persistent warps, as many blocks as stay
// resident (or fewer, one warp per unit of work at most); the others one warp per unit
struct StepShape {
    dim3 grid, block;
    int form;
};
StepShape step_shape(const Group& g)
{
    if (g.staged) {
        const int per_block = kStagedThreads / kChunk;
        const int blocks = std::max(1, std::min((step_warps(g) + per_block - 1) / per_block, g.staged_max_blocks));
        return {dim3(blocks), dim3(kStagedThreads), FORM_STAGED};
    }
    const int per_block = g.block / kChunk;
    return {dim3((step_warps(g) + per_block - 1) / per_block), dim3(g.block), g.paired ? FORM_PAIRED : FORM_ONE};
}

// enqueue one step of a group (no host synchronisation); `odd` is the A-A parity
int enqueue_step(nnlbm_ctx* ctx, Group& g, bool odd)
{
    const AuxLaunchers& A = aux_launchers(g.dtype);
    const int per_block = g.block / kChunk;
    const dim3 cblk(g.block);
    const StepShape sh = step_shape(g);
    const dim3 rgrid((std::max(g.n_chunks, 1) + per_block - 1) / per_block); // one warp per chunk
    if (g.any_refd) {
        A.refd_velocity(odd, rgrid, cblk, ctx->stream, g.args.data());
        A.refd_stress(odd, rgrid, cblk, ctx->stream, g.args.data());
    }
    if (g.n_gather > 0) A.gather(odd, dim3((g.n_gather + 63) / 64), dim3(64), ctx->stream, g.args.data());
    step_launcher(g.dtype, g.collision)(odd, g.n_gather > 0, sh.form, sh.grid, sh.block, ctx->stream, g.args.data());
    CK(cudaGetLastError());
    return NNLBM_OK;
}

int ensure_graphs(nnlbm_ctx* ctx, Group& g)
{
    if (g.graph[0] && g.graph[1] && g.graph_gen == g.gen) return NNLBM_OK;
    for (int p = 0; p < 2; ++p) {
        if (g.graph[p]) { cudaGraphExecDestroy(g.graph[p]); g.graph[p] = nullptr; }
        cudaGraph_t gr = nullptr;
        CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_step(ctx, g, p == 1);
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &gr);
        if (rc != NNLBM_OK) { if (gr) cudaGraphDestroy(gr); return rc; }
        if (e != cudaSuccess) return set_err(ctx, NNLBM_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
        e = cudaGraphInstantiate(&g.graph[p], gr, 0);
        cudaGraphDestroy(gr);
        if (e != cudaSuccess) return set_err(ctx, NNLBM_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
    }
    g.graph_gen = g.gen;
    return NNLBM_OK;
}

// a call's new control rows, carried in the launch's parameters, plus the zeroing of a status
// range (the call's step cursors and sums, or one case's sums) and of the group's step cursors:
// one kernel before the step, where a host-to-device copy and memsets were separate operations
constexpr int kPutRowWords = 64;  // 512 B of control rows: 16 FP32 steps or 9 FP64 steps
struct CtlRows {
    unsigned long long w[kPutRowWords];
};
__global__ void __launch_bounds__(256) k_step_prologue(const __grid_constant__ CtlRows rows, int words,
                                                       unsigned long long* __restrict__ ctl,
                                                       unsigned long long* __restrict__ zero, int zero_words,
                                                       int* __restrict__ cursors)
{
    const int t = threadIdx.x;
    if (t < words) ctl[t] = rows.w[t];
    if (zero)
        for (int i = t; i < zero_words; i += blockDim.x) zero[i] = 0ull;
    if (cursors && t < 2) cursors[t] = 0;
}

// host side of one nnlbm_step call for every case of a group, up to the launches
// `reset`: clear the group's step cursors (and its cases' sums for NNLBM_STEP_REDUCE); a
// caller that cleared the whole status block already passes false
int prepare_steps(nnlbm_ctx* ctx, Group& g, int64_t n, int flags, bool reset = true)
{
    int rc;
    int64_t parity = -1;
    ctx->status_fresh = false;
    bool ints_zeroed = false;
    for (int ic : g.cases) {
        Case& c = ctx->cases[ic];
        if (!c.has_map || !c.has_state) return set_err(ctx, NNLBM_ERR_ARG, "case %d has no map or initial state", ic);
        if (parity >= 0 && c.parity != parity)
            return set_err(ctx, NNLBM_ERR_ARG, "cases of one launch group are at different step parities "
                           "(re-initialise or re-import all of them)");
        parity = c.parity;
        if ((flags & NNLBM_STEP_MACRO) || c.d.cy_mode == NNLBM_CY_REF_FD)
            if ((rc = ensure_macro(ctx, c)) != NNLBM_OK) return rc;
        if (flags & NNLBM_STEP_STATS)
            if ((rc = ensure_stats(ctx, c)) != NNLBM_OK) return rc;
        if ((rc = ensure_ctl(ctx, c, n)) != NNLBM_OK) return rc;
        std::vector<char>& buf = c.ctl_buf;
        if (c.ct_bytes == 8) fill_ctl<double>(c, buf, n, flags);
        else fill_ctl<float>(c, buf, n, flags);
        // rows already on the device (a constant inflow stepped call after call) are not sent again;
        // a few new ones travel in the parameters of k_step_prologue, more go through a pinned
        // staging buffer, reused once its last copy has completed
        const bool send = buf.size() > c.ctl_dev.size() || memcmp(buf.data(), c.ctl_dev.data(), buf.size()) != 0;
        const bool zero_red = reset && (flags & NNLBM_STEP_REDUCE);
        const bool small = buf.size() % 8 == 0 && buf.size() <= sizeof(CtlRows);
        // new rows that fit go in the parameters of k_step_prologue, which also clears the status
        // range nnlbm_step left for the first launch (else this case's sums) and the group's
        // cursors; without new rows the clearing stays with memsets (cheaper than a launch)
        const bool put = !ctx->prologue_copy && send && small;
        if (put) {
            unsigned long long* zero = ctx->zero_next ? ctx->zero_next : zero_red ? (unsigned long long*)c.d_red : nullptr;
            const int zero_words = ctx->zero_next ? ctx->zero_next_words : (int)(kRedBytes / 8);
            if (ctx->zero_next && zero_red) CK(cudaMemsetAsync(c.d_red, 0, kRedBytes, ctx->stream));
            CtlRows rows;
            memcpy(rows.w, buf.data(), buf.size());
            int* cursors = (reset && !ints_zeroed) ? g.d_ints : nullptr;
            k_step_prologue<<<1, 256, 0, ctx->stream>>>(rows, (int)(buf.size() / 8), (unsigned long long*)c.d_ctl, zero,
                                                         zero_words, cursors);
            CK(cudaGetLastError());
            ctx->zero_next = nullptr;
            ctx->zero_next_words = 0;
            ints_zeroed = ints_zeroed || cursors;
            c.ctl_dev = buf;
        } else {
            if (ctx->zero_next) {
                CK(cudaMemsetAsync(ctx->zero_next, 0, (size_t)ctx->zero_next_words * 8, ctx->stream));
                ctx->zero_next = nullptr;
                ctx->zero_next_words = 0;
            }
            if (zero_red) CK(cudaMemsetAsync(c.d_red, 0, kRedBytes, ctx->stream));
        }
        if (send && !put) {
            const int k = c.ctl_slot;
            c.ctl_slot = (k + 1) % Case::kCtlSlots;
            if (!c.ctl_done[k]) CK(cudaEventCreateWithFlags(&c.ctl_done[k], cudaEventDisableTiming));
            else CK(cudaEventSynchronize(c.ctl_done[k]));
            if (c.h_ctl_bytes[k] < buf.size()) {
                if (c.h_ctl[k]) cudaFreeHost(c.h_ctl[k]);
                c.h_ctl[k] = nullptr;
                c.h_ctl_bytes[k] = 0;
                CK(cudaMallocHost((void**)&c.h_ctl[k], std::max<size_t>(buf.size(), 4096)));
                c.h_ctl_bytes[k] = std::max<size_t>(buf.size(), 4096);
            }
            memcpy(c.h_ctl[k], buf.data(), buf.size());
            CK(cudaMemcpyAsync(c.d_ctl, c.h_ctl[k], buf.size(), cudaMemcpyHostToDevice, ctx->stream));
            CK(cudaEventRecord(c.ctl_done[k], ctx->stream));
            c.ctl_dev = buf;
        }
    }
    if ((rc = prepare_group(ctx, g)) != NNLBM_OK) return rc;
    if (reset && !ints_zeroed) CK(cudaMemsetAsync(g.d_ints, 0, 2 * sizeof(int), ctx->stream));
    return NNLBM_OK;
}

void finish_steps(nnlbm_ctx* ctx, Group& g, int64_t n, int flags)
{
    for (int ic : g.cases) {
        Case& c = ctx->cases[ic];
        c.parity = (c.parity + n) & 1;
        c.iterations += n;
        if (flags & NNLBM_STEP_STATS) c.n_stats += n;
    }
}

int run_group_steps(nnlbm_ctx* ctx, Group& g, int64_t n, int flags, bool use_graph, bool reset = true)
{
    int rc = prepare_steps(ctx, g, n, flags, reset);
    if (rc) return rc;
    if (use_graph && (rc = ensure_graphs(ctx, g)) != NNLBM_OK) return rc;
    const int64_t parity = ctx->cases[g.cases[0]].parity;
    for (int64_t k = 0; k < n; ++k) {
        const int p = (int)((parity + k) & 1);
        if (use_graph) CK(cudaGraphLaunch(g.graph[p], ctx->stream));
        else if ((rc = enqueue_step(ctx, g, p == 1)) != NNLBM_OK) return rc;
    }
    finish_steps(ctx, g, n, flags);
    return NNLBM_OK;
}

// the status block into its host mirror: one copy, one wait
int read_status(nnlbm_ctx* ctx)
{
    CK(cudaMemcpyAsync(ctx->h_status, ctx->d_status, StatusLayout(ctx->cases.size()).bytes, cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->status_fresh = true;
    return NNLBM_OK;
}

// the watchdog flags of a status block copy (the host mirror by default)
int check_watchdog(nnlbm_ctx* ctx, const char* status = nullptr)
{
    const StatusLayout sl(ctx->cases.size());
    const int* err = (const int*)((status ? status : ctx->h_status) + sl.err);
    for (size_t i = 0; i < ctx->cases.size(); ++i)
        if (err[2 * i] & ERR_STALL)
            return set_err(ctx, NNLBM_ERR_TIMEOUT, "case %zu: a staged step waited %.3f s for its bulk copies and gave up", i,
                           ctx->stage_wait_ns * 1e-9);
    for (size_t i = 0; i < ctx->cases.size(); ++i)
        if (err[2 * i]) return set_err(ctx, NNLBM_ERR_NAN, "case %zu: density left (0.25, 4) or became non-finite", i);
    return NNLBM_OK;
}

// the step cursors of a status block copy after n steps that left group i at parity[i]
int check_cursors(nnlbm_ctx* ctx, const char* status, int64_t n, const std::vector<int>& parity)
{
    const int* cur = (const int*)(status + StatusLayout(ctx->cases.size()).cur);
    for (size_t i = 0; i < ctx->groups.size(); ++i) {
        // the last step stored n into the cursor of the parity the group is at now
        const int k = 4 * (int)i + (parity[i] & 1);
        if (cur[k] != n)
            return set_err(ctx, NNLBM_ERR_CUDA, "launch group %zu: step cursor %d after %lld steps", i, cur[k], (long long)n);
    }
    return NNLBM_OK;
}

std::vector<int> group_parities(const nnlbm_ctx* ctx)
{
    std::vector<int> p;
    for (const Group& g : ctx->groups) p.push_back((int)(ctx->cases[g.cases[0]].parity & 1));
    return p;
}

int wait_and_check(nnlbm_ctx* ctx, int64_t n)
{
    int rc = read_status(ctx);
    if (rc != NNLBM_OK) return rc;
    if ((rc = check_cursors(ctx, ctx->h_status, n, group_parities(ctx))) != NNLBM_OK) return rc;
    return check_watchdog(ctx);
}

bool is_pull_bc(int lab) { return lab == L_IN_L || lab == L_IN_R || lab == L_OUT_F || lab == L_OUT_B || lab == L_OUT_REQ; }

// storage element <-> double on the host
double decode(const Case& c, const void* base, size_t i, int q)
{
    switch (c.d.dtype) {
    case NNLBM_F64: return ((const double*)base)[i];
    case NNLBM_F32: return (double)(weight<float>(q) + ((const float*)base)[i]);
    case NNLBM_F16: return (double)(weight<float>(q) + __half2float(((const __half*)base)[i]) * (float)(1.0 / c.scale));
    default: return (double)(weight<float>(q) + __bfloat162float(((const __nv_bfloat16*)base)[i]) * (float)(1.0 / c.scale));
    }
}

void encode(const Case& c, void* base, size_t i, int q, double v)
{
    switch (c.d.dtype) {
    case NNLBM_F64: ((double*)base)[i] = v; break;
    case NNLBM_F32: ((float*)base)[i] = (float)v - weight<float>(q); break;
    case NNLBM_F16: ((__half*)base)[i] = __float2half_rn(((float)v - weight<float>(q)) * (float)c.scale); break;
    default: ((__nv_bfloat16*)base)[i] = __float2bfloat16_rn(((float)v - weight<float>(q)) * (float)c.scale); break;
    }
}

// location of the canonical population q of cell (x,y,z) in the current A-A layout
size_t canon_index(const Case& c, int x, int y, int z, int q, int* slot)
{
    const int nx = c.d.nx, ny = c.d.ny, nz = c.d.nz;
    if (c.parity & 1) { // after an even step: slot opp(q) at x
        *slot = oppq(q);
        return (size_t)x + (size_t)nx * (y + (size_t)ny * z);
    }
    const size_t self = (size_t)x + (size_t)nx * (y + (size_t)ny * z);
    if (!c.hw.empty() && ((c.hw[self] >> q) & 1u)) { // halfway bounce-back towards a wall: own slot opp(q)
        *slot = oppq(q);
        return self;
    }
    *slot = q; // after an odd step (or the initial state): slot q at x + c_q
    const int xx = (x + cxq(q) + nx) % nx, yy = (y + cyq(q) + ny) % ny, zz = (z + czq(q) + nz) % nz;
    return (size_t)xx + (size_t)nx * (yy + (size_t)ny * zz);
}

// ---------------------------------------------------------------------------------------
// scratch of nnlbm_step_noalloc: one file-scope device array per device (the module's
// global), never allocated or freed by this library.  Layout: [0, 1024) the step cursors,
// four ints per launch group in the order of the status block (two used: one per A-A
// parity), then the gathered open-plane node values (rho, ux, uy, uz per node) of the launch
// group being stepped.
// ---------------------------------------------------------------------------------------
constexpr size_t kNoallocHead = 1024;
constexpr size_t kNoallocGroups = kNoallocHead / (4 * sizeof(int));
constexpr int kNoallocDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[kNoallocDevices] = {};

} // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[NNLBM_NOALLOC_SCRATCH_BYTES];

namespace {

// the status block into a readback slot of mapped pinned host memory: one block of plain
// stores in the stream, where a device-to-host copy waits for the copy engine between two steps.
// The event recorded after it completes once the stores are visible to the host.
__global__ void __launch_bounds__(256) k_publish_status(const unsigned long long* __restrict__ src,
                                                        unsigned long long* __restrict__ dst, int words)
{
    for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
}

// device address of the scratch array on the context's device, looked up once per device
// with that device current (the caller has made it current).  nnlbm_create calls it, so that
// the module holding the array is loaded then (under lazy module loading a first lookup inside
// nnlbm_step_noalloc would load it, and allocate, there).
int noalloc_scratch(nnlbm_ctx* ctx, char** out)
{
    if (ctx->device < 0 || ctx->device >= kNoallocDevices)
        return set_err(ctx, NNLBM_ERR_ARG, "nnlbm_step_noalloc: device %d beyond the %d supported", ctx->device,
                       kNoallocDevices);
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[ctx->device]) {
        void* p = nullptr;
        CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_ptr[ctx->device] = p;
    }
    *out = (char*)g_noalloc_ptr[ctx->device];
    return NNLBM_OK;
}

// the control rows of fill_ctl, staged through a fixed host buffer (no allocation)
template <class CT>
int upload_ctl_rows(nnlbm_ctx* ctx, const Case& c, int64_t n, int flags)
{
    constexpr int kRows = 64;
    StepCtl<CT> r[kRows];
    const int64_t ns = (int64_t)c.sched.size() / 3;
    for (int64_t k0 = 0; k0 < n; k0 += kRows) {
        const int cnt = (int)std::min<int64_t>(kRows, n - k0);
        for (int j = 0; j < cnt; ++j) {
            const int64_t k = k0 + j;
            double ivc = c.ivc_flux, svc = c.svc_flux, ps = 1.0;
            if (ns > 0) {
                const int64_t t = std::min(k, ns - 1);
                ivc = c.sched[3 * t]; svc = c.sched[3 * t + 1]; ps = c.sched[3 * t + 2];
            }
            int f = flags & NNLBM_STEP_STATS;
            if (k == n - 1) f |= flags & (NNLBM_STEP_MACRO | NNLBM_STEP_REDUCE);
            r[j].flags = f;
            r[j].pad = 0;
            r[j].u_left = c.left_area > 0 ? (CT)ivc / (CT)c.left_area : CT(0);
            r[j].u_right = c.right_area > 0 ? (CT)(-svc) / (CT)c.right_area : CT(0);
            r[j].rho_left = (CT)c.rho_left; r[j].rho_right = (CT)c.rho_right; r[j].rho_eq = (CT)c.rho_eq;
            r[j].prof_scale = (CT)ps;
        }
        c.ctl_dev.clear();
    // pageable source: the call returns once the rows have been staged, so r is reusable
        CK(cudaMemcpyAsync((StepCtl<CT>*)c.d_ctl + k0, r, cnt * sizeof(StepCtl<CT>), cudaMemcpyHostToDevice, ctx->stream));
    }
    return NNLBM_OK;
}

// the kernel arguments of launch group gi with the per-call scratch moved into the static
// array
template <class CT>
void noalloc_args(const Group& g, size_t gi, char* scratch, char* out)
{
    GroupArgs<CT>& ga = *(GroupArgs<CT>*)out;
    memcpy(&ga, g.args.data(), sizeof ga);
    ga.cursor = (int*)scratch + 4 * gi;
    ga.bc_buf = (CT*)(scratch + kNoallocHead);
}

} // namespace

// ======================================================================================
// C ABI
// ======================================================================================
extern "C" {

int nnlbm_create(const nnlbm_case_desc* desc, int n_cases, int device, nnlbm_ctx** out)
{
    if (!desc || n_cases < 1 || n_cases > CH_CASE_MASK + 1 || !out) return NNLBM_ERR_ARG;
    nnlbm_ctx* ctx = new nnlbm_ctx();
    *out = ctx; // on failure the context carries the message; the caller destroys it
    ctx->device = device;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return set_err(ctx, NNLBM_ERR_CUDA, "no CUDA device %d (found %d)", device, ndev);
    }
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess)
        return set_err(ctx, NNLBM_ERR_CUDA, "cannot initialise device %d", device);
    ctx->cases.resize(n_cases);
    // a group per case at most
    const StatusLayout sl((size_t)n_cases);
    if (cudaMalloc(&ctx->d_status, sl.bytes) != cudaSuccess || cudaMallocHost(&ctx->h_status, sl.bytes) != cudaSuccess) {
        cudaGetLastError();
        return set_err(ctx, NNLBM_ERR_OOM, "allocation of the %zu-byte status block failed", sl.bytes);
    }
    cudaMemset(ctx->d_status, 0, sl.bytes);
    for (int i = 0; i < n_cases; ++i) {
        Case& c = ctx->cases[i];
        c.d = desc[i];
        const nnlbm_case_desc& d = c.d;
        if (d.nx < 3 || d.ny < 3 || d.nz < 3 || d.dtype < 0 || d.dtype > 3 || d.collision < 0 || d.collision > 10 ||
            d.equilibrium < 0 || d.equilibrium > 3 || d.cy_mode < 0 || d.cy_mode > 2 || !(d.nu > 0))
            return set_err(ctx, NNLBM_ERR_ARG, "case %d: invalid descriptor (dims >= 3, dtype 0..3, collision 0..10, "
                           "equilibrium 0..3, cy_mode 0..2, nu > 0)", i);
        if (d.cy_mode != NNLBM_CY_NONE && !(d.cy_a > 0 && d.cy_nu0 > 0))
            return set_err(ctx, NNLBM_ERR_ARG, "case %d: Carreau-Yasuda needs a > 0 and nu0 > 0", i);
        if (d.bounce_back != NNLBM_BB_FULLWAY && d.bounce_back != NNLBM_BB_HALFWAY)
            return set_err(ctx, NNLBM_ERR_ARG, "case %d: bounce_back must be NNLBM_BB_FULLWAY or NNLBM_BB_HALFWAY", i);
        if (d.ny > 65535 || d.nz > 65535) return set_err(ctx, NNLBM_ERR_ARG, "case %d: ny and nz are limited to 65535", i);
        c.N = (int64_t)d.nx * d.ny * d.nz;
        if (c.N >= (int64_t)1 << 31) return set_err(ctx, NNLBM_ERR_ARG, "case %d: %lld cells exceed 2^31", i, (long long)c.N);
        c.ct_bytes = d.dtype == NNLBM_F64 ? 8 : 4;
        c.scale = (d.dtype == NNLBM_F16 || d.dtype == NNLBM_BF16) && d.storage_scale > 0 ? d.storage_scale
                  : (d.dtype == NNLBM_F16 ? 1024.0 : 1.0);
        const size_t eb = kStorageBytes[d.dtype];
        c.q_stride = ((size_t)c.N + 127) / 128 * 128;
        if (cudaMalloc(&c.df_base, 27 * c.q_stride * eb + 2 * kDfPad) != cudaSuccess ||
            cudaMalloc(&c.d_label, ((size_t)c.N + kLabelPad + 15) / 16 * 16) != cudaSuccess) {
            cudaGetLastError();
            return set_err(ctx, NNLBM_ERR_OOM, "case %d: device allocation of %.2f GB failed", i, 27.0 * c.q_stride * eb / 1e9);
        }
        c.df = (char*)c.df_base + kDfPad;
        c.d_err = (int*)(ctx->d_status + sl.err) + 2 * i;
        c.d_red = (double*)(ctx->d_status + sl.red + kRedBytes * i);
        c.label.assign((size_t)c.N, (uint8_t)L_WALL);
        c.dlabel = c.label;
        // launch groups: cases of one storage type and collision run in the same kernels
        int gi = -1;
        for (size_t k = 0; k < ctx->groups.size(); ++k)
            if (ctx->groups[k].dtype == d.dtype && ctx->groups[k].collision == d.collision) gi = (int)k;
        if (gi < 0) {
            ctx->groups.emplace_back();
            gi = (int)ctx->groups.size() - 1;
            ctx->groups[gi].dtype = d.dtype;
            ctx->groups[gi].collision = d.collision;
            ctx->groups[gi].paired = pairs_chunks(d.dtype, d.collision);
            ctx->groups[gi].d_ints = (int*)(ctx->d_status + sl.cur) + 4 * gi;
        }
        c.group = gi;
        ctx->groups[gi].cases.push_back(i);
        int rc = ensure_ctl(ctx, c, 1024);
        if (rc != NNLBM_OK) return rc;
        rebuild_case_args(ctx, c);
    }
    // load the kernels of every launch group and the module of nnlbm_step_noalloc's scratch
    // now, so that no later call loads code (and allocates) on first use
    CK(cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device));
    for (Group& g : ctx->groups) {
        const cudaError_t e = load_group_kernels(g.dtype, g.collision);
        if (e != cudaSuccess)
            return set_err(ctx, NNLBM_ERR_CUDA, "loading the kernels of storage %d, collision %d failed: %s", g.dtype,
                           g.collision, cudaGetErrorString(e));
        g.staged_max_blocks = staged_occupancy(g.dtype, g.collision)() * ctx->sm_count;
    }
    // a test's stall of the staged step: every wait expects 16 bytes that never arrive and
    // gives up after a millisecond (NNLBM_ERR_TIMEOUT); all its copies still complete
    if (const char* t = getenv("NNLBM_READBACK_COPY"); t && atoi(t) == 1) ctx->rb_copy = true;
    if (const char* t = getenv("NNLBM_PROLOGUE_COPY"); t && atoi(t) == 1) ctx->prologue_copy = true;
    if (const char* t = getenv("NNLBM_TEST_STAGE_STALL"); t && atoi(t) == 1) {
        ctx->stage_wait_ns = 1000000LL;
        ctx->stage_pad = 16;
    }
    char* scratch = nullptr;
    return noalloc_scratch(ctx, &scratch);
}

int nnlbm_set_map(nnlbm_ctx* ctx, int ic, const uint8_t* map)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    if (!map) return set_err(ctx, NNLBM_ERR_ARG, "null map");
    Case& c = ctx->cases[ic];
    const int nx = c.d.nx, ny = c.d.ny, nz = c.d.nz;
    auto id = [&](int x, int y, int z) { return (size_t)x + (size_t)nx * (y + (size_t)ny * z); };
    int64_t nfl = 0, la = 0, ra = 0, neq = 0, nbc = 0;
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const int lab = map[id(x, y, z)];
                if (lab > L_OUT_REQ) return set_err(ctx, NNLBM_ERR_ARG, "label %d at (%d,%d,%d) is not a solver label", lab, x, y, z);
                const bool face = x == 0 || y == 0 || z == 0 || x == nx - 1 || y == ny - 1 || z == nz - 1;
                if (lab == L_FLUID && face)
                    return set_err(ctx, NNLBM_ERR_ARG, "FLUID cell on the domain face at (%d,%d,%d): faces must hold walls, "
                                   "open planes or PERIODIC cells", x, y, z);
                // the re-centred stencils of the open planes reach two cells inward
                if ((lab == L_IN_L && x > nx - 3) || ((lab == L_IN_R || lab == L_OUT_REQ) && x < 2) ||
                    (lab == L_OUT_F && y > ny - 3) || (lab == L_OUT_B && y < 2))
                    return set_err(ctx, NNLBM_ERR_ARG, "open-plane label %d at (%d,%d,%d) has no room for its inward stencil",
                                   lab, x, y, z);
                nfl += lab == L_FLUID || lab == L_PERIODIC;
                la += lab == L_IN_L;
                ra += lab == L_IN_R;
                neq += lab == L_IN_EQ;
                nbc += lab >= L_IN_L;
            }
    // Open-plane nodes whose re-centred stencil is the pull of their inward neighbour (a
    // FLUID or PERIODIC cell off every face, so that nothing wraps or is clamped) are finished
    // by that neighbour within the step (serve_nodes in nnlbm_kernels.cuh).  Not with the
    // finite-difference Carreau-Yasuda force, which the neighbour adds to its own velocity.
    std::vector<uint8_t> dl(map, map + c.N);
    std::vector<uint8_t> serves((size_t)c.N, 0);
    const bool can_fuse = c.d.cy_mode != NNLBM_CY_REF_FD;
    auto fused_source = [&](size_t i, int lab) -> int64_t {
        const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((size_t)nx * ny));
        const int sx = x + (lab == L_IN_L) - (lab == L_IN_R || lab == L_OUT_REQ);
        const int sy = y + (lab == L_OUT_F) - (lab == L_OUT_B);
        if (sx < 1 || sx > nx - 2 || sy < 1 || sy > ny - 2 || z < 1 || z > nz - 2) return -1;
        const size_t s = id(sx, sy, z);
        return map[s] == L_FLUID || map[s] == L_PERIODIC ? (int64_t)s : -1;
    };
    // the other boundary nodes (open planes and GEO_INFLOW cells), in cell order: each is
    // written by its own lane of the node warps; the open-plane ones are gathered first
    std::vector<int32_t> self_cell, gather_self;
    for (size_t i = 0; i < (size_t)c.N; ++i) {
        const int lab = map[i];
        if (lab != L_IN_EQ && !is_pull_bc(lab)) continue;
        if (can_fuse && lab != L_IN_EQ) {
            const int64_t s = fused_source(i, lab);
            if (s >= 0) {
                serves[(size_t)s] |= lab == L_IN_L ? kServeXneg : lab == L_IN_R ? kServeXpos
                                   : lab == L_OUT_REQ ? (kServeXpos | kServeXreq) : lab == L_OUT_F ? kServeYneg : kServeYpos;
                continue;
            }
        }
        dl[i] |= LF_SELF;
        if (lab != L_IN_EQ) gather_self.push_back((int32_t)self_cell.size());
        self_cell.push_back((int32_t)i);
    }
    // halfway bounce-back: per cell, bit q where the neighbour x + c_q (wrapped) is a wall
    std::vector<uint32_t> hw;
    if (c.d.bounce_back == NNLBM_BB_HALFWAY) {
        hw.assign((size_t)c.N, 0u);
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) {
                    uint32_t m = 0;
                    for (int q = 0; q < 27; ++q) {
                        const int xx = (x + cxq(q) + nx) % nx, yy = (y + cyq(q) + ny) % ny, zz = (z + czq(q) + nz) % nz;
                        if (q != 13 && map[id(xx, yy, zz)] == L_WALL) m |= 1u << q;
                    }
                    hw[id(x, y, z)] = m;
                }
    }
    // packed work list of 32-cell row chunks of colliding cells: a chunk starts at the first
    // colliding cell not yet covered in its row, rounded down to a 32-byte boundary of the
    // population rows (but not into the previous chunk), so that a short row segment fills
    // one chunk instead of straddling two and each row load touches as few sectors as it can
    std::vector<Chunk> chunks;
    std::vector<ChunkNodes> chunk_nodes;
    auto collides = [&](size_t i) { return map[i] == L_FLUID || map[i] == L_PERIODIC; };
    const int align = 32 / kStorageBytes[c.d.dtype];
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x0 = 0, end = 0; x0 < nx; x0 += kChunk, end = x0) {
                while (x0 < nx && !collides(id(x0, y, z))) ++x0;
                if (x0 >= nx) break;
                x0 = std::max(x0 / align * align, end);
                Chunk ch{};
                ChunkNodes cn{};
                ch.c0 = (int)id(x0, y, z);
                ch.yz = y | (z << 16);
                for (int x = x0; x < std::min(nx, x0 + kChunk); ++x) {
                    const size_t i = id(x, y, z);
                    const unsigned bit = 1u << (x - x0);
                    if (collides(i)) {
                        ch.fluid |= bit;
                        if (map[i] == L_PERIODIC) ch.periodic |= bit;
                        if (serves[i] & kServeXneg) cn.xneg |= bit;
                        if (serves[i] & kServeXpos) cn.xpos |= bit;
                        if (serves[i] & kServeXreq) cn.xreq |= bit;
                        if (serves[i] & kServeYneg) cn.yneg |= bit;
                        if (serves[i] & kServeYpos) cn.ypos |= bit;
                        if (!hw.empty() && hw[i]) ch.cflags |= CH_HW;
                    }
                }
                // flags: the chunk lies on a y or z face; the chunk is plain (no colliding cell
                // on an x face either, so no neighbour index wraps)
                const bool face = y == 0 || y == ny - 1 || z == 0 || z == nz - 1;
                const unsigned xface = (x0 == 0 ? 1u : 0u) | (nx - 1 - x0 < kChunk ? 1u << (nx - 1 - x0) : 0u);
                const bool plain = !face && !(ch.fluid & xface) && !(ch.cflags & CH_HW);
                const bool serving = (cn.xneg | cn.xpos | cn.yneg | cn.ypos) != 0;
                ch.cflags |= CH_FLUID | (face ? CH_FACE : 0) | (plain ? CH_PLAIN : 0) | (serving ? CH_SRC : 0);
                chunks.push_back(ch);
                chunk_nodes.push_back(cn);
            }
    c.label.assign(map, map + c.N);
    c.dlabel = dl;
    c.chunks = chunks;
    c.chunk_nodes = chunk_nodes;
    c.self_cell = self_cell;
    c.gather_self = gather_self;
    c.self_prof.assign(self_cell.size() * 3, 0.0);
    c.n_fluid = nfl; c.left_area = la; c.right_area = ra; c.n_inflow_eq = neq; c.n_bc = nbc;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream)); // no queued step still reads the old labels
    CK(cudaMemcpy(c.d_label, dl.data(), (size_t)c.N, cudaMemcpyHostToDevice));
    if (!hw.empty()) {
        if (!c.d_hw) CK(cudaMalloc(&c.d_hw, (size_t)c.N * sizeof(uint32_t)));
        CK(cudaMemcpy(c.d_hw, hw.data(), (size_t)c.N * sizeof(uint32_t), cudaMemcpyHostToDevice));
    }
    c.hw = hw;
    c.has_map = true;
    rebuild_case_args(ctx, c);
    return NNLBM_OK;
}

// StateTcpc::setupBoundaries (sim_tcpc.cu:494-645) + LBM::projectWall (lbm.hpp:144-155)
int nnlbm_tcpc_labels(int32_t X, int32_t Y, int32_t Z, const int32_t* wall, uint8_t* map_out, uint8_t* wall_flags_out,
                      int64_t* counts)
{
    if (X < 3 || Y < 3 || Z < 3 || !wall || !map_out) return NNLBM_ERR_ARG;
    const size_t N = (size_t)X * Y * Z;
    auto id = [&](int x, int y, int z) { return (size_t)x + (size_t)X * (y + (size_t)Y * z); };
    uint8_t* map = map_out;
    std::vector<uint8_t> wf(N, 0);
    int64_t in[7] = {0};
    for (size_t i = 0; i < N; ++i) {
        const int lab = wall[i];
        if (lab >= 3 && lab <= 6) in[lab]++;
        wf[i] = lab == 1;
        map[i] = L_FLUID;
    }
    // plane labels; later calls win at edges (sim_tcpc.cu:524-529)
    for (int z = 0; z < Z; ++z)
        for (int y = 0; y < Y; ++y) { map[id(0, y, z)] = L_IN_L; map[id(X - 1, y, z)] = L_IN_R; }
    for (int z = 0; z < Z; ++z)
        for (int x = 0; x < X; ++x) { map[id(x, 0, z)] = L_OUT_F; map[id(x, Y - 1, z)] = L_OUT_B; }
    for (int y = 0; y < Y; ++y)
        for (int x = 0; x < X; ++x) { map[id(x, y, 0)] = L_WALL; map[id(x, y, Z - 1)] = L_WALL; }
    // open each inflow / outflow plane where the first open inward plane is open
    // (openBoundaryX / openBoundaryY, sim_tcpc.cu:531-586)
    auto open_plane = [&](int axis, int b, int step) {
        const int n = axis == 0 ? X : Y;
        const int nu = axis == 0 ? Y : X;
        auto cell = [&](int a, int u, int z) { return axis == 0 ? id(a, u, z) : id(u, a, z); };
        int s = b + step;
        while (s > 0 && s < n - 1) {
            int64_t open = 0;
            for (int z = 0; z < Z; ++z)
                for (int u = 0; u < nu; ++u) open += !wf[cell(s, u, z)];
            if (open) break;
            s += step;
        }
        if (s <= 0 || s >= n - 1) return;
        for (int z = 0; z < Z; ++z)
            for (int u = 0; u < nu; ++u)
                if (!wf[cell(s, u, z)])
                    for (int a = b; a != s + step; a += step) wf[cell(a, u, z)] = 0;
    };
    open_plane(0, 0, 1);
    open_plane(0, X - 1, -1);
    open_plane(1, 0, 1);
    open_plane(1, Y - 1, -1);
    int64_t la = 0, ra = 0, of = 0, ob = 0, wc = 0, fc = 0;
    for (size_t i = 0; i < N; ++i) {
        const int lab = map[i];
        const bool w = wf[i] || lab == L_WALL;
        la += lab == L_IN_L && !w; ra += lab == L_IN_R && !w;
        of += lab == L_OUT_F && !w; ob += lab == L_OUT_B && !w;
        wc += w; fc += lab == L_FLUID && !w;
    }
    for (size_t i = 0; i < N; ++i)
        if (wf[i]) map[i] = L_WALL;
    if (wall_flags_out) memcpy(wall_flags_out, wf.data(), N);
    if (counts) {
        const int64_t v[10] = {la, ra, of, ob, wc, fc, in[3], in[4], in[5], in[6]};
        memcpy(counts, v, sizeof v);
    }
    return (la <= 0 || ra <= 0 || of <= 0 || ob <= 0) ? NNLBM_ERR_AREA : NNLBM_OK;
}

int nnlbm_setup_tcpc(nnlbm_ctx* ctx, int ic, const int32_t* wall, int64_t* counts)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    if (!wall) return set_err(ctx, NNLBM_ERR_ARG, "null wall array");
    Case& c = ctx->cases[ic];
    std::vector<uint8_t> map((size_t)c.N);
    int64_t cnt[10];
    const int lrc = nnlbm_tcpc_labels(c.d.nx, c.d.ny, c.d.nz, wall, map.data(), nullptr, cnt);
    if (counts) memcpy(counts, cnt, sizeof cnt);
    if ((rc = nnlbm_set_map(ctx, ic, map.data())) != NNLBM_OK) return rc;
    if (lrc == NNLBM_ERR_AREA)
        return set_err(ctx, NNLBM_ERR_AREA, "zero inlet or outlet area: left=%lld right=%lld outlet5=%lld outlet6=%lld",
                       (long long)cnt[0], (long long)cnt[1], (long long)cnt[2], (long long)cnt[3]);
    return lrc;
}

int nnlbm_init_equilibrium(nnlbm_ctx* ctx, int ic, double rho, double ux, double uy, double uz)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    Case& c = ctx->cases[ic];
    if (!c.has_map) return set_err(ctx, NNLBM_ERR_ARG, "set the map before the initial state");
    CK(cudaSetDevice(ctx->device));
    const AuxLaunchers& A = aux_launchers(c.d.dtype);
    A.fill_eq(c.args.data(), rho, ux, uy, uz, ctx->stream);
    CK(cudaGetLastError());
    if (c.d_macro) A.init_macro(c.args.data(), rho, ux, uy, uz, ctx->stream);
    if (c.d_stats) CK(cudaMemsetAsync(c.d_stats, 0, (size_t)6 * c.N * (c.d.stats_f64 ? 8 : 4), ctx->stream));
    CK(cudaMemsetAsync(c.d_err, 0, sizeof(int), ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->status_fresh = false;
    c.parity = 0; c.iterations = 0; c.n_stats = 0;
    c.init[0] = rho; c.init[1] = ux; c.init[2] = uy; c.init[3] = uz;
    c.has_state = true;
    return NNLBM_OK;
}

int nnlbm_set_inflow(nnlbm_ctx* ctx, int ic, double ivc_flux, double svc_flux, double rho_left, double rho_right, double rho_eq)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    Case& c = ctx->cases[ic];
    c.ivc_flux = ivc_flux; c.svc_flux = svc_flux; c.rho_left = rho_left; c.rho_right = rho_right; c.rho_eq = rho_eq;
    return NNLBM_OK;
}

int nnlbm_set_inflow_profile(nnlbm_ctx* ctx, int ic, const double* u, int64_t n)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    Case& c = ctx->cases[ic];
    if (n != c.n_inflow_eq || (n > 0 && !u))
        return set_err(ctx, NNLBM_ERR_ARG, "profile has %lld rows, the map has %lld INFLOW_EQ cells", (long long)n,
                       (long long)c.n_inflow_eq);
    int64_t k = 0;
    for (size_t s = 0; s < c.self_cell.size(); ++s)
        if (c.label[c.self_cell[s]] == L_IN_EQ) {
            for (int j = 0; j < 3; ++j) c.self_prof[3 * s + j] = u[3 * k + j];
            ++k;
        }
    ctx->groups[c.group].dirty = true;
    return NNLBM_OK;
}

int nnlbm_set_schedule(nnlbm_ctx* ctx, int ic, const double* rows, int64_t n)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    if (n < 0 || (n > 0 && !rows)) return set_err(ctx, NNLBM_ERR_ARG, "bad schedule");
    ctx->cases[ic].sched.assign(rows, rows + 3 * n);
    return NNLBM_OK;
}

int nnlbm_step(nnlbm_ctx* ctx, int64_t n_steps, int flags)
{
    if (!ctx) return NNLBM_ERR_ARG;
    if (n_steps < 0) return set_err(ctx, NNLBM_ERR_ARG, "negative step count");
    if (n_steps == 0) return NNLBM_OK;
    if ((flags & NNLBM_STEP_READBACK) && !(flags & NNLBM_STEP_ASYNC))
        return set_err(ctx, NNLBM_ERR_ARG, "NNLBM_STEP_READBACK needs NNLBM_STEP_ASYNC");
    if ((flags & NNLBM_STEP_READBACK) && ctx->rb_count == NNLBM_READBACK_SLOTS)
        return set_err(ctx, NNLBM_ERR_ARG, "%d status copies pending: call nnlbm_readback first", NNLBM_READBACK_SLOTS);
    CK(cudaSetDevice(ctx->device));
    // every group's step cursors (and, for a reduction, every case's sums) restart from zero: the
    // first group's first k_step_prologue clears them, or one memset
    const StatusLayout sl(ctx->cases.size());
    const size_t zero_bytes = (flags & NNLBM_STEP_REDUCE) ? sl.err : sl.red;
    if (ctx->prologue_copy) {
        CK(cudaMemsetAsync(ctx->d_status, 0, zero_bytes, ctx->stream));
    } else {
        ctx->zero_next = (unsigned long long*)ctx->d_status;
        ctx->zero_next_words = (int)(zero_bytes / 8);
    }
    for (Group& g : ctx->groups) {
        int rc = run_group_steps(ctx, g, n_steps, flags, true, false);
        if (rc != NNLBM_OK) {
            ctx->zero_next = nullptr;
            return rc;
        }
    }
    for (Case& c : ctx->cases) {
        if (c.sched.empty()) continue;
        // consume the rows that were used; the last row stays in force
        const int64_t rows = (int64_t)c.sched.size() / 3;
        if (n_steps < rows) c.sched.erase(c.sched.begin(), c.sched.begin() + 3 * n_steps);
        else c.sched.erase(c.sched.begin(), c.sched.end() - 3);
    }
    if (flags & NNLBM_STEP_READBACK) {
        nnlbm_ctx::Readback& r = ctx->rb[(ctx->rb_head + ctx->rb_count) % NNLBM_READBACK_SLOTS];
        if (!r.h) {
            CK(cudaHostAlloc((void**)&r.h, sl.bytes, cudaHostAllocMapped));
            CK(cudaHostGetDevicePointer((void**)&r.d, r.h, 0));
            CK(cudaEventCreateWithFlags(&r.done, cudaEventDisableTiming));
        }
        if (ctx->rb_copy || sl.bytes % 8 != 0) {
            CK(cudaMemcpyAsync(r.h, ctx->d_status, sl.bytes, cudaMemcpyDeviceToHost, ctx->stream));
        } else {
            k_publish_status<<<1, 256, 0, ctx->stream>>>((const unsigned long long*)ctx->d_status, r.d,
                                                           (int)(sl.bytes / 8));
            CK(cudaGetLastError());
        }
        CK(cudaEventRecord(r.done, ctx->stream));
        r.n = n_steps;
        r.parity = group_parities(ctx);
        ctx->rb_count++;
    }
    if (flags & NNLBM_STEP_ASYNC) return NNLBM_OK;
    return wait_and_check(ctx, n_steps);
}

int nnlbm_readback(nnlbm_ctx* ctx, double* out, int n_cases)
{
    if (!ctx) return NNLBM_ERR_ARG;
    if (!out || n_cases < (int)ctx->cases.size())
        return set_err(ctx, NNLBM_ERR_ARG, "the output holds %d cases, the context has %zu", n_cases, ctx->cases.size());
    if (ctx->rb_count == 0) return set_err(ctx, NNLBM_ERR_ARG, "no status copy pending (NNLBM_STEP_READBACK)");
    CK(cudaSetDevice(ctx->device));
    nnlbm_ctx::Readback& r = ctx->rb[ctx->rb_head];
    ctx->rb_head = (ctx->rb_head + 1) % NNLBM_READBACK_SLOTS;
    ctx->rb_count--;
    CK(cudaEventSynchronize(r.done));
    int rc = check_cursors(ctx, r.h, r.n, r.parity);
    if (rc == NNLBM_OK) rc = check_watchdog(ctx, r.h);
    if (rc != NNLBM_OK) return rc;
    const StatusLayout sl(ctx->cases.size());
    for (size_t ic = 0; ic < ctx->cases.size(); ++ic) {
        const double* red = (const double*)(r.h + sl.red + kRedBytes * ic);
        for (int k = 0; k < 5; ++k) {
            double v = 0.0;
            for (int i = 0; i < kRedStripes; ++i) v += red[8 * i + k];
            out[5 * ic + k] = v;
        }
    }
    return NNLBM_OK;
}

int nnlbm_sync(nnlbm_ctx* ctx)
{
    if (!ctx) return NNLBM_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    const int rc = read_status(ctx);
    return rc != NNLBM_OK ? rc : check_watchdog(ctx);
}

int nnlbm_stat_reset(nnlbm_ctx* ctx, int ic)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    Case& c = ctx->cases[ic];
    CK(cudaSetDevice(ctx->device));
    if (c.d_stats) {
        CK(cudaMemsetAsync(c.d_stats, 0, (size_t)6 * c.N * (c.d.stats_f64 ? 8 : 4), ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    c.n_stats = 0;
    return NNLBM_OK;
}

int nnlbm_get_macro(nnlbm_ctx* ctx, int ic, int field, double* out)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    if (field < 0 || field >= M_N || !out) return set_err(ctx, NNLBM_ERR_ARG, "bad macro field %d", field);
    Case& c = ctx->cases[ic];
    CK(cudaSetDevice(ctx->device));
    if (!c.d_macro) { // the initial state (LBMKernelInit, core.h:833-863)
        if ((rc = ensure_macro(ctx, c)) != NNLBM_OK) return rc;
        CK(cudaStreamSynchronize(ctx->stream));
    }
    // the copies below run on the legacy stream: let the context's queued steps finish first
    CK(cudaStreamSynchronize(ctx->stream));
    if (c.ct_bytes == 8) {
        CK(cudaMemcpy(out, (char*)c.d_macro + (size_t)field * c.N * 8, (size_t)c.N * 8, cudaMemcpyDeviceToHost));
    } else {
        std::vector<float> tmp((size_t)c.N);
        CK(cudaMemcpy(tmp.data(), (char*)c.d_macro + (size_t)field * c.N * 4, (size_t)c.N * 4, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < tmp.size(); ++i) out[i] = tmp[i];
    }
    return NNLBM_OK;
}

int nnlbm_get_stats(nnlbm_ctx* ctx, int ic, double* out, int64_t* n_accumulated)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    Case& c = ctx->cases[ic];
    if (n_accumulated) *n_accumulated = c.n_stats;
    if (!out) return NNLBM_OK;
    CK(cudaSetDevice(ctx->device));
    const size_t n = (size_t)6 * c.N;
    if (!c.d_stats) { memset(out, 0, n * sizeof(double)); return NNLBM_OK; }
    CK(cudaStreamSynchronize(ctx->stream));
    if (c.d.stats_f64) {
        CK(cudaMemcpy(out, c.d_stats, n * 8, cudaMemcpyDeviceToHost));
    } else {
        std::vector<float> tmp(n);
        CK(cudaMemcpy(tmp.data(), c.d_stats, n * 4, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < n; ++i) out[i] = tmp[i];
    }
    return NNLBM_OK;
}

int nnlbm_import_stats(nnlbm_ctx* ctx, int ic, const double* in, int64_t n_accumulated)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    if (!in || n_accumulated < 0) return set_err(ctx, NNLBM_ERR_ARG, "null input or negative step count");
    Case& c = ctx->cases[ic];
    CK(cudaSetDevice(ctx->device));
    if ((rc = ensure_stats(ctx, c)) != NNLBM_OK) return rc;
    const size_t n = (size_t)6 * c.N;
    if (c.d.stats_f64) {
        CK(cudaMemcpyAsync(c.d_stats, in, n * 8, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    } else {
        std::vector<float> tmp(n);
        for (size_t i = 0; i < n; ++i) tmp[i] = (float)in[i];
        CK(cudaMemcpyAsync(c.d_stats, tmp.data(), n * 4, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    c.n_stats = n_accumulated;
    return NNLBM_OK;
}

int nnlbm_import_macro(nnlbm_ctx* ctx, int ic, const double* in)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    if (!in) return set_err(ctx, NNLBM_ERR_ARG, "null input");
    Case& c = ctx->cases[ic];
    CK(cudaSetDevice(ctx->device));
    if ((rc = ensure_macro(ctx, c)) != NNLBM_OK) return rc;
    const size_t n = (size_t)M_N * c.N;
    if (c.ct_bytes == 8) {
        CK(cudaMemcpyAsync(c.d_macro, in, n * 8, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    } else {
        std::vector<float> tmp(n);
        for (size_t i = 0; i < n; ++i) tmp[i] = (float)in[i];
        CK(cudaMemcpyAsync(c.d_macro, tmp.data(), n * 4, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return NNLBM_OK;
}

int nnlbm_export_df(nnlbm_ctx* ctx, int ic, double* out)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    if (!out) return set_err(ctx, NNLBM_ERR_ARG, "null output");
    Case& c = ctx->cases[ic];
    CK(cudaSetDevice(ctx->device));
    const size_t eb = kStorageBytes[c.d.dtype];
    std::vector<char> raw(27 * c.q_stride * eb);
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaMemcpy(raw.data(), c.df, raw.size(), cudaMemcpyDeviceToHost));
    const int nx = c.d.nx, ny = c.d.ny, nz = c.d.nz;
    for (int q = 0; q < 27; ++q)
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) {
                    int slot;
                    const size_t i = canon_index(c, x, y, z, q, &slot);
                    out[(size_t)q * c.N + x + (size_t)nx * (y + (size_t)ny * z)] =
                        decode(c, raw.data() + (size_t)slot * c.q_stride * eb, i, q);
                }
    return NNLBM_OK;
}

int nnlbm_import_df(nnlbm_ctx* ctx, int ic, const double* in)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    if (!in) return set_err(ctx, NNLBM_ERR_ARG, "null input");
    Case& c = ctx->cases[ic];
    if (!c.has_map) return set_err(ctx, NNLBM_ERR_ARG, "set the map before importing a state");
    CK(cudaSetDevice(ctx->device));
    const size_t eb = kStorageBytes[c.d.dtype];
    std::vector<char> raw(27 * c.q_stride * eb, 0);
    c.parity = 0; // write the layout an odd step leaves behind
    const int nx = c.d.nx, ny = c.d.ny, nz = c.d.nz;
    for (int q = 0; q < 27; ++q)
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) {
                    // with halfway bounce-back nothing reads a wall cell's populations, and
                    // the slots the layout would give them hold their neighbours' reflections
                    if (!c.hw.empty() && c.label[x + (size_t)nx * (y + (size_t)ny * z)] == L_WALL) continue;
                    int slot;
                    const size_t i = canon_index(c, x, y, z, q, &slot);
                    encode(c, raw.data() + (size_t)slot * c.q_stride * eb, i, q,
                           in[(size_t)q * c.N + x + (size_t)nx * (y + (size_t)ny * z)]);
                }
    // on the context's stream, after whatever steps it still holds; a new state also clears
    // the case's watchdog flag, which reported on the state it replaces
    CK(cudaMemcpyAsync(c.df, raw.data(), raw.size(), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync(c.d_err, 0, sizeof(int), ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->status_fresh = false;
    c.has_state = true;
    return NNLBM_OK;
}

int nnlbm_reduce(nnlbm_ctx* ctx, int ic, double* out5)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    if (!out5) return set_err(ctx, NNLBM_ERR_ARG, "null output");
    CK(cudaSetDevice(ctx->device));
    // a synchronous step has just read the sums back with its cursors and watchdog flags
    if (!ctx->status_fresh && (rc = read_status(ctx)) != NNLBM_OK) return rc;
    const double* r = (const double*)(ctx->h_status + StatusLayout(ctx->cases.size()).red + kRedBytes * ic);
    for (int k = 0; k < 5; ++k) {
        double v = 0.0;
        for (int i = 0; i < kRedStripes; ++i) v += r[8 * i + k];
        out5[k] = v;
    }
    return NNLBM_OK;
}

int nnlbm_output_fields(nnlbm_ctx* ctx, int ic, const double* params, const uint8_t* wall_flags, float* out)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    if (!params || !out) return set_err(ctx, NNLBM_ERR_ARG, "null parameters or output");
    Case& c = ctx->cases[ic];
    const OutputParams p = {params[0], params[1], params[2], params[3], params[4], params[5],
                            params[6], params[7], params[8], std::max(1.0, params[9])};
    if (!(p.dx > 0 && p.dt > 0) || (p.cy != 0.0 && !(p.a > 0)))
        return set_err(ctx, NNLBM_ERR_ARG, "output fields need dx > 0, dt > 0 and, with Carreau-Yasuda, a > 0");
    CK(cudaSetDevice(ctx->device));
    if ((rc = ensure_macro(ctx, c)) != NNLBM_OK) return rc;
    const size_t N = (size_t)c.N;
    uint8_t* d_wall = nullptr;
    float* d_out = nullptr;
    CK(cudaMalloc(&d_wall, N));
    const cudaError_t e = cudaMalloc(&d_out, (size_t)kOutputValues * N * sizeof(float));
    if (e != cudaSuccess) {
        cudaFree(d_wall);
        return set_err(ctx, NNLBM_ERR_OOM, "output buffer of %zu bytes: %s", (size_t)kOutputValues * N * sizeof(float),
                       cudaGetErrorString(e));
    }
    // the field values of the last step that stored them, after every step still queued
    cudaError_t err = wall_flags ? cudaMemcpyAsync(d_wall, wall_flags, N, cudaMemcpyHostToDevice, ctx->stream)
                                 : cudaMemsetAsync(d_wall, 0, N, ctx->stream);
    if (err == cudaSuccess) {
        aux_launchers(c.d.dtype).output_fields(c.args.data(), p, d_wall, d_out, ctx->stream);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(out, d_out, (size_t)kOutputValues * N * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(ctx->stream);
    cudaFree(d_wall);
    cudaFree(d_out);
    if (err != cudaSuccess) return set_err(ctx, NNLBM_ERR_CUDA, "output fields: %s", cudaGetErrorString(err));
    return NNLBM_OK;
}

int nnlbm_autotune_flags(nnlbm_ctx* ctx, int flags)
{
    if (!ctx) return NNLBM_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    static const int blocks[] = {64, 128, 256};
    const int tf = flags & (NNLBM_STEP_STATS | NNLBM_STEP_MACRO);
    for (Group& g : ctx->groups) {
        bool ready = true;
        for (int ic : g.cases) ready = ready && ctx->cases[ic].has_map && ctx->cases[ic].has_state;
        if (!ready) continue;
        int rc;
        // tune on copies of the states (populations, macro fields, mean/rms sums) so that the
        // lattices do not advance
        std::vector<void*> saved, msaved, ssaved;
        std::vector<int64_t> par, it, nst;
        for (int ic : g.cases) {
            Case& c = ctx->cases[ic];
            if ((tf & NNLBM_STEP_MACRO) && (rc = ensure_macro(ctx, c)) != NNLBM_OK) return rc;
            if ((tf & NNLBM_STEP_STATS) && (rc = ensure_stats(ctx, c)) != NNLBM_OK) return rc;
            const size_t bytes = 27 * c.q_stride * kStorageBytes[c.d.dtype];
            void* p = nullptr;
            CK(cudaMalloc(&p, bytes));
            CK(cudaMemcpyAsync(p, c.df, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
            saved.push_back(p);
            void* m = nullptr;
            if (c.d_macro) {
                const size_t mb = (size_t)M_N * c.N * c.ct_bytes;
                CK(cudaMalloc(&m, mb));
                CK(cudaMemcpyAsync(m, c.d_macro, mb, cudaMemcpyDeviceToDevice, ctx->stream));
            }
            msaved.push_back(m);
            void* st = nullptr;
            if (c.d_stats && (tf & NNLBM_STEP_STATS)) {
                const size_t sb = (size_t)6 * c.N * (c.d.stats_f64 ? 8 : 4);
                CK(cudaMalloc(&st, sb));
                CK(cudaMemcpyAsync(st, c.d_stats, sb, cudaMemcpyDeviceToDevice, ctx->stream));
            }
            ssaved.push_back(st);
            par.push_back(c.parity); it.push_back(c.iterations); nst.push_back(c.n_stats);
        }
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        // every launch shape: the staged form (fixed block), and block size x one or two cells
        // a thread; the forms other than one cell a thread only where the collision pairs
        float best = 1e30f;
        int bb = g.block;
        bool bp = g.paired, bs = g.staged;
        const bool pairs = pairs_chunks(g.dtype, g.collision), stages = can_stage(ctx, g);
        for (int form = FORM_STAGED; form >= FORM_ONE; --form) {
            if ((form == FORM_PAIRED && !pairs) || (form == FORM_STAGED && !stages)) continue;
            for (int b : blocks) {
                if (form == FORM_STAGED && b != blocks[0]) continue; // its block is fixed
                g.block = b;
                g.paired = form != FORM_ONE;
                g.staged = form == FORM_STAGED;
                g.gen++;
                if ((rc = run_group_steps(ctx, g, 3, tf, false)) != NNLBM_OK) return rc;
                CK(cudaEventRecord(e0, ctx->stream));
                if ((rc = run_group_steps(ctx, g, 10, tf, false)) != NNLBM_OK) return rc;
                CK(cudaEventRecord(e1, ctx->stream));
                CK(cudaEventSynchronize(e1));
                float ms = 0;
                CK(cudaEventElapsedTime(&ms, e0, e1));
                if (ms < best) { best = ms; bb = b; bp = g.paired; bs = g.staged; }
            }
        }
        g.block = bb;
        g.paired = bp;
        g.staged = bs;
        g.gen++; // the graphs captured another launch shape
        for (size_t j = 0; j < g.cases.size(); ++j) {
            Case& c = ctx->cases[g.cases[j]];
            c.parity = par[j]; c.iterations = it[j]; c.n_stats = nst[j];
            CK(cudaMemcpyAsync(c.df, saved[j], 27 * c.q_stride * kStorageBytes[c.d.dtype], cudaMemcpyDeviceToDevice, ctx->stream));
            if (msaved[j]) CK(cudaMemcpyAsync(c.d_macro, msaved[j], (size_t)M_N * c.N * c.ct_bytes, cudaMemcpyDeviceToDevice, ctx->stream));
            if (ssaved[j])
                CK(cudaMemcpyAsync(c.d_stats, ssaved[j], (size_t)6 * c.N * (c.d.stats_f64 ? 8 : 4), cudaMemcpyDeviceToDevice,
                                   ctx->stream));
        }
        CK(cudaStreamSynchronize(ctx->stream));
        for (void* p : saved) cudaFree(p);
        for (void* p : msaved)
            if (p) cudaFree(p);
        for (void* p : ssaved)
            if (p) cudaFree(p);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    return NNLBM_OK;
}

int nnlbm_autotune(nnlbm_ctx* ctx) { return nnlbm_autotune_flags(ctx, 0); }

int nnlbm_set_launch(nnlbm_ctx* ctx, int block, int cells_per_thread)
{
    if (!ctx) return NNLBM_ERR_ARG;
    if (block != 64 && block != 128 && block != 256)
        return set_err(ctx, NNLBM_ERR_ARG, "block size %d: use 64, 128 or 256", block);
    if (cells_per_thread != 1 && cells_per_thread != 2 && cells_per_thread != (2 | NNLBM_LAUNCH_STAGED))
        return set_err(ctx, NNLBM_ERR_ARG, "cells per thread %d: use 1, 2 or 2 | NNLBM_LAUNCH_STAGED", cells_per_thread);
    for (Group& g : ctx->groups) {
        g.block = block;
        g.paired = (cells_per_thread & 2) && pairs_chunks(g.dtype, g.collision);
        g.staged = (cells_per_thread & NNLBM_LAUNCH_STAGED) && can_stage(ctx, g);
        g.gen++; // the graphs captured another launch shape
    }
    return NNLBM_OK;
}

int nnlbm_get_launch(nnlbm_ctx* ctx, int ic, int* block, int* cells_per_thread)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    const Group& g = ctx->groups[ctx->cases[ic].group];
    if (block) *block = g.staged ? kStagedThreads : g.block;
    if (cells_per_thread) *cells_per_thread = g.staged ? (2 | NNLBM_LAUNCH_STAGED) : g.paired ? 2 : 1;
    return NNLBM_OK;
}

int nnlbm_step_info(nnlbm_ctx* ctx, int ic, int64_t* fluid_cells, int64_t* bc_cells, int64_t* launches_per_step,
                    double* bytes_per_step)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    Case& c = ctx->cases[ic];
    Group& g = ctx->groups[c.group];
    CK(cudaSetDevice(ctx->device));
    if ((rc = prepare_group(ctx, g)) != NNLBM_OK) return rc;
    if (fluid_cells) *fluid_cells = c.n_fluid;
    if (bc_cells) *bc_cells = c.n_bc;
    if (launches_per_step) *launches_per_step = 1 + (g.n_gather > 0 ? 1 : 0) + (g.any_refd ? 2 : 0);
    if (bytes_per_step) *bytes_per_step = (double)c.n_fluid * (54.0 * kStorageBytes[c.d.dtype] + 1.0);
    return NNLBM_OK;
}

int nnlbm_profile_step(nnlbm_ctx* ctx, int ic, int64_t n_steps, int flags, double* ms, int64_t* launches)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    if (!ms || !launches || n_steps < 1) return set_err(ctx, NNLBM_ERR_ARG, "bad profile arguments");
    CK(cudaSetDevice(ctx->device));
    Group& g = ctx->groups[ctx->cases[ic].group];
    if ((rc = prepare_steps(ctx, g, n_steps, flags)) != NNLBM_OK) return rc;
    const AuxLaunchers& A = aux_launchers(g.dtype);
    const int per_block = g.block / kChunk;
    const dim3 cblk(g.block);
    const dim3 rgrid((std::max(g.n_chunks, 1) + per_block - 1) / per_block); // one warp per chunk
    for (int i = 0; i < 5; ++i) { ms[i] = 0; launches[i] = 0; }
    const int64_t parity = ctx->cases[g.cases[0]].parity;
    // kinds: 0 gather, 1 step, 3 CY_REF_FD velocity, 4 CY_REF_FD strain
    std::vector<cudaEvent_t> ev;
    std::vector<int> kind;
    auto mark = [&](int k) -> int {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return -1;
        ev.push_back(e);
        kind.push_back(k);
        return cudaEventRecord(e, ctx->stream) == cudaSuccess ? 0 : -1;
    };
    for (int64_t k = 0; k < n_steps; ++k) {
        const bool odd = ((parity + k) & 1) != 0;
        if (mark(-1)) return set_err(ctx, NNLBM_ERR_CUDA, "event record failed");
        if (g.any_refd) {
            A.refd_velocity(odd, rgrid, cblk, ctx->stream, g.args.data());
            mark(3);
            A.refd_stress(odd, rgrid, cblk, ctx->stream, g.args.data());
            mark(4);
        }
        if (g.n_gather > 0) {
            A.gather(odd, dim3((g.n_gather + 63) / 64), dim3(64), ctx->stream, g.args.data());
            mark(0);
        }
        const StepShape sh = step_shape(g);
        step_launcher(g.dtype, g.collision)(odd, false, sh.form, sh.grid, sh.block, ctx->stream, g.args.data());
        mark(1);
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(ctx->stream));
    for (size_t i = 1; i < ev.size(); ++i) {
        if (kind[i] < 0) continue;
        float t = 0;
        CK(cudaEventElapsedTime(&t, ev[i - 1], ev[i]));
        ms[kind[i]] += t;
        launches[kind[i]] += 1;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    finish_steps(ctx, g, n_steps, flags);
    return NNLBM_OK;
}

int nnlbm_step_noalloc(nnlbm_ctx* ctx, int64_t n_steps, int flags)
{
    if (!ctx) return NNLBM_ERR_ARG;
    if (n_steps < 0) return set_err(ctx, NNLBM_ERR_ARG, "negative step count");
    if (n_steps == 0) return NNLBM_OK;
    CK(cudaSetDevice(ctx->device));
    char* scratch = nullptr;
    int rc = noalloc_scratch(ctx, &scratch);
    if (rc != NNLBM_OK) return rc;
    const size_t n_groups = ctx->groups.size();
    if (n_groups > kNoallocGroups)
        return set_err(ctx, NNLBM_ERR_ARG, "nnlbm_step_noalloc: more than %zu launch groups", kNoallocGroups);
    // refuse everything that nnlbm_step would have to allocate, before any launch
    for (size_t gi = 0; gi < n_groups; ++gi) {
        const Group& g = ctx->groups[gi];
        if (g.dirty)
            return set_err(ctx, NNLBM_ERR_ARG, "nnlbm_step_noalloc: launch group %zu has no device work list yet; call "
                           "nnlbm_step or nnlbm_step_info once after the map is set", gi);
        const size_t need = (size_t)g.n_self * 4 * (g.dtype == NNLBM_F64 ? 8 : 4);
        if (need > NNLBM_NOALLOC_SCRATCH_BYTES - kNoallocHead)
            return set_err(ctx, NNLBM_ERR_ARG, "nnlbm_step_noalloc: launch group %zu has %lld open-plane nodes written by "
                           "their own thread, %zu bytes of scratch, above the %zu bytes of NNLBM_NOALLOC_SCRATCH_BYTES",
                           gi, (long long)g.n_self, need, (size_t)NNLBM_NOALLOC_SCRATCH_BYTES - kNoallocHead);
        int64_t parity = -1;
        for (int ic : g.cases) {
            const Case& c = ctx->cases[ic];
            if (!c.has_map || !c.has_state) return set_err(ctx, NNLBM_ERR_ARG, "case %d has no map or initial state", ic);
            if (parity >= 0 && c.parity != parity)
                return set_err(ctx, NNLBM_ERR_ARG, "cases of one launch group are at different step parities "
                               "(re-initialise or re-import all of them)");
            parity = c.parity;
            if (((flags & NNLBM_STEP_MACRO) || c.d.cy_mode == NNLBM_CY_REF_FD) && !c.d_macro)
                return set_err(ctx, NNLBM_ERR_ARG, "nnlbm_step_noalloc: case %d has no macro buffer yet; run one "
                               "nnlbm_step with NNLBM_STEP_MACRO first", ic);
            if ((flags & NNLBM_STEP_STATS) && !c.d_stats)
                return set_err(ctx, NNLBM_ERR_ARG, "nnlbm_step_noalloc: case %d has no mean/rms buffer yet; run one "
                               "nnlbm_step with NNLBM_STEP_STATS first", ic);
            if (n_steps > c.ctl_cap)
                return set_err(ctx, NNLBM_ERR_ARG, "nnlbm_step_noalloc: %lld steps exceed the %lld control rows of case %d",
                               (long long)n_steps, (long long)c.ctl_cap, ic);
        }
    }
    ctx->status_fresh = false;
    // every group's cursors start at zero; the groups run one after another in stream order,
    // so they share the node values that follow the cursors
    CK(cudaMemsetAsync(scratch, 0, 4 * sizeof(int) * n_groups, ctx->stream));
    for (size_t gi = 0; gi < n_groups; ++gi) {
        Group& g = ctx->groups[gi];
        const bool f64 = g.dtype == NNLBM_F64;
        for (int ic : g.cases) {
            Case& c = ctx->cases[ic];
            rc = f64 ? upload_ctl_rows<double>(ctx, c, n_steps, flags) : upload_ctl_rows<float>(ctx, c, n_steps, flags);
            if (rc != NNLBM_OK) return rc;
            if (flags & NNLBM_STEP_REDUCE) CK(cudaMemsetAsync(c.d_red, 0, kRedBytes, ctx->stream));
        }
        alignas(64) char args[kGroupArgsBytes];
        if (f64) noalloc_args<double>(g, gi, scratch, args);
        else noalloc_args<float>(g, gi, scratch, args);
        const AuxLaunchers& A = aux_launchers(g.dtype);
        const int per_block = g.block / kChunk;
        const dim3 cblk(g.block);
        const StepShape sh = step_shape(g);
        const dim3 rgrid((std::max(g.n_chunks, 1) + per_block - 1) / per_block); // one warp per chunk
        const int64_t parity = ctx->cases[g.cases[0]].parity;
        for (int64_t k = 0; k < n_steps; ++k) {
            const bool odd = ((parity + k) & 1) != 0;
            if (g.any_refd) {
                A.refd_velocity(odd, rgrid, cblk, ctx->stream, args);
                A.refd_stress(odd, rgrid, cblk, ctx->stream, args);
            }
            if (g.n_gather > 0) A.gather(odd, dim3((g.n_gather + 63) / 64), dim3(64), ctx->stream, args);
            step_launcher(g.dtype, g.collision)(odd, false, sh.form, sh.grid, sh.block, ctx->stream, args);
        }
        CK(cudaGetLastError());
        finish_steps(ctx, g, n_steps, flags);
    }
    // the cursors into the status block, where nnlbm_step keeps them (same layout), so that the
    // synchronous path below, or the caller's nnlbm_sync, reads them with the watchdog flags
    CK(cudaMemcpyAsync(ctx->d_status + StatusLayout(ctx->cases.size()).cur, scratch, 4 * sizeof(int) * n_groups,
                       cudaMemcpyDeviceToDevice, ctx->stream));
    for (Case& c : ctx->cases) {
        if (c.sched.empty()) continue;
        const int64_t rows = (int64_t)c.sched.size() / 3;
        if (n_steps < rows) c.sched.erase(c.sched.begin(), c.sched.begin() + 3 * n_steps);
        else c.sched.erase(c.sched.begin(), c.sched.end() - 3);
    }
    if (flags & NNLBM_STEP_ASYNC) return NNLBM_OK;
    return wait_and_check(ctx, n_steps);
}

void* nnlbm_stream(nnlbm_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int nnlbm_last_error(nnlbm_ctx* ctx, char* buf, size_t n)
{
    if (!ctx) return 0;
    if (buf && n) {
        strncpy(buf, ctx->err.c_str(), n - 1);
        buf[n - 1] = 0;
    }
    return (int)ctx->err.size();
}

int nnlbm_destroy(nnlbm_ctx* ctx)
{
    if (!ctx) return NNLBM_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (Group& g : ctx->groups) {
        for (int p = 0; p < 2; ++p)
            if (g.graph[p]) cudaGraphExecDestroy(g.graph[p]);
        void* ptrs[] = {g.d_cases, g.d_chunks, g.d_chunk_nodes, g.d_gather, g.d_nodes, g.d_bc_prof, g.d_bc_buf};
        for (void* p : ptrs)
            if (p) cudaFree(p);
    }
    for (Case& c : ctx->cases) {
        for (int k = 0; k < Case::kCtlSlots; ++k) {
            if (c.h_ctl[k]) cudaFreeHost(c.h_ctl[k]);
            if (c.ctl_done[k]) cudaEventDestroy(c.ctl_done[k]);
        }
        void* ptrs[] = {c.df_base, c.d_label, c.d_macro, c.d_stats, c.d_ctl, c.d_hw};
        for (void* p : ptrs)
            if (p) cudaFree(p);
    }
    for (auto& r : ctx->rb) {
        if (r.h) cudaFreeHost(r.h);
        if (r.done) cudaEventDestroy(r.done);
    }
    if (ctx->d_status) cudaFree(ctx->d_status);
    if (ctx->h_status) cudaFreeHost(ctx->h_status);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return NNLBM_OK;
}

} // extern "C"
