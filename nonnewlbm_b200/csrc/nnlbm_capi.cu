// nnlbm_capi.cu -- the C ABI of libnnlbm.so (declared in include/nnlbm.h): contexts, device
// buffers, the TCPC boundary setup, the per-step launch sequence and its CUDA graph.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/nnlbm.h"
#include "nnlbm_kernels.cuh"

namespace nnlbm {
#define NNLBM_DECL_STEP(DT, COL) void launch_step_##DT##_##COL(bool, dim3, dim3, cudaStream_t, const void*);
#define NNLBM_DECL_STEP_DT(DT)                                                                                        \
    NNLBM_DECL_STEP(DT, 0) NNLBM_DECL_STEP(DT, 1) NNLBM_DECL_STEP(DT, 2) NNLBM_DECL_STEP(DT, 3) NNLBM_DECL_STEP(DT, 4) \
    NNLBM_DECL_STEP(DT, 5) NNLBM_DECL_STEP(DT, 6) NNLBM_DECL_STEP(DT, 7) NNLBM_DECL_STEP(DT, 8) NNLBM_DECL_STEP(DT, 9) \
    NNLBM_DECL_STEP(DT, 10)
NNLBM_DECL_STEP_DT(0) NNLBM_DECL_STEP_DT(1) NNLBM_DECL_STEP_DT(2) NNLBM_DECL_STEP_DT(3)
#define NNLBM_DECL_BC(DT)                                                                \
    void launch_bc_gather_##DT(bool, dim3, dim3, cudaStream_t, const void*);            \
    void launch_bc_write_##DT(bool, dim3, dim3, cudaStream_t, const void*);             \
    void launch_refd_velocity_##DT(bool, dim3, dim3, cudaStream_t, const void*);        \
    void launch_refd_stress_##DT(bool, dim3, dim3, cudaStream_t, const void*);          \
    void launch_fill_eq_##DT(const void*, double, double, double, double, cudaStream_t); \
    void launch_init_macro_##DT(const void*, double, double, double, double, cudaStream_t);
NNLBM_DECL_BC(0) NNLBM_DECL_BC(1) NNLBM_DECL_BC(2) NNLBM_DECL_BC(3)

StepLauncher step_launcher(int dt, int col)
{
#define NNLBM_ROW(DT)                                                                                     \
    {launch_step_##DT##_0, launch_step_##DT##_1, launch_step_##DT##_2, launch_step_##DT##_3,             \
     launch_step_##DT##_4, launch_step_##DT##_5, launch_step_##DT##_6, launch_step_##DT##_7,             \
     launch_step_##DT##_8, launch_step_##DT##_9, launch_step_##DT##_10}
    static const StepLauncher table[4][11] = {NNLBM_ROW(0), NNLBM_ROW(1), NNLBM_ROW(2), NNLBM_ROW(3)};
    return table[dt][col];
}

struct BcLaunchers {
    StepLauncher gather, write, refd_velocity, refd_stress;
    void (*fill_eq)(const void*, double, double, double, double, cudaStream_t);
    void (*init_macro)(const void*, double, double, double, double, cudaStream_t);
};
static const BcLaunchers& bc_launchers(int dt)
{
#define NNLBM_BCROW(DT)                                                                                      \
    {launch_bc_gather_##DT, launch_bc_write_##DT, launch_refd_velocity_##DT, launch_refd_stress_##DT,      \
     launch_fill_eq_##DT, launch_init_macro_##DT}
    static const BcLaunchers t[4] = {NNLBM_BCROW(0), NNLBM_BCROW(1), NNLBM_BCROW(2), NNLBM_BCROW(3)};
    return t[dt];
}
} // namespace nnlbm

using namespace nnlbm;

namespace {

const int kStorageBytes[4] = {8, 4, 2, 2};

struct Case {
    nnlbm_case_desc d{};
    int64_t N = 0;
    int ct_bytes = 4;        // arithmetic type size (8 for F64 storage)
    double scale = 1.0;      // 16-bit storage scale
    // device buffers
    void* df = nullptr;      // 27 direction arrays
    size_t q_stride = 0;     // elements between direction arrays
    uint8_t* d_label = nullptr;
    int32_t* d_bc_cell = nullptr;
    void* d_bc_prof = nullptr;
    void* d_bc_buf = nullptr;
    void* d_macro = nullptr;
    void* d_stats = nullptr;
    void* d_ctl = nullptr;
    int64_t ctl_cap = 0;
    int* d_ints = nullptr;   // cursor, done, err
    double* d_red = nullptr;
    // host state
    std::vector<uint8_t> label;
    std::vector<int32_t> bc_cell;
    std::vector<double> bc_prof;     // [n_bc][3]
    int64_t n_fluid = 0, left_area = 0, right_area = 0, n_inflow_eq = 0;
    double ivc_flux = 0, svc_flux = 0, rho_left = 1, rho_right = 1, rho_eq = 1;
    std::vector<double> sched;       // rows of {ivc_flux, svc_flux, profile_scale}
    int64_t parity = 0;              // steps done since the layout was last reset, mod 2
    int64_t iterations = 0;
    int64_t n_stats = 0;
    bool has_map = false, has_state = false;
    int bx = 64, by = 4;
    // one captured step per A-A parity
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    uint64_t graph_gen = ~0ull, gen = 0;
    std::vector<char> args;          // KArgs<CT>
};

} // namespace

struct nnlbm_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<Case> cases;
    std::string err;
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

template <class CT>
void fill_args(Case& c, KArgs<CT>& a)
{
    memset(&a, 0, sizeof a);
    const size_t eb = kStorageBytes[c.d.dtype];
    for (int q = 0; q < 27; ++q) a.dfq[q] = (char*)c.df + (size_t)q * c.q_stride * eb;
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
    a.cursor = c.d_ints; a.done = c.d_ints + 1; a.err = c.d_ints + 2;
    a.red = c.d_red;
    a.bc_cell = c.d_bc_cell; a.bc_prof = (const CT*)c.d_bc_prof; a.bc_buf = (CT*)c.d_bc_buf;
    a.n_bc = (int)c.bc_cell.size();
}

void rebuild_args(Case& c)
{
    if (c.ct_bytes == 8) {
        c.args.resize(sizeof(KArgs<double>));
        fill_args<double>(c, *(KArgs<double>*)c.args.data());
    } else {
        c.args.resize(sizeof(KArgs<float>));
        fill_args<float>(c, *(KArgs<float>*)c.args.data());
    }
    c.gen++;
}

int check_case(nnlbm_ctx* ctx, int ic)
{
    if (!ctx) return NNLBM_ERR_ARG;
    if (ic < 0 || ic >= (int)ctx->cases.size()) return set_err(ctx, NNLBM_ERR_ARG, "case index %d out of range", ic);
    return NNLBM_OK;
}

// upload a host vector of doubles to a device array of the case's arithmetic type
int upload_ct(nnlbm_ctx* ctx, Case& c, void** dptr, const std::vector<double>& v)
{
    if (*dptr) { cudaFree(*dptr); *dptr = nullptr; }
    size_t n = std::max<size_t>(v.size(), 1);
    CK(cudaMalloc(dptr, n * c.ct_bytes));
    if (!v.empty()) {
        if (c.ct_bytes == 8) {
            CK(cudaMemcpy(*dptr, v.data(), v.size() * 8, cudaMemcpyHostToDevice));
        } else {
            std::vector<float> f(v.begin(), v.end());
            CK(cudaMemcpy(*dptr, f.data(), f.size() * 4, cudaMemcpyHostToDevice));
        }
    }
    return NNLBM_OK;
}

int ensure_macro(nnlbm_ctx* ctx, Case& c)
{
    if (c.d_macro) return NNLBM_OK;
    CK(cudaMalloc(&c.d_macro, (size_t)M_N * c.N * c.ct_bytes));
    rebuild_args(c);
    bc_launchers(c.d.dtype).init_macro(c.args.data(), 1.0, 0.0, 0.0, 0.0, ctx->stream);
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
    rebuild_args(c);
    return NNLBM_OK;
}

int ensure_ctl(nnlbm_ctx* ctx, Case& c, int64_t n)
{
    if (c.ctl_cap >= n && c.d_ctl) return NNLBM_OK;
    int64_t cap = std::max<int64_t>(n, 1024);
    if (c.d_ctl) cudaFree(c.d_ctl);
    c.d_ctl = nullptr;
    const size_t row = c.ct_bytes == 8 ? sizeof(StepCtl<double>) : sizeof(StepCtl<float>);
    CK(cudaMalloc(&c.d_ctl, cap * row));
    c.ctl_cap = cap;
    rebuild_args(c);
    return NNLBM_OK;
}

template <class CT>
void fill_ctl(Case& c, std::vector<char>& buf, int64_t n, int flags)
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
        // inflow_right = -svc_flux (sim_tcpc.cu:660)
        r[k].u_left = (CT)(c.left_area > 0 ? (CT)ivc / (CT)c.left_area : 0);
        r[k].u_right = (CT)(c.right_area > 0 ? (CT)(-svc) / (CT)c.right_area : 0);
        r[k].rho_left = (CT)c.rho_left; r[k].rho_right = (CT)c.rho_right; r[k].rho_eq = (CT)c.rho_eq;
        r[k].prof_scale = (CT)ps;
    }
}

// enqueue one step (no host synchronisation); `odd` is the A-A parity of this step
int enqueue_step(nnlbm_ctx* ctx, Case& c, bool odd)
{
    const BcLaunchers& B = bc_launchers(c.d.dtype);
    const dim3 blk(c.bx, c.by, 1);
    const dim3 grd((c.d.nx + c.bx - 1) / c.bx, (c.d.ny + c.by - 1) / c.by, c.d.nz);
    const int nbc = (int)c.bc_cell.size();
    const dim3 bgrd((std::max(nbc, 1) + 127) / 128), bblk(128);
    if (c.d.cy_mode == NNLBM_CY_REF_FD) {
        B.refd_velocity(odd, grd, blk, ctx->stream, c.args.data());
        B.refd_stress(odd, grd, blk, ctx->stream, c.args.data());
    }
    B.gather(odd, bgrd, bblk, ctx->stream, c.args.data());
    step_launcher(c.d.dtype, c.d.collision)(odd, grd, blk, ctx->stream, c.args.data());
    B.write(odd, bgrd, bblk, ctx->stream, c.args.data());
    CK(cudaGetLastError());
    return NNLBM_OK;
}

int ensure_graphs(nnlbm_ctx* ctx, Case& c)
{
    if (c.graph[0] && c.graph[1] && c.graph_gen == c.gen) return NNLBM_OK;
    for (int p = 0; p < 2; ++p) {
        if (c.graph[p]) { cudaGraphExecDestroy(c.graph[p]); c.graph[p] = nullptr; }
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_step(ctx, c, p == 1);
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
        if (rc != NNLBM_OK) { if (g) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) return set_err(ctx, NNLBM_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
        e = cudaGraphInstantiate(&c.graph[p], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return set_err(ctx, NNLBM_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
    }
    c.graph_gen = c.gen;
    return NNLBM_OK;
}

int run_case_steps(nnlbm_ctx* ctx, Case& c, int64_t n, int flags, bool use_graph)
{
    int rc;
    if ((flags & NNLBM_STEP_MACRO) || c.d.cy_mode == NNLBM_CY_REF_FD) {
        if ((rc = ensure_macro(ctx, c)) != NNLBM_OK) return rc;
    }
    if (flags & NNLBM_STEP_STATS) {
        if ((rc = ensure_stats(ctx, c)) != NNLBM_OK) return rc;
    }
    if ((rc = ensure_ctl(ctx, c, n)) != NNLBM_OK) return rc;
    std::vector<char> buf;
    if (c.ct_bytes == 8) fill_ctl<double>(c, buf, n, flags);
    else fill_ctl<float>(c, buf, n, flags);
    CK(cudaMemcpyAsync(c.d_ctl, buf.data(), buf.size(), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync(c.d_ints, 0, 2 * sizeof(int), ctx->stream)); // cursor, done
    if (use_graph && (rc = ensure_graphs(ctx, c)) != NNLBM_OK) return rc;
    for (int64_t k = 0; k < n; ++k) {
        const int p = (int)((c.parity + k) & 1);
        if (use_graph) CK(cudaGraphLaunch(c.graph[p], ctx->stream));
        else if ((rc = enqueue_step(ctx, c, p == 1)) != NNLBM_OK) return rc;
    }
    c.parity = (c.parity + n) & 1;
    c.iterations += n;
    if (flags & NNLBM_STEP_STATS) c.n_stats += n;
    return NNLBM_OK;
}

bool is_bc(int lab) { return lab >= L_IN_L && lab <= L_OUT_REQ; }

// storage element <-> double on the host
double decode(const Case& c, const void* base, size_t i, int q)
{
    const double w = q == 13 ? 8.0 / 27.0 : (nnzq(q) == 1 ? 2.0 / 27.0 : (nnzq(q) == 2 ? 1.0 / 54.0 : 1.0 / 216.0));
    switch (c.d.dtype) {
    case NNLBM_F64: return ((const double*)base)[i];
    case NNLBM_F32: return (double)(weight<float>(q) + ((const float*)base)[i]);
    case NNLBM_F16: return (double)(weight<float>(q) + __half2float(((const __half*)base)[i]) * (float)(1.0 / c.scale));
    default: return (double)(weight<float>(q) + __bfloat162float(((const __nv_bfloat16*)base)[i]) * (float)(1.0 / c.scale));
    }
    (void)w;
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
    *slot = q; // after an odd step (or the initial state): slot q at x + c_q
    const int xx = (x + cxq(q) + nx) % nx, yy = (y + cyq(q) + ny) % ny, zz = (z + czq(q) + nz) % nz;
    return (size_t)xx + (size_t)nx * (yy + (size_t)ny * zz);
}

} // namespace

// ======================================================================================
// C ABI
// ======================================================================================
extern "C" {

int nnlbm_create(const nnlbm_case_desc* desc, int n_cases, int device, nnlbm_ctx** out)
{
    if (!desc || n_cases < 1 || !out) return NNLBM_ERR_ARG;
    *out = nullptr;
    nnlbm_ctx* ctx = new nnlbm_ctx();
    ctx->device = device;
    auto fail = [&](int rc) { nnlbm_destroy(ctx); return rc; };
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        // the context is returned so that the caller can read the message
        set_err(ctx, NNLBM_ERR_CUDA, "no CUDA device %d (found %d)", device, ndev);
        *out = ctx;
        return NNLBM_ERR_CUDA;
    }
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        set_err(ctx, NNLBM_ERR_CUDA, "cannot initialise device %d", device);
        *out = ctx;
        return NNLBM_ERR_CUDA;
    }
    ctx->cases.resize(n_cases);
    for (int i = 0; i < n_cases; ++i) {
        Case& c = ctx->cases[i];
        c.d = desc[i];
        const nnlbm_case_desc& d = c.d;
        if (d.nx < 3 || d.ny < 3 || d.nz < 3 || d.dtype < 0 || d.dtype > 3 || d.collision < 0 || d.collision > 10 ||
            d.equilibrium < 0 || d.equilibrium > 3 || d.cy_mode < 0 || d.cy_mode > 2 || !(d.nu > 0)) {
            set_err(ctx, NNLBM_ERR_ARG, "case %d: invalid descriptor (dims >= 3, dtype 0..3, collision 0..10, "
                    "equilibrium 0..3, cy_mode 0..2, nu > 0)", i);
            *out = ctx;
            return NNLBM_ERR_ARG;
        }
        if (d.cy_mode != NNLBM_CY_NONE && !(d.cy_a > 0 && d.cy_nu0 > 0)) {
            set_err(ctx, NNLBM_ERR_ARG, "case %d: Carreau-Yasuda needs a > 0 and nu0 > 0", i);
            *out = ctx;
            return NNLBM_ERR_ARG;
        }
        c.N = (int64_t)d.nx * d.ny * d.nz;
        if (c.N >= (int64_t)1 << 31) {
            set_err(ctx, NNLBM_ERR_ARG, "case %d: %lld cells exceed 2^31", i, (long long)c.N);
            *out = ctx;
            return NNLBM_ERR_ARG;
        }
        c.ct_bytes = d.dtype == NNLBM_F64 ? 8 : 4;
        c.scale = d.storage_scale > 0 ? d.storage_scale : (d.dtype == NNLBM_F16 ? 1024.0 : 1.0);
        if (d.dtype == NNLBM_F64 || d.dtype == NNLBM_F32) c.scale = 1.0;
        const size_t eb = kStorageBytes[d.dtype];
        c.q_stride = ((size_t)c.N + 127) / 128 * 128;
        if (cudaMalloc(&c.df, 27 * c.q_stride * eb) != cudaSuccess ||
            cudaMalloc(&c.d_label, (size_t)c.N) != cudaSuccess ||
            cudaMalloc(&c.d_ints, 4 * sizeof(int)) != cudaSuccess || cudaMalloc(&c.d_red, 8 * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            set_err(ctx, NNLBM_ERR_OOM, "case %d: device allocation of %.2f GB failed", i, 27.0 * c.q_stride * eb / 1e9);
            *out = ctx;
            return NNLBM_ERR_OOM;
        }
        cudaMemset(c.d_ints, 0, 4 * sizeof(int));
        cudaMemset(c.d_red, 0, 8 * sizeof(double));
        c.label.assign((size_t)c.N, (uint8_t)NNLBM_WALL);
        if (upload_ct(ctx, c, &c.d_bc_prof, {}) != NNLBM_OK || upload_ct(ctx, c, &c.d_bc_buf, {}) != NNLBM_OK) {
            *out = ctx;
            return NNLBM_ERR_OOM;
        }
        int rc = ensure_ctl(ctx, c, 1024);
        if (rc != NNLBM_OK) { *out = ctx; return rc; }
        rebuild_args(c);
    }
    (void)fail;
    *out = ctx;
    return NNLBM_OK;
}

int nnlbm_set_map(nnlbm_ctx* ctx, int ic, const uint8_t* map)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    if (!map) return set_err(ctx, NNLBM_ERR_ARG, "null map");
    Case& c = ctx->cases[ic];
    const int nx = c.d.nx, ny = c.d.ny, nz = c.d.nz;
    int64_t nfl = 0, la = 0, ra = 0, neq = 0;
    std::vector<int32_t> bcs;
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const int64_t i = x + (int64_t)nx * (y + (int64_t)ny * z);
                const int lab = map[i];
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
                if (is_bc(lab)) bcs.push_back((int32_t)i);
            }
    c.label.assign(map, map + c.N);
    c.bc_cell = bcs;
    c.bc_prof.assign(bcs.size() * 3, 0.0);
    c.n_fluid = nfl; c.left_area = la; c.right_area = ra; c.n_inflow_eq = neq;
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpy(c.d_label, map, (size_t)c.N, cudaMemcpyHostToDevice));
    if (c.d_bc_cell) { cudaFree(c.d_bc_cell); c.d_bc_cell = nullptr; }
    CK(cudaMalloc(&c.d_bc_cell, std::max<size_t>(bcs.size(), 1) * sizeof(int32_t)));
    if (!bcs.empty()) CK(cudaMemcpy(c.d_bc_cell, bcs.data(), bcs.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    if ((rc = upload_ct(ctx, c, &c.d_bc_prof, c.bc_prof)) != NNLBM_OK) return rc;
    std::vector<double> zeros(bcs.size() * 4, 0.0);
    if ((rc = upload_ct(ctx, c, &c.d_bc_buf, zeros)) != NNLBM_OK) return rc;
    c.has_map = true;
    rebuild_args(c);
    return NNLBM_OK;
}

// StateTcpc::setupBoundaries (sim_tcpc.cu:494-645) + LBM::projectWall (lbm.hpp:144-155)
int nnlbm_setup_tcpc(nnlbm_ctx* ctx, int ic, const int32_t* wall, int64_t* counts)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    if (!wall) return set_err(ctx, NNLBM_ERR_ARG, "null wall array");
    Case& c = ctx->cases[ic];
    const int X = c.d.nx, Y = c.d.ny, Z = c.d.nz;
    auto id = [&](int x, int y, int z) { return (size_t)x + (size_t)X * (y + (size_t)Y * z); };
    std::vector<uint8_t> map((size_t)c.N, (uint8_t)L_FLUID), wf((size_t)c.N, 0);
    int64_t in[7] = {0};
    for (size_t i = 0; i < (size_t)c.N; ++i) {
        const int lab = wall[i];
        if (lab >= 3 && lab <= 6) in[lab]++;
        wf[i] = lab == 1;
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
        int s = b + step;
        auto cell = [&](int a, int u, int z) { return axis == 0 ? id(a, u, z) : id(u, a, z); };
        const int nu = axis == 0 ? Y : X;
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
    for (size_t i = 0; i < (size_t)c.N; ++i) {
        const int lab = map[i];
        const bool w = wf[i] || lab == L_WALL;
        la += lab == L_IN_L && !w; ra += lab == L_IN_R && !w;
        of += lab == L_OUT_F && !w; ob += lab == L_OUT_B && !w;
        wc += w; fc += lab == L_FLUID && !w;
    }
    for (size_t i = 0; i < (size_t)c.N; ++i)
        if (wf[i]) map[i] = L_WALL;
    if (counts) {
        const int64_t v[10] = {la, ra, of, ob, wc, fc, in[3], in[4], in[5], in[6]};
        memcpy(counts, v, sizeof v);
    }
    if ((rc = nnlbm_set_map(ctx, ic, map.data())) != NNLBM_OK) return rc;
    if (la <= 0 || ra <= 0 || of <= 0 || ob <= 0)
        return set_err(ctx, NNLBM_ERR_AREA, "zero inlet or outlet area: left=%lld right=%lld outlet5=%lld outlet6=%lld",
                       (long long)la, (long long)ra, (long long)of, (long long)ob);
    return NNLBM_OK;
}

int nnlbm_init_equilibrium(nnlbm_ctx* ctx, int ic, double rho, double ux, double uy, double uz)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    Case& c = ctx->cases[ic];
    if (!c.has_map) return set_err(ctx, NNLBM_ERR_ARG, "set the map before the initial state");
    CK(cudaSetDevice(ctx->device));
    const BcLaunchers& B = bc_launchers(c.d.dtype);
    B.fill_eq(c.args.data(), rho, ux, uy, uz, ctx->stream);
    CK(cudaGetLastError());
    if (c.d_macro) B.init_macro(c.args.data(), rho, ux, uy, uz, ctx->stream);
    if (c.d_stats) CK(cudaMemsetAsync(c.d_stats, 0, (size_t)6 * c.N * (c.d.stats_f64 ? 8 : 4), ctx->stream));
    CK(cudaMemsetAsync(c.d_ints, 0, 3 * sizeof(int), ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    c.parity = 0; c.iterations = 0; c.n_stats = 0;
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
    for (size_t b = 0; b < c.bc_cell.size(); ++b)
        if (c.label[c.bc_cell[b]] == L_IN_EQ) {
            for (int j = 0; j < 3; ++j) c.bc_prof[3 * b + j] = u[3 * k + j];
            ++k;
        }
    CK(cudaSetDevice(ctx->device));
    if ((rc = upload_ct(ctx, c, &c.d_bc_prof, c.bc_prof)) != NNLBM_OK) return rc;
    rebuild_args(c);
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
    CK(cudaSetDevice(ctx->device));
    for (size_t i = 0; i < ctx->cases.size(); ++i) {
        Case& c = ctx->cases[i];
        if (!c.has_map || !c.has_state) return set_err(ctx, NNLBM_ERR_ARG, "case %zu has no map or initial state", i);
        int rc = run_case_steps(ctx, c, n_steps, flags, true);
        if (rc != NNLBM_OK) return rc;
        if (!c.sched.empty()) {
            // consume the rows that were used
            const int64_t used = std::min<int64_t>(n_steps, (int64_t)c.sched.size() / 3);
            if (used < (int64_t)c.sched.size() / 3) c.sched.erase(c.sched.begin(), c.sched.begin() + 3 * used);
            else c.sched.erase(c.sched.begin(), c.sched.end() - 3); // keep the last row
        }
    }
    std::vector<int> errs(ctx->cases.size() * 3);
    for (size_t i = 0; i < ctx->cases.size(); ++i)
        CK(cudaMemcpyAsync(&errs[3 * i], ctx->cases[i].d_ints, 3 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (size_t i = 0; i < ctx->cases.size(); ++i) {
        if (errs[3 * i] != n_steps)
            return set_err(ctx, NNLBM_ERR_CUDA, "case %zu: step cursor %d after %lld steps", i, errs[3 * i], (long long)n_steps);
        if (errs[3 * i + 2])
            return set_err(ctx, NNLBM_ERR_NAN, "case %zu: density left (0.25, 4) or became non-finite", i);
    }
    return NNLBM_OK;
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
    if (!c.d_macro) return set_err(ctx, NNLBM_ERR_ARG, "no macro state yet: run a step with NNLBM_STEP_MACRO");
    CK(cudaSetDevice(ctx->device));
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
    if (c.d.stats_f64) {
        CK(cudaMemcpy(out, c.d_stats, n * 8, cudaMemcpyDeviceToHost));
    } else {
        std::vector<float> tmp(n);
        CK(cudaMemcpy(tmp.data(), c.d_stats, n * 4, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < n; ++i) out[i] = tmp[i];
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
                    int slot;
                    const size_t i = canon_index(c, x, y, z, q, &slot);
                    encode(c, raw.data() + (size_t)slot * c.q_stride * eb, i, q,
                           in[(size_t)q * c.N + x + (size_t)nx * (y + (size_t)ny * z)]);
                }
    CK(cudaMemcpy(c.df, raw.data(), raw.size(), cudaMemcpyHostToDevice));
    c.has_state = true;
    return NNLBM_OK;
}

int nnlbm_reduce(nnlbm_ctx* ctx, int ic, double* out5)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    if (!out5) return set_err(ctx, NNLBM_ERR_ARG, "null output");
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpy(out5, ctx->cases[ic].d_red, 5 * sizeof(double), cudaMemcpyDeviceToHost));
    return NNLBM_OK;
}

int nnlbm_autotune(nnlbm_ctx* ctx)
{
    if (!ctx) return NNLBM_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    static const int shapes[][2] = {{32, 4}, {32, 8}, {64, 2}, {64, 4}, {128, 1}, {128, 2}, {256, 1}};
    for (Case& c : ctx->cases) {
        if (!c.has_map || !c.has_state) continue;
        // tune on a copy of the state so that the lattice does not advance
        const size_t eb = kStorageBytes[c.d.dtype];
        const size_t bytes = 27 * c.q_stride * eb;
        void* save = nullptr;
        CK(cudaMalloc(&save, bytes));
        CK(cudaMemcpyAsync(save, c.df, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
        void* msave = nullptr;
        const size_t mbytes = (size_t)M_N * c.N * c.ct_bytes;
        if (c.d_macro) {
            CK(cudaMalloc(&msave, mbytes));
            CK(cudaMemcpyAsync(msave, c.d_macro, mbytes, cudaMemcpyDeviceToDevice, ctx->stream));
        }
        const int64_t parity0 = c.parity, it0 = c.iterations;
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        float best = 1e30f;
        int bbx = c.bx, bby = c.by;
        for (auto& s : shapes) {
            c.bx = s[0]; c.by = s[1];
            int rc = run_case_steps(ctx, c, 2, 0, false);
            if (rc) return rc;
            CK(cudaEventRecord(e0, ctx->stream));
            rc = run_case_steps(ctx, c, 6, 0, false);
            if (rc) return rc;
            CK(cudaEventRecord(e1, ctx->stream));
            CK(cudaEventSynchronize(e1));
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            if (ms < best) { best = ms; bbx = s[0]; bby = s[1]; }
        }
        c.bx = bbx; c.by = bby;
        c.parity = parity0; c.iterations = it0;
        CK(cudaMemcpyAsync(c.df, save, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
        if (msave) CK(cudaMemcpyAsync(c.d_macro, msave, mbytes, cudaMemcpyDeviceToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        cudaFree(save);
        if (msave) cudaFree(msave);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        c.gen++; // the graph captured the old launch shape
    }
    return NNLBM_OK;
}

int nnlbm_step_info(nnlbm_ctx* ctx, int ic, int64_t* fluid_cells, int64_t* bc_cells, int64_t* launches_per_step,
                    double* bytes_per_step)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    Case& c = ctx->cases[ic];
    if (fluid_cells) *fluid_cells = c.n_fluid;
    if (bc_cells) *bc_cells = (int64_t)c.bc_cell.size();
    if (launches_per_step) *launches_per_step = c.d.cy_mode == NNLBM_CY_REF_FD ? 5 : 3;
    if (bytes_per_step) *bytes_per_step = (double)c.n_fluid * (54.0 * kStorageBytes[c.d.dtype] + 1.0);
    return NNLBM_OK;
}

int nnlbm_profile_step(nnlbm_ctx* ctx, int ic, int64_t n_steps, int flags, double* ms, int64_t* launches)
{
    int rc = check_case(ctx, ic);
    if (rc) return rc;
    if (!ms || !launches || n_steps < 1) return set_err(ctx, NNLBM_ERR_ARG, "bad profile arguments");
    Case& c = ctx->cases[ic];
    if (!c.has_map || !c.has_state) return set_err(ctx, NNLBM_ERR_ARG, "case has no map or initial state");
    CK(cudaSetDevice(ctx->device));
    if ((flags & NNLBM_STEP_MACRO) || c.d.cy_mode == NNLBM_CY_REF_FD)
        if ((rc = ensure_macro(ctx, c)) != NNLBM_OK) return rc;
    if (flags & NNLBM_STEP_STATS)
        if ((rc = ensure_stats(ctx, c)) != NNLBM_OK) return rc;
    if ((rc = ensure_ctl(ctx, c, n_steps)) != NNLBM_OK) return rc;
    std::vector<char> buf;
    if (c.ct_bytes == 8) fill_ctl<double>(c, buf, n_steps, flags);
    else fill_ctl<float>(c, buf, n_steps, flags);
    CK(cudaMemcpyAsync(c.d_ctl, buf.data(), buf.size(), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync(c.d_ints, 0, 2 * sizeof(int), ctx->stream));
    const BcLaunchers& B = bc_launchers(c.d.dtype);
    const dim3 blk(c.bx, c.by, 1);
    const dim3 grd((c.d.nx + c.bx - 1) / c.bx, (c.d.ny + c.by - 1) / c.by, c.d.nz);
    const int nbc = (int)c.bc_cell.size();
    const dim3 bgrd((std::max(nbc, 1) + 127) / 128), bblk(128);
    const bool refd = c.d.cy_mode == NNLBM_CY_REF_FD;
    const int nk = refd ? 5 : 3;
    std::vector<cudaEvent_t> ev((size_t)n_steps * (nk + 1));
    for (auto& e : ev) CK(cudaEventCreate(&e));
    for (int64_t k = 0; k < n_steps; ++k) {
        const bool odd = ((c.parity + k) & 1) != 0;
        cudaEvent_t* e = &ev[(size_t)k * (nk + 1)];
        int j = 0;
        CK(cudaEventRecord(e[j++], ctx->stream));
        if (refd) {
            B.refd_velocity(odd, grd, blk, ctx->stream, c.args.data());
            CK(cudaEventRecord(e[j++], ctx->stream));
            B.refd_stress(odd, grd, blk, ctx->stream, c.args.data());
            CK(cudaEventRecord(e[j++], ctx->stream));
        }
        B.gather(odd, bgrd, bblk, ctx->stream, c.args.data());
        CK(cudaEventRecord(e[j++], ctx->stream));
        step_launcher(c.d.dtype, c.d.collision)(odd, grd, blk, ctx->stream, c.args.data());
        CK(cudaEventRecord(e[j++], ctx->stream));
        B.write(odd, bgrd, bblk, ctx->stream, c.args.data());
        CK(cudaEventRecord(e[j++], ctx->stream));
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(ctx->stream));
    for (int i = 0; i < 5; ++i) { ms[i] = 0; launches[i] = 0; }
    // kinds in launch order: [refd velocity, refd strain,] gather, step, write
    const int kinds_refd[5] = {3, 4, 0, 1, 2}, kinds[3] = {0, 1, 2};
    for (int64_t k = 0; k < n_steps; ++k) {
        cudaEvent_t* e = &ev[(size_t)k * (nk + 1)];
        for (int j = 0; j < nk; ++j) {
            float t = 0;
            CK(cudaEventElapsedTime(&t, e[j], e[j + 1]));
            const int kind = refd ? kinds_refd[j] : kinds[j];
            ms[kind] += t;
            launches[kind] += 1;
        }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    c.parity = (c.parity + n_steps) & 1;
    c.iterations += n_steps;
    if (flags & NNLBM_STEP_STATS) c.n_stats += n_steps;
    return NNLBM_OK;
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
    for (Case& c : ctx->cases) {
        for (int p = 0; p < 2; ++p)
            if (c.graph[p]) cudaGraphExecDestroy(c.graph[p]);
        void* ptrs[] = {c.df, c.d_label, c.d_bc_cell, c.d_bc_prof, c.d_bc_buf, c.d_macro, c.d_stats, c.d_ctl, c.d_ints, c.d_red};
        for (void* p : ptrs)
            if (p) cudaFree(p);
    }
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return NNLBM_OK;
}

} // extern "C"
