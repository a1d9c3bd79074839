// C ABI of libcutcell_b200.so: contexts, cooperative launches, status codes.
// The persistent kernels live in pcg.cuh / ops.cuh.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <cstring>
#include <string>

#include "pcg.cuh"
#include "learned.cuh"
#include "coarse.cuh"
#include "fastdiag.cuh"
#include "kron.cuh"
#include "dgemm.cuh"

namespace {

thread_local std::string g_last_error;

int cuda_fail(cudaError_t e, const char* what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return CUTCELL_E_CUDA;
}

#define CK(call)                                          \
    do {                                                  \
        cudaError_t _e = (call);                          \
        if (_e != cudaSuccess) return cuda_fail(_e, #call); \
    } while (0)

enum { KIND_CSR = 0, KIND_TILES = 1, KIND_KRON = 2 };
constexpr int BAR_WORDS = 160;

__global__ void csr_diag_inv_kernel(int n, const int* ptr, const int* idx, const double* val, double* dinv) {
    for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
        double d = 0.0;
        for (int k = ptr[row]; k < ptr[row + 1]; ++k)
            if (idx[k] == row) d += val[k];
        dinv[row] = (fabs(d) > 0.0) ? 1.0 / d : 1.0;
    }
}

// One grid barrier over a cooperative grid that waits for `arrivals`
// arrivals (the diagnostic of cutcell_barrier_selftest).
__global__ void barrier_probe_kernel(GridSync gs) { grid_sync(gs); }

__global__ void fill_kernel(int n, double v, double* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = v;
}

__global__ void diag_inv_kernel(int n, const double* diag, double* dinv) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double d = diag[i];
        dinv[i] = (fabs(d) > 0.0) ? 1.0 / d : 1.0;
    }
}

__global__ void to_f32_kernel(size_t n, const double* in, float* out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

// two-plane BF16: hi = bf16(v), lo = bf16(v - hi)
__global__ void to_bf16x2_kernel(size_t n, const double* in, bf16x2_t* out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double v = in[i];
        const __nv_bfloat16 h = __float2bfloat16_rn((float)v);
        out[i].hi = h;
        out[i].lo = __float2bfloat16_rn((float)(v - (double)__bfloat162float(h)));
    }
}

// Dense symmetric 64 x 64 cut blocks -> the 2080-entry split storage of
// sym64_index (upper triangle, row <= column, of each row-major block).
__global__ void pack_sym64_kernel(int n_cut, const double* dense, double* packed) {
    const size_t n = (size_t)n_cut * 64 * 64;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const int e = (int)(k / 4096), i = (int)((k / 64) % 64), j = (int)(k % 64);
        if (i <= j) packed[(size_t)e * SYM64_ENTRIES + sym64_index(i, j)] = dense[k];
    }
}

__global__ void ext_gather_kernel(ExtDev e, const double* xr, double* xf) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < e.n_full; i += gridDim.x * blockDim.x)
        xf[i] = e.gather(xr, i);
}

__global__ void ext_scatter_kernel(ExtDev e, const double* yf, double* yr) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < e.n_red; j += gridDim.x * blockDim.x) {
        double y = yf[e.full_of_red[j]];
        for (int k = e.smallT_ptr[j]; k < e.smallT_ptr[j + 1]; ++k) y += e.smallT_val[k] * yf[e.smallT_row[k]];
        yr[j] = y;
    }
}

template <class K>
int occupancy_blocks(K kernel, size_t smem, int* out) {
    int dev = 0, sms = 0, per = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (smem > 48 * 1024) CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, CUTCELL_BLOCK, smem));
    if (per < 1) {
        g_last_error = "kernel does not fit on an SM";
        return CUTCELL_E_CUDA;
    }
    *out = sms * per;
    return CUTCELL_OK;
}

}  // namespace

struct cutcell_mlp {
    int device = 0;
    float* theta = nullptr;
    float* m = nullptr;
    float* v = nullptr;
    float* grad = nullptr;
    __nv_bfloat16* wbf = nullptr;
    int step = 0;
    int cap = 0;  // batch capacity of the training scratch
    int act = 0;  // 0 ReLU, 1 identity
    float *H1 = nullptr, *H2 = nullptr, *D1 = nullptr, *D2 = nullptr, *DY = nullptr, *Y = nullptr, *L = nullptr;
    MlpWeights weights() const { return MlpWeights{wbf, theta, act}; }
};

__global__ void sum_in_order_kernel(const float* v, int n, float scale, float* out) {
    __shared__ double sh[CUTCELL_WARPS + 1];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += v[i];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) *out = (float)(s * scale);
}

struct cutcell_fastdiag {
    int device = 0;
    FastDiagDev d;
    double *X = nullptr, *T = nullptr, *UT = nullptr, *G = nullptr, *U = nullptr, *S2 = nullptr;
    double *QxT = nullptr, *QyT = nullptr, *cosT = nullptr, *sinT = nullptr;
    double* part = nullptr;
};

struct cutcell_ctx {
    int kind = KIND_CSR;
    int n = 0;
    int device = 0;
    // CSR
    CsrOp<double> csr64;
    CsrOp<float> csr32;
    CsrOp<bf16x2_t> csr16;
    float* val32 = nullptr;
    bf16x2_t* val16 = nullptr;
    // tiles
    TileData td;
    const double* cut64 = nullptr;
    double* cutsym = nullptr;  // degree 3: owned split-storage copy of the cut blocks
    float* cut32 = nullptr;
    bf16x2_t* cut16 = nullptr;
    double* ypart = nullptr;
    double* ycut = nullptr;
    double* yfv = nullptr;
    double* psmall = nullptr;
    int4* need_rec = nullptr;
    int* cut_pos = nullptr;
    int4* row_rec = nullptr;
    // Kronecker cut box: banded reduced 1D factors [axis][H, K, Q, S, A]
    int kn[3] = {0, 0, 0};
    KronBand kb[3][5];
    int* klo = nullptr;
    double* kband = nullptr;
    double* kscratch = nullptr;  // U1 U2 V1 V2
    // scratch
    double* dinv = nullptr;
    double* ones = nullptr;
    bool use_jacobi = true;
    double* r = nullptr;
    double* p = nullptr;
    double* p2 = nullptr;
    double* Ap = nullptr;
    double* d = nullptr;
    double* rhat = nullptr;
    double* part = nullptr;
    unsigned* bar = nullptr;  // control words, one 128-byte line each: [0] arrival, [32] err, [64] tile work, [96] cut work, [128..] debug
    DevResult* res = nullptr;
    int max_blocks = 0;
    // learned preconditioner
    cutcell_mlp* mlp = nullptr;
    PatchMap pmap = {0, nullptr, nullptr, nullptr, nullptr};
    int* pslot_all = nullptr;  // identity patch -> block map of cutcell_pcg_set_block_inverses
    double* zl = nullptr;
    double* rold = nullptr;
    // two-level preconditioner: coarse-grid tables (caller-owned) and work arrays
    bool has_coarse = false;
    CoarseDev coarse = {};
    double* cwork = nullptr;  // t1 | rc | yc | zc | azc
    double* czx[ZSUM_MAX] = {nullptr, nullptr, nullptr};  // the extra tilings' corrections
    // reduced-precision forms: residual-replacement factor and cap
    double inner_tol = 0.1;
    int inner_maxiter = 0;
    int max_outer = 200;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

static int alloc_scratch(cutcell_ctx* c) {
    const size_t nb = (size_t)c->n * sizeof(double);
    CK(cudaMalloc(&c->dinv, nb));
    CK(cudaMalloc(&c->ones, nb));
    fill_kernel<<<ceil_div(c->n, 256), 256>>>(c->n, 1.0, c->ones);
    CK(cudaMalloc(&c->r, nb));
    CK(cudaMalloc(&c->p, nb));
    CK(cudaMalloc(&c->p2, nb));
    CK(cudaMalloc(&c->Ap, nb));
    CK(cudaMalloc(&c->d, nb));
    CK(cudaMalloc(&c->rhat, nb));
    CK(cudaMalloc(&c->bar, BAR_WORDS * sizeof(unsigned)));
    CK(cudaMalloc(&c->res, sizeof(DevResult)));
    CK(cudaEventCreate(&c->ev0));
    CK(cudaEventCreate(&c->ev1));
    return CUTCELL_OK;
}

template <class K>
static int ensure_part(cutcell_ctx* c, K kernel, size_t smem, int* blocks) {
    int st = occupancy_blocks(kernel, smem, blocks);
    if (st) return st;
    if (*blocks > c->max_blocks) {
        if (c->part) cudaFree(c->part);
        c->part = nullptr;
        CK(cudaMalloc(&c->part, (size_t)8 * (*blocks) * sizeof(double)));
        c->max_blocks = *blocks;
    }
    return CUTCELL_OK;
}

static GridSync make_gs(cutcell_ctx* c, int blocks) {
    GridSync gs;
    gs.count = c->bar;
    gs.limit_ns = cutcell_internal_wait_limit_ns();
    gs.err = (int*)(c->bar + 32);
    gs.nblocks = (unsigned)blocks;
    return gs;
}

static PcgBufs make_bufs(cutcell_ctx* c) {
    PcgBufs B;
    B.n = c->n;
    B.dinv = c->use_jacobi ? c->dinv : c->ones;
    B.r = c->r;
    B.p = c->p;
    B.Ap = c->Ap;
    B.part = c->part;
    B.p2 = c->p2;
    return B;
}

template <class K, class... Args>
static int launch_coop(K kernel, int blocks, size_t smem, cudaStream_t s, Args... args) {
    void* ptrs[] = {(void*)&args...};
    CK(cudaLaunchCooperativeKernel((const void*)kernel, dim3(blocks), dim3(CUTCELL_BLOCK), ptrs, smem, s));
    return CUTCELL_OK;
}

template <class Op>
static int run_plain(cutcell_ctx* c, const Op& op, size_t smem, SolveArgs& a, cudaStream_t s, int* blocks) {
    auto kern = pcg_kernel<Op>;
    int st = ensure_part(c, kern, smem, blocks);
    if (st) return st;
    a.gs = make_gs(c, *blocks);
    a.B = make_bufs(c);
    return launch_coop(kern, *blocks, smem, s, op, a);
}

template <class OpHi, class OpLo>
static int run_ru(cutcell_ctx* c, const OpHi& hi, const OpLo& lo, size_t smem, SolveArgs& a, cudaStream_t s,
                  int* blocks) {
    auto kern = ru_kernel<OpHi, OpLo>;
    int st = ensure_part(c, kern, smem, blocks);
    if (st) return st;
    a.gs = make_gs(c, *blocks);
    a.B = make_bufs(c);
    return launch_coop(kern, *blocks, smem, s, hi, lo, a);
}

// Patch-preconditioned PCG (ppcg_kernel): mode 1 = exact blocks where set and
// the network elsewhere, mode 2 = exact blocks where set and Jacobi elsewhere.
template <class Op>
static int run_fcg(cutcell_ctx* c, const Op& op, size_t op_smem, SolveArgs& a, cudaStream_t s, int* blocks,
                   int mode) {
    const size_t op_al = (op_smem + 15) & ~(size_t)15;
    // the network's weights and per-warp scratch only for the learned form
    // (mode 1); the block form needs the operator's shared memory alone
    const size_t smem =
        op_al + (mode == 1 ? MlpSmem::bytes() + (size_t)CUTCELL_WARPS * (MLP_IN + 3 * 64) * sizeof(float) : 0);
    LearnedArgs L;
    memset(&L, 0, sizeof(L));
    if (mode == 1) L.W = c->mlp->weights();
    L.pm = c->pmap;
    L.z = c->zl;
    L.rold = c->rold;
    L.use_mlp = mode;
    L.ones = c->ones;
    int st;
    if (mode == 1) {
        auto kern = ppcg_kernel<Op, true>;
        st = ensure_part(c, kern, smem, blocks);
        if (st) return st;
        a.gs = make_gs(c, *blocks);
        a.B = make_bufs(c);
        return launch_coop(kern, *blocks, smem, s, op, a, L, op_al);
    }
    auto kern = ppcg_kernel<Op, false>;
    st = ensure_part(c, kern, smem, blocks);
    if (st) return st;
    a.gs = make_gs(c, *blocks);
    a.B = make_bufs(c);
    return launch_coop(kern, *blocks, smem, s, op, a, L, op_al);
}

// Two-level patch PCG: shared memory of the operator, or the staged coarse
// vector and the per-warp x-lines if larger.
template <class Op>
static int run_tl(cutcell_ctx* c, const Op& op, size_t op_smem, SolveArgs& a, cudaStream_t s, int* blocks) {
    size_t smem = op_smem;
    const size_t need = std::max((size_t)c->coarse.ncg, (size_t)CUTCELL_WARPS * c->coarse.nb) * sizeof(double);
    if (need > smem) smem = need;
    smem = (smem + 15) & ~(size_t)15;
    LearnedArgs L;
    memset(&L, 0, sizeof(L));
    L.pm = c->pmap;
    L.z = c->zl;
    L.rold = c->rold;
    L.ones = c->ones;
    auto kern = tlpcg_kernel<Op>;
    int st = ensure_part(c, kern, smem, blocks);
    if (st) return st;
    a.gs = make_gs(c, *blocks);
    a.B = make_bufs(c);
    return launch_coop(kern, *blocks, smem, s, op, a, L, c->coarse);
}

template <class Op>
static int run_apply(cutcell_ctx* c, const Op& op, size_t smem, const double* x, double* y, cudaStream_t s) {
    auto kern = apply_kernel<Op>;
    int blocks = 0;
    int st = ensure_part(c, kern, smem, &blocks);
    if (st) return st;
    CK(cudaMemsetAsync(c->bar, 0, BAR_WORDS * sizeof(unsigned), s));
    GridSync gs = make_gs(c, blocks);
    return launch_coop(kern, blocks, smem, s, op, x, y, gs);
}

// mode 0: solve (plain or refinement), mode 1: one apply
// Reduced-precision refinement is built for p >= 3 only: an earlier fused
// refinement kernel instantiated for p = 2 faulted (misaligned address) on
// the B200 while the same code with self-checks compiled in ran clean, and
// reading the p = 2 paths did not show the cause; until it is found the
// p = 2 reduced-precision instantiations are not built.
template <int P1>
static int tiles_run(cutcell_ctx* c, int mode, int precision, SolveArgs* a, const double* x, double* y, cudaStream_t s,
                     int* blocks) {
    TileOp<double, P1> o64{c->td, c->cut64};
    TileOp<float, P1> o32{c->td, c->cut32};
    TileOp<bf16x2_t, P1> o16{c->td, c->cut16};
    const size_t sm = TileOp<double, P1>::smem_bytes();
    if (mode == 2) return run_fcg(c, o64, sm, *a, s, blocks, 1);
    if (mode == 3) return run_fcg(c, o64, sm, *a, s, blocks, 2);
    if (mode == 4) return run_tl(c, o64, sm, *a, s, blocks);
    if (mode == 1) {
        if (precision == CUTCELL_FP64) return run_apply(c, o64, sm, x, y, s);
        if (precision == CUTCELL_FP32_IR) return run_apply(c, o32, sm, x, y, s);
        return run_apply(c, o16, sm, x, y, s);
    }
    if (precision == CUTCELL_FP64) return run_plain(c, o64, sm, *a, s, blocks);
    if constexpr (P1 >= 4) {
        if (precision == CUTCELL_FP32_IR) return run_ru(c, o64, o32, sm, *a, s, blocks);
        return run_ru(c, o64, o16, sm, *a, s, blocks);
    } else {
        g_last_error = "reduced-precision refinement needs degree >= 3";
        return CUTCELL_E_ARG;
    }
}

static int tiles_dispatch(cutcell_ctx* c, int mode, int precision, SolveArgs* a, const double* x, double* y,
                          cudaStream_t s, int* blocks) {
    switch (c->td.p) {
        case 1: return tiles_run<2>(c, mode, precision, a, x, y, s, blocks);
        case 2: return tiles_run<3>(c, mode, precision, a, x, y, s, blocks);
        case 3: return tiles_run<4>(c, mode, precision, a, x, y, s, blocks);
        case 4: return tiles_run<5>(c, mode, precision, a, x, y, s, blocks);
        case 5: return tiles_run<6>(c, mode, precision, a, x, y, s, blocks);
        default: return CUTCELL_E_SHAPE;
    }
}

extern "C" {

const char* cutcell_status_string(int status) {
    switch (status) {
        case CUTCELL_OK: return "converged";
        case CUTCELL_E_NOCONV: return "maximum iterations reached";
        case CUTCELL_E_BREAKDOWN: return "CG breakdown: non-positive curvature";
        case CUTCELL_E_NAN: return "non-finite residual";
        case CUTCELL_E_SHAPE: return "inconsistent sizes";
        case CUTCELL_E_CUDA: return "CUDA runtime error";
        case CUTCELL_E_BARRIER: return "device-wide wait timed out";
        case CUTCELL_E_ARG: return "invalid argument";
        default: return "unknown status";
    }
}

const char* cutcell_last_error(void) { return g_last_error.c_str(); }
}

// Library-internal (C++ linkage, not exported in the header): lets the other
// translation units report through cutcell_last_error.
void cutcell_internal_set_error(const std::string& what) { g_last_error = what; }

// Bounded-wait limit shared by every persistent launch of the library: 0 means
// "not set yet" (the first read takes CUTCELL_WAIT_LIMIT_S or the default).
static std::atomic<unsigned long long> g_wait_limit_ns{0};

unsigned long long cutcell_internal_wait_limit_ns() {
    unsigned long long v = g_wait_limit_ns.load();
    if (v == 0) {
        double s = CUTCELL_DEFAULT_WAIT_LIMIT_S;
        if (const char* e = std::getenv("CUTCELL_WAIT_LIMIT_S")) {
            const double t = std::atof(e);
            if (t > 0.0 && t <= 3600.0) s = t;
        }
        unsigned long long expect = 0;
        g_wait_limit_ns.compare_exchange_strong(expect, (unsigned long long)(s * 1e9));
        v = g_wait_limit_ns.load();
    }
    return v;
}

extern "C" {

int cutcell_set_wait_limit(double seconds) {
    if (!(seconds >= 1e-3 && seconds <= 3600.0)) return CUTCELL_E_ARG;
    g_wait_limit_ns.store((unsigned long long)(seconds * 1e9));
    return CUTCELL_OK;
}

double cutcell_get_wait_limit(void) { return (double)cutcell_internal_wait_limit_ns() * 1e-9; }

int cutcell_barrier_selftest(int32_t blocks, int32_t arrivals, int32_t* status_out) {
    if (!status_out || blocks < 1 || arrivals < 1) return CUTCELL_E_ARG;
    int dev = 0, sms = 0, per = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, barrier_probe_kernel, CUTCELL_BLOCK, 0));
    if (blocks > sms * per) return CUTCELL_E_ARG;  // the grid must be co-resident
    unsigned* bar = nullptr;
    CK(cudaMalloc(&bar, BAR_WORDS * sizeof(unsigned)));
    int st = CUTCELL_OK;
    int err = 0;
    GridSync gs;
    gs.count = bar;
    gs.limit_ns = cutcell_internal_wait_limit_ns();
    gs.err = (int*)(bar + 32);
    gs.nblocks = (unsigned)arrivals;
    void* args[] = {(void*)&gs};
    cudaError_t e = cudaMemset(bar, 0, BAR_WORDS * sizeof(unsigned));
    if (e == cudaSuccess)
        e = cudaLaunchCooperativeKernel((const void*)barrier_probe_kernel, dim3(blocks), dim3(CUTCELL_BLOCK), args, 0,
                                        (cudaStream_t)0);
    if (e == cudaSuccess) e = cudaMemcpy(&err, bar + 32, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) st = cuda_fail(e, "barrier self-test");
    cudaFree(bar);
    if (st == CUTCELL_OK) *status_out = err == 0 ? CUTCELL_OK : err;
    return st;
}

}  // extern "C"

// Validates a device CSR (sizes n, nnz) with csr_check_kernel; CUTCELL_E_SHAPE
// if malformed.  `flag` is one device int of scratch.
static int validate_csr(int n, int nnz, const int* ptr, const int* idx, int* flag) {
    CK(cudaMemset(flag, 0, sizeof(int)));
    const int blocks = std::min(ceil_div(std::max(n, nnz), 256), 1184);
    csr_check_kernel<<<std::max(blocks, 1), 256>>>(n, nnz, ptr, idx, flag);
    CK(cudaGetLastError());
    int bad = 0;
    CK(cudaMemcpy(&bad, flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (bad) {
        g_last_error = "malformed CSR: row offsets must rise from 0 to nnz and columns lie in [0, n)";
        return CUTCELL_E_SHAPE;
    }
    return CUTCELL_OK;
}

extern "C" {

int cutcell_pcg_create_csr(int32_t n, int32_t nnz, const int32_t* indptr, const int32_t* indices, const double* data,
                           cutcell_ctx** out) {
    if (!out || n <= 0 || nnz < 0 || !indptr || (nnz > 0 && (!indices || !data))) return CUTCELL_E_ARG;
    cutcell_ctx* c = new cutcell_ctx();
    c->kind = KIND_CSR;
    c->n = n;
    CK(cudaGetDevice(&c->device));
    int st = alloc_scratch(c);
    if (!st) st = validate_csr(n, nnz, indptr, indices, reinterpret_cast<int*>(c->bar));
    if (st) {
        cutcell_destroy(c);
        return st;
    }
    // threads per row from the mean row length (power of two in [1, 32])
    const double mean = nnz / (double)n;
    int l2 = 0;
    while ((1 << l2) < 32 && (1 << l2) * 2 <= mean) ++l2;
    c->csr64 = CsrOp<double>{n, l2, indptr, indices, data};
    if (nnz > 0) {
        CK(cudaMalloc(&c->val32, (size_t)nnz * sizeof(float)));
        CK(cudaMalloc(&c->val16, (size_t)nnz * sizeof(bf16x2_t)));
        to_f32_kernel<<<592, 256>>>((size_t)nnz, data, c->val32);
        to_bf16x2_kernel<<<592, 256>>>((size_t)nnz, data, c->val16);
    }
    c->csr32 = CsrOp<float>{n, l2, indptr, indices, c->val32};
    c->csr16 = CsrOp<bf16x2_t>{n, l2, indptr, indices, c->val16};
    csr_diag_inv_kernel<<<ceil_div(n, 256), 256>>>(n, indptr, indices, data, c->dinv);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    *out = c;
    return CUTCELL_OK;
}

// Phase-2 work records, built once on the host from the descriptor's lists:
//   need_rec[k] = {full DOF i, row j whose y_j is i's value alone (no E^T
//                  entries) or -1, first, end of i's cut partials in ycut}
//   row_rec[k]  = {reduced row j, full DOF of j, first, end of j's E^T entries}
// The records with a list come first, by list length in buckets of 4 entries,
// longest first; the records without one (plain tile-partial sums and
// identity rows, most of them) follow in index order, so neighbouring lanes
// read neighbouring partials.  Lists longer than kHeavyList entries go to
// groups of 4 lanes even where the rest runs one per thread.  Also validates
// every index the phase-2 loops follow.
constexpr int kHeavyList = 12;

static int build_phase2(cutcell_ctx* c, const CutcellTileDesc* t) {
    const int nneed = t->n_need, nred = t->n_red, nfull = (int)t->n_full;
    std::vector<int> need(nneed), slot(nfull), rof(nfull), fred(nred), tptr((size_t)nred + 1);
    CK(cudaMemcpy(need.data(), t->need, sizeof(int) * nneed, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(slot.data(), t->cut_dof_slot, sizeof(int) * nfull, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(rof.data(), t->red_of_full, sizeof(int) * nfull, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(fred.data(), t->full_of_red, sizeof(int) * nred, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(tptr.data(), t->smallT_ptr, sizeof(int) * (nred + 1), cudaMemcpyDeviceToHost));
    int nslots = 0;
    for (int s : slot) nslots = std::max(nslots, s + 1);
    std::vector<int> cptr((size_t)nslots + 1, 0);
    CK(cudaMemcpy(cptr.data(), t->cut_dof_ptr, sizeof(int) * (nslots + 1), cudaMemcpyDeviceToHost));
    // every cut partial index must lie in ycut ([n_cut][(p+1)^3])
    const int P1 = t->degree + 1;
    const long ncp = (long)t->n_cut * P1 * P1 * P1;
    const int nent = cptr[nslots];
    if (cptr[0] != 0 || nent < 0) return CUTCELL_E_SHAPE;
    for (int s = 0; s < nslots; ++s)
        if (cptr[s + 1] < cptr[s]) return CUTCELL_E_SHAPE;
    std::vector<int> ent((size_t)nent);
    if (nent) CK(cudaMemcpy(ent.data(), t->cut_dof_ent, sizeof(int) * nent, cudaMemcpyDeviceToHost));
    // the lists hold every (cut element, local row) exactly once: ycut is
    // stored in list order and each cut element writes row r to pos[c P + r]
    if ((long)nent != ncp) return CUTCELL_E_SHAPE;
    std::vector<int> pos((size_t)std::max<long>(ncp, 1), -1);
    for (int k = 0; k < nent; ++k) {
        const int e = ent[k];
        if (e < 0 || e >= ncp || pos[e] >= 0) return CUTCELL_E_SHAPE;
        pos[e] = k;
    }
    std::vector<int4> nr(nneed), rr(nred);
    std::vector<char> needed((size_t)nfull, 0);
    for (int k = 0; k < nneed; ++k) {
        const int i = need[k];
        if (i < 0 || i >= nfull || needed[i]) return CUTCELL_E_SHAPE;  // in range, listed once
        if (rof[i] < -1 || rof[i] >= nred) return CUTCELL_E_SHAPE;
        const int s = slot[i];
        nr[k] = s >= 0 ? make_int4(i, -1, cptr[s], cptr[s + 1]) : make_int4(i, -1, 0, 0);
        needed[i] = 1;
    }
    if (tptr[0] != 0) return CUTCELL_E_SHAPE;
    for (int j = 0; j < nred; ++j) {
        const int f = fred[j];
        if (f < 0 || f >= nfull || rof[f] != j || !needed[f] || tptr[j + 1] < tptr[j]) return CUTCELL_E_SHAPE;
        rr[j] = make_int4(j, f, tptr[j], tptr[j + 1]);
    }
    // the E^T lists may only read needed DOFs
    std::vector<int> trow((size_t)tptr[nred]);
    if (!trow.empty())
        CK(cudaMemcpy(trow.data(), t->smallT_row, sizeof(int) * trow.size(), cudaMemcpyDeviceToHost));
    for (int i : trow)  // only small (non-identity) DOFs are read by other rows
        if (i < 0 || i >= nfull || !needed[i] || rof[i] >= 0) return CUTCELL_E_SHAPE;
    // a row without E^T entries is y_j = yf of its own DOF: the gather of
    // that DOF writes y_j directly (need_rec.y = j), the scatter skips it
    for (int4& r : nr)
        if (rof[r.x] >= 0 && tptr[rof[r.x] + 1] == tptr[rof[r.x]]) r.y = rof[r.x];
    auto order = [](std::vector<int4>& v, int* heavy, int* listed) {
        auto key = [](const int4& a) { return a.w > a.z ? 1 + (a.w - a.z) / 4 : 0; };
        std::stable_sort(v.begin(), v.end(), [&](const int4& a, const int4& b) { return key(a) > key(b); });
        *heavy = 0;
        while (*heavy < (int)v.size() && v[*heavy].w - v[*heavy].z > kHeavyList) ++*heavy;
        *listed = *heavy;
        while (*listed < (int)v.size() && v[*listed].w > v[*listed].z) ++*listed;
    };
    order(nr, &c->td.n_need_heavy, &c->td.n_need_list);
    order(rr, &c->td.n_row_heavy, &c->td.n_row_list);
    CK(cudaMalloc(&c->cut_pos, sizeof(int) * pos.size()));
    CK(cudaMemcpy(c->cut_pos, pos.data(), sizeof(int) * pos.size(), cudaMemcpyHostToDevice));
    c->td.cut_pos = c->cut_pos;
    CK(cudaMalloc(&c->need_rec, sizeof(int4) * std::max(nneed, 1)));
    CK(cudaMalloc(&c->row_rec, sizeof(int4) * std::max(nred, 1)));
    if (nneed) CK(cudaMemcpy(c->need_rec, nr.data(), sizeof(int4) * nneed, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->row_rec, rr.data(), sizeof(int4) * nred, cudaMemcpyHostToDevice));
    c->td.need_rec = c->need_rec;
    c->td.row_rec = c->row_rec;
    return CUTCELL_OK;
}

int cutcell_pcg_create_tiles(const CutcellTileDesc* t, cutcell_ctx** out) {
    if (!out || !t) return CUTCELL_E_ARG;
    const int p = t->degree, P1 = p + 1, P = P1 * P1 * P1, D = t->tile + p;
    const int nb = t->n_elements + p;
    if (p < 1 || p > 5 || t->tile != 4 || t->n_tiles_axis * t->tile < t->n_elements ||
        (long)nb * nb * nb != t->n_full || t->n_red <= 0 || t->cut_chunk < 1 || t->n_mixed < 0 ||
        t->n_mixed > t->n_items)
        return CUTCELL_E_SHAPE;
    cutcell_ctx* c = new cutcell_ctx();
    c->kind = KIND_TILES;
    c->n = t->n_red;
    CK(cudaGetDevice(&c->device));
    int st = alloc_scratch(c);
    if (st) {
        delete c;
        return st;
    }
    // DOF-major tile partials: ceil(D / tile)^3 slots per DOF, absent tiles' slots stay zero
    const int NC = (D + t->tile - 1) / t->tile;
    const size_t nyp = (size_t)t->n_full * NC * NC * NC;
    CK(cudaMalloc(&c->ypart, nyp * sizeof(double)));
    CK(cudaMemset(c->ypart, 0, nyp * sizeof(double)));
    CK(cudaMalloc(&c->ycut, ((size_t)t->n_cut * P + 1) * sizeof(double)));
    CK(cudaMemset(c->ycut, 0, ((size_t)t->n_cut * P + 1) * sizeof(double)));
    CK(cudaMalloc(&c->yfv, (size_t)t->n_full * sizeof(double)));
    CK(cudaMalloc(&c->psmall, ((size_t)t->n_small + 1) * sizeof(double)));
    CK(cudaMemset(c->yfv, 0, (size_t)t->n_full * sizeof(double)));
    // degree 3 keeps its (symmetric) cut blocks in the split storage of
    // sym64_index, half the bytes of the dense blocks; other degrees read the
    // caller's dense blocks
    c->cut64 = t->cut_mats;
    size_t ncm = (size_t)t->n_cut * P * P;
    if (p == 3 && t->n_cut > 0) {
        ncm = (size_t)t->n_cut * SYM64_ENTRIES;
        CK(cudaMalloc(&c->cutsym, ncm * sizeof(double)));
        pack_sym64_kernel<<<592, 256>>>(t->n_cut, t->cut_mats, c->cutsym);
        c->cut64 = c->cutsym;
    }
    if (ncm) {
        CK(cudaMalloc(&c->cut32, ncm * sizeof(float)));
        CK(cudaMalloc(&c->cut16, ncm * sizeof(bf16x2_t)));
        to_f32_kernel<<<592, 256>>>(ncm, c->cut64, c->cut32);
        to_bf16x2_kernel<<<592, 256>>>(ncm, c->cut64, c->cut16);
    }
    ExtDev e;
    e.n_full = t->n_full;
    e.n_red = t->n_red;
    e.n_small = t->n_small;
    e.red_of_full = t->red_of_full;
    e.small_slot = t->small_slot;
    e.small_ptr = t->small_ptr;
    e.small_idx = t->small_idx;
    e.small_val = t->small_val;
    e.full_of_red = t->full_of_red;
    e.smallT_ptr = t->smallT_ptr;
    e.smallT_row = t->smallT_row;
    e.smallT_val = t->smallT_val;
    e.psmall = c->psmall;
    TileData& d = c->td;
    d.n = t->n_elements;
    d.p = p;
    d.T = t->tile;
    d.nta = t->n_tiles_axis;
    d.nb = nb;
    d.n_items = t->n_items;
    d.n_mixed = t->n_mixed;
    {
        // warp-level full tiles: always where their passes run on the FP64
        // tensor cores (window D <= 8), else once there are many per SM
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
        d.full_warp = (D <= 8 || (t->n_items - t->n_mixed) >= 8 * (sms > 0 ? sms : 148)) ? 1 : 0;
        // one thread per DOF once there are more than about two per thread of a 2 x 256 x SMs grid
        d.lane1 = t->n_need > 2 * 512 * (sms > 0 ? sms : 148) ? 1 : 0;
    }
    d.n_cut = t->n_cut;
    d.cut_chunk = t->cut_chunk;
    d.a_mass = t->a_mass;
    d.item_list = t->item_list;
    d.tile_kind = t->tile_kind;
    d.tile_eptr = t->tile_eptr;
    d.tile_elem = t->tile_elem;
    d.tile_ecut = t->tile_ecut;
    d.M1 = t->M1;
    d.Kt1 = t->Kt1;
    d.TM = t->TM;
    d.TA = t->TA;
    d.TK = t->TK;
    d.cut_base = t->cut_base;
    d.cut_dof_slot = t->cut_dof_slot;
    d.cut_dof_ptr = t->cut_dof_ptr;
    d.cut_dof_ent = t->cut_dof_ent;
    d.ext = e;
    d.ypart = c->ypart;
    d.ycut = c->ycut;
    d.yfv = c->yfv;
    d.need = t->need;
    d.n_need = t->n_need;
    d.work = c->bar + 64;
    d.work2 = c->bar + 96;
    st = build_phase2(c, t);
    if (st) {
        cutcell_destroy(c);
        return st;
    }
    diag_inv_kernel<<<ceil_div(t->n_red, 256), 256>>>(t->n_red, t->diag, c->dinv);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    *out = c;
    return CUTCELL_OK;
}

// KronOp of a form: which = CUTCELL_FORM_* (see the header).
static KronOp make_kron_op(cutcell_ctx* c, int which) {
    KronOp o;
    memset(&o, 0, sizeof(o));
    o.nx = c->kn[0];
    o.ny = c->kn[1];
    o.nz = c->kn[2];
    const size_t N = (size_t)o.nx * o.ny * o.nz;
    o.U1 = c->kscratch;
    o.U2 = c->kscratch + N;
    o.V1 = c->kscratch + 2 * N;
    o.V2 = c->kscratch + 3 * N;
    enum { H = 0, K = 1, Q = 2, S = 3, A = 4 };
    const KronBand(&b)[3][5] = c->kb;
    if (which == CUTCELL_FORM_A || which == CUTCELL_FORM_K) {
        const int f = which == CUTCELL_FORM_A ? A : K;
        o.X0 = b[0][H];
        o.X1 = b[0][f];
        o.Y0 = b[1][H];
        o.Y1 = b[1][H];
        o.Y2 = b[1][f];
        o.Z0 = b[2][H];
        o.Z1 = b[2][f];
        return o;
    }
    // single products: H, or Q / S on one axis and H on the others
    int f[3] = {H, H, H};
    if (which >= CUTCELL_FORM_QX && which <= CUTCELL_FORM_QZ) f[which - CUTCELL_FORM_QX] = Q;
    if (which >= CUTCELL_FORM_SX && which <= CUTCELL_FORM_SZ) f[which - CUTCELL_FORM_SX] = S;
    o.X0 = b[0][f[0]];
    o.Y0 = b[1][f[1]];
    o.Z1 = b[2][f[2]];
    return o;
}

int cutcell_kron_create(const CutcellKronDesc* d, cutcell_ctx** out) {
    if (!out || !d || !d->diag) return CUTCELL_E_ARG;
    for (int a = 0; a < 3; ++a) {
        if (d->n[a] < 1 || d->n[a] > 65536) return CUTCELL_E_SHAPE;
        for (int f = 0; f < 5; ++f)
            if (!d->factors[a][f]) return CUTCELL_E_ARG;
    }
    const long N = (long)d->n[0] * d->n[1] * d->n[2];
    if (N > (1L << 30)) return CUTCELL_E_SHAPE;
    cutcell_ctx* c = new cutcell_ctx();
    c->kind = KIND_KRON;
    c->n = (int)N;
    CK(cudaGetDevice(&c->device));
    int st = alloc_scratch(c);
    if (st) {
        cutcell_destroy(c);
        return st;
    }
    // band form of every factor: row i's nonzeros in [lo_i, lo_i + W), the
    // band start moved left where it would run past the last column
    std::vector<int> lo_all;
    std::vector<double> band_all;
    size_t lo_off[3][5], band_off[3][5];
    for (int a = 0; a < 3; ++a) {
        const int n = d->n[a];
        std::vector<double> M((size_t)n * n);
        for (int f = 0; f < 5; ++f) {
            CK(cudaMemcpy(M.data(), d->factors[a][f], M.size() * sizeof(double), cudaMemcpyDeviceToHost));
            std::vector<int> lo(n), hi(n);
            int W = 1;
            for (int i = 0; i < n; ++i) {
                int l = -1, h = -1;
                for (int j = 0; j < n; ++j)
                    if (M[(size_t)i * n + j] != 0.0) {
                        if (l < 0) l = j;
                        h = j;
                    }
                if (l < 0) l = h = i;
                lo[i] = l;
                hi[i] = h;
                W = std::max(W, h - l + 1);
            }
            lo_off[a][f] = lo_all.size();
            band_off[a][f] = band_all.size();
            for (int i = 0; i < n; ++i) {
                const int l = std::min(lo[i], n - W);
                lo_all.push_back(l);
                for (int w = 0; w < W; ++w) band_all.push_back(M[(size_t)i * n + l + w]);
            }
            c->kb[a][f].W = W;
        }
        c->kn[a] = n;
    }
    CK(cudaMalloc(&c->klo, lo_all.size() * sizeof(int)));
    CK(cudaMalloc(&c->kband, band_all.size() * sizeof(double)));
    CK(cudaMemcpy(c->klo, lo_all.data(), lo_all.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->kband, band_all.data(), band_all.size() * sizeof(double), cudaMemcpyHostToDevice));
    for (int a = 0; a < 3; ++a)
        for (int f = 0; f < 5; ++f) {
            c->kb[a][f].lo = c->klo + lo_off[a][f];
            c->kb[a][f].band = c->kband + band_off[a][f];
        }
    CK(cudaMalloc(&c->kscratch, (size_t)4 * N * sizeof(double)));
    diag_inv_kernel<<<ceil_div(N, 256), 256>>>((int)N, d->diag, c->dinv);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    *out = c;
    return CUTCELL_OK;
}

int cutcell_apply_form(cutcell_ctx* c, const double* x, double* y, int32_t which, void* stream) {
    if (!c || !x || !y || which < CUTCELL_FORM_A || which > CUTCELL_FORM_SZ) return CUTCELL_E_ARG;
    if (c->kind == KIND_KRON) return run_apply(c, make_kron_op(c, which), 0, x, y, (cudaStream_t)stream);
    if (which != CUTCELL_FORM_A) {
        g_last_error = "this context holds only its SPD system form (CUTCELL_FORM_A)";
        return CUTCELL_E_ARG;
    }
    return cutcell_apply(c, x, y, CUTCELL_FP64, stream);
}

int cutcell_dgemm_nt(int32_t M, int32_t N, int32_t K, const double* A, int64_t lda, int64_t strideA, const double* B,
                     int64_t ldb, int64_t strideB, const double* s, int64_t strideS, double beta, double* C, int64_t ldc,
                     int64_t strideC, int32_t batch, void* stream) {
    if (M < 0 || N < 0 || K < 0 || batch < 0 || !A || !B || !C || lda < K || ldb < K || ldc < N) return CUTCELL_E_ARG;
    if (M == 0 || N == 0 || batch == 0) return CUTCELL_OK;
    if (batch > 65535 || ceil_div(M, DG_BM) > 65535) return CUTCELL_E_SHAPE;
    DgemmArgs g{M, N, K, A, lda, strideA, B, ldb, strideB, s, strideS, beta, C, ldc, strideC};
    dim3 grid(ceil_div(N, DG_BN), ceil_div(M, DG_BM), batch);
    dgemm_nt_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(g);
    CK(cudaGetLastError());
    return CUTCELL_OK;
}

int cutcell_set_refinement(cutcell_ctx* c, double replace_factor, int32_t reserved, int32_t max_replacements) {
    if (!c || !(replace_factor > 0.0 && replace_factor < 1.0) || max_replacements < 1) return CUTCELL_E_ARG;
    (void)reserved;
    c->inner_tol = replace_factor;
    c->max_outer = max_replacements;
    return CUTCELL_OK;
}

int cutcell_pcg_solve(cutcell_ctx* c, const double* b, double* x, double tol, int32_t maxiter, int32_t precision,
                      int32_t precond, CutcellReport* report, void* stream) {
    if (!c || !b || !x || maxiter < 0 || !(tol >= 0.0)) return CUTCELL_E_ARG;
    if (precision < CUTCELL_FP64 || precision > CUTCELL_BF16_IR) return CUTCELL_E_ARG;
    if (precond < CUTCELL_PRECOND_NONE || precond > CUTCELL_PRECOND_TWOLEVEL) return CUTCELL_E_ARG;
    if (precond == CUTCELL_PRECOND_JACOBI_LEARNED && (!c->mlp || precision != CUTCELL_FP64 || c->kind != KIND_TILES))
        return CUTCELL_E_ARG;
    if (precond == CUTCELL_PRECOND_BLOCK &&
        (!c->pmap.binv || !c->pmap.slot || !c->zl || precision != CUTCELL_FP64 || c->kind != KIND_TILES)) {
        g_last_error = "CUTCELL_PRECOND_BLOCK needs patch blocks (cutcell_pcg_set_patch_blocks), FP64, a tile context";
        return CUTCELL_E_ARG;
    }
    if (precond == CUTCELL_PRECOND_TWOLEVEL &&
        (!c->has_coarse || !c->pmap.red || !c->zl || precision != CUTCELL_FP64 || c->kind != KIND_TILES)) {
        g_last_error = "CUTCELL_PRECOND_TWOLEVEL needs a coarse level (cutcell_pcg_set_coarse), a patch layout "
                       "(cutcell_pcg_set_patch_blocks), FP64, a tile context";
        return CUTCELL_E_ARG;
    }
    if (c->kind == KIND_KRON && precision != CUTCELL_FP64) {
        g_last_error = "the Kronecker cut-box operator is solved in FP64";
        return CUTCELL_E_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    CK(cudaSetDevice(c->device));
    c->use_jacobi = (precond != CUTCELL_PRECOND_NONE);
    SolveArgs a;
    memset(&a, 0, sizeof(a));
    a.b = b;
    a.x = x;
    a.tol = tol;
    a.maxiter = maxiter;
    a.inner_tol = c->inner_tol;
    a.inner_maxiter = c->inner_maxiter;
    a.max_outer = c->max_outer;
    a.d = c->d;
    a.rhat = c->rhat;
    a.res = c->res;
    CK(cudaMemsetAsync(c->bar, 0, BAR_WORDS * sizeof(unsigned), s));
    CK(cudaEventRecord(c->ev0, s));
    int blocks = 0;
    int st = CUTCELL_OK;
    if (c->kind == KIND_KRON) {
        st = run_plain(c, make_kron_op(c, CUTCELL_FORM_A), 0, a, s, &blocks);
    } else if (c->kind == KIND_CSR) {
        if (precision == CUTCELL_FP64)
            st = run_plain(c, c->csr64, 0, a, s, &blocks);
        else if (precision == CUTCELL_FP32_IR)
            st = run_ru(c, c->csr64, c->csr32, 0, a, s, &blocks);
        else
            st = run_ru(c, c->csr64, c->csr16, 0, a, s, &blocks);
    } else if (precond == CUTCELL_PRECOND_JACOBI_LEARNED) {
        st = tiles_dispatch(c, 2, precision, &a, nullptr, nullptr, s, &blocks);
    } else if (precond == CUTCELL_PRECOND_BLOCK) {
        st = tiles_dispatch(c, 3, precision, &a, nullptr, nullptr, s, &blocks);
    } else if (precond == CUTCELL_PRECOND_TWOLEVEL) {
        st = tiles_dispatch(c, 4, precision, &a, nullptr, nullptr, s, &blocks);
    } else {
        st = tiles_dispatch(c, 0, precision, &a, nullptr, nullptr, s, &blocks);
    }
    if (st) return st;
    CK(cudaEventRecord(c->ev1, s));
#ifdef CUTCELL_DEBUG_CHECKS
    {
        unsigned w[BAR_WORDS];
        CK(cudaMemcpyAsync(w, c->bar, sizeof(w), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (w[128]) fprintf(stderr, "cutcell debug check failed: code %u info %u\n", w[128], w[129]);
    }
#endif
    DevResult hr;
    CK(cudaMemcpyAsync(&hr, c->res, sizeof(hr), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    if (report) {
        report->status = hr.status;
        report->iterations = hr.iterations;
        report->outer_iterations = hr.outer;
        report->blocks = blocks;
        report->relative_residual = hr.rel;
        report->true_relative_residual = hr.true_rel;
        report->elapsed_ms = ms;
    }
    return hr.status == CUTCELL_E_BARRIER ? CUTCELL_E_BARRIER : CUTCELL_OK;
}

int cutcell_apply(cutcell_ctx* c, const double* x, double* y, int32_t precision, void* stream) {
    if (!c || !x || !y) return CUTCELL_E_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    if (c->kind == KIND_KRON)
        return precision == CUTCELL_FP64 ? run_apply(c, make_kron_op(c, CUTCELL_FORM_A), 0, x, y, s) : CUTCELL_E_ARG;
    if (c->kind == KIND_CSR) {
        if (precision == CUTCELL_FP64) return run_apply(c, c->csr64, 0, x, y, s);
        if (precision == CUTCELL_FP32_IR) return run_apply(c, c->csr32, 0, x, y, s);
        if (precision == CUTCELL_BF16_IR) return run_apply(c, c->csr16, 0, x, y, s);
    } else if (precision >= CUTCELL_FP64 && precision <= CUTCELL_BF16_IR) {
        int blocks = 0;
        return tiles_dispatch(c, 1, precision, nullptr, x, y, s, &blocks);
    }
    return CUTCELL_E_ARG;
}

int cutcell_ext_gather(cutcell_ctx* c, const double* x_red, double* x_full, void* stream) {
    if (!c || c->kind != KIND_TILES || !x_red || !x_full) return CUTCELL_E_ARG;
    ext_gather_kernel<<<ceil_div(c->td.ext.n_full, 256), 256, 0, (cudaStream_t)stream>>>(c->td.ext, x_red, x_full);
    CK(cudaGetLastError());
    return CUTCELL_OK;
}

int cutcell_ext_scatter(cutcell_ctx* c, const double* y_full, double* y_red, void* stream) {
    if (!c || c->kind != KIND_TILES || !y_full || !y_red) return CUTCELL_E_ARG;
    ext_scatter_kernel<<<ceil_div(c->td.ext.n_red, 256), 256, 0, (cudaStream_t)stream>>>(c->td.ext, y_full, y_red);
    CK(cudaGetLastError());
    return CUTCELL_OK;
}

int cutcell_destroy(cutcell_ctx* c) {
    if (!c) return CUTCELL_E_ARG;
    cudaSetDevice(c->device);  // cudaFree below waits for the work that may still use the buffers
    void* bufs[] = {c->cwork, c->czx[0], c->czx[1], c->czx[2], c->pslot_all, c->klo, c->kband, c->kscratch, c->val32, c->val16, c->cutsym, c->cut32, c->cut16, c->need_rec, c->row_rec, c->cut_pos, c->ypart, c->ycut, c->yfv, c->psmall, c->zl, c->rold, c->dinv, c->ones, c->r,
                    c->p,     c->p2,    c->Ap,    c->d,     c->rhat,  c->part,  c->bar,  c->res};
    for (void* b : bufs)
        if (b) cudaFree(b);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    delete c;
    return CUTCELL_OK;
}

int cutcell_mlp_create(const float* theta_init, int32_t activation, cutcell_mlp** out) {
    if (!theta_init || !out || activation < 0 || activation > 1) return CUTCELL_E_ARG;
    cutcell_mlp* m = new cutcell_mlp();
    m->act = activation;
    CK(cudaGetDevice(&m->device));
    CK(cudaMalloc(&m->theta, MLP_NPARAM * sizeof(float)));
    CK(cudaMalloc(&m->m, MLP_NPARAM * sizeof(float)));
    CK(cudaMalloc(&m->v, MLP_NPARAM * sizeof(float)));
    CK(cudaMalloc(&m->grad, MLP_NPARAM * sizeof(float)));
    CK(cudaMalloc(&m->wbf, MLP_NW * sizeof(__nv_bfloat16)));
    CK(cudaMemcpy(m->theta, theta_init, MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToDevice));
    CK(cudaMemset(m->m, 0, MLP_NPARAM * sizeof(float)));
    CK(cudaMemset(m->v, 0, MLP_NPARAM * sizeof(float)));
    mlp_refresh_bf16_kernel<<<ceil_div(MLP_NPARAM, 256), 256>>>(m->theta, m->wbf);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    *out = m;
    return CUTCELL_OK;
}

int cutcell_mlp_params(cutcell_mlp* m, float* theta_out, float* grad_out) {
    if (!m) return CUTCELL_E_ARG;
    if (theta_out) CK(cudaMemcpy(theta_out, m->theta, MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToDevice));
    if (grad_out) CK(cudaMemcpy(grad_out, m->grad, MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToDevice));
    return CUTCELL_OK;
}

int cutcell_mlp_forward(cutcell_mlp* m, const float* X, int32_t batch, float* Y, void* stream) {
    if (!m || !X || !Y || batch < 0) return CUTCELL_E_ARG;
    if (batch == 0) return CUTCELL_OK;
    const size_t smem = MlpTcSmem::bytes();
    CK(cudaFuncSetAttribute(mlp_forward_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int tiles = ceil_div(batch, 16);
    const int nblk = std::min(ceil_div(tiles, MLPT_WARPS), 2 * 148);
    mlp_forward_tc_kernel<<<nblk, MLPT_WARPS * 32, smem, (cudaStream_t)stream>>>(m->weights(), X, batch, Y);
    CK(cudaGetLastError());
    return CUTCELL_OK;
}

int cutcell_mlp_train_step(cutcell_mlp* m, const float* X, const float* T, int32_t batch, float lr, float* loss_out,
                           void* stream) {
    if (!m || !X || !T || batch <= 0) return CUTCELL_E_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    if (batch > m->cap) {
        float** bufs[] = {&m->H1, &m->H2, &m->D1, &m->D2, &m->DY, &m->Y};
        for (float** b : bufs) {
            if (*b) cudaFree(*b);
            CK(cudaMalloc(b, (size_t)batch * 64 * sizeof(float)));
        }
        if (m->L) cudaFree(m->L);
        CK(cudaMalloc(&m->L, (size_t)batch * sizeof(float)));
        m->cap = batch;
    }
    const size_t smem = MlpTcSmem::bytes();
    CK(cudaFuncSetAttribute(mlp_fwd_bwd_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int nblk = std::min(ceil_div(ceil_div(batch, 16), MLPT_WARPS), 2 * 148);
    mlp_fwd_bwd_tc_kernel<<<nblk, MLPT_WARPS * 32, smem, s>>>(m->weights(), X, T, batch, m->H1, m->H2, m->D1, m->D2,
                                                             m->DY, m->Y, m->L);
    mlp_wgrad_tc_kernel<<<4, 128, 0, s>>>(X, m->H1, m->H2, m->D1, m->D2, m->DY, batch, m->grad);
    mlp_bgrad_kernel<<<1, 192, 0, s>>>(m->D1, m->D2, m->DY, batch, m->grad);
    if (loss_out) sum_in_order_kernel<<<1, CUTCELL_BLOCK, 0, s>>>(m->L, batch, 1.0f / (float)((long)batch * 64), loss_out);
    if (lr > 0.f) {
        m->step += 1;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - powf(b1, (float)m->step), c2 = 1.f - powf(b2, (float)m->step);
        mlp_adam_kernel<<<ceil_div(MLP_NPARAM, 256), 256, 0, s>>>(m->theta, m->m, m->v, m->grad, m->wbf, lr, b1, b2,
                                                                  1e-8f, c1, c2);
    }
    CK(cudaGetLastError());
    return CUTCELL_OK;
}

int cutcell_mlp_destroy(cutcell_mlp* m) {
    if (!m) return CUTCELL_E_ARG;
    cudaSetDevice(m->device);  // cudaFree below waits for the work that may still use the buffers
    void* bufs[] = {m->theta, m->m, m->v, m->grad, m->wbf, m->H1, m->H2, m->D1, m->D2, m->DY, m->Y, m->L};
    for (void* b : bufs)
        if (b) cudaFree(b);
    delete m;
    return CUTCELL_OK;
}

int cutcell_patch_features(cutcell_ctx* c, const int32_t* patch_red, const float* patch_gamma, int32_t n_patch,
                           const double* r, float* X, float* S, void* stream) {
    if (!c || !patch_red || !patch_gamma || !r || !X || !S || n_patch < 0) return CUTCELL_E_ARG;
    if (n_patch == 0) return CUTCELL_OK;
    PatchMap pm{n_patch, patch_red, patch_gamma, nullptr, nullptr};
    patch_features_kernel<<<ceil_div(n_patch, CUTCELL_WARPS), CUTCELL_BLOCK, 0, (cudaStream_t)stream>>>(pm, r, c->dinv,
                                                                                                      X, S);
    CK(cudaGetLastError());
    return CUTCELL_OK;
}

int cutcell_patch_targets(cutcell_ctx* c, const int32_t* patch_red, int32_t n_patch, const double* e,
                          const double* r, const float* S, float* T, void* stream) {
    if (!c || !patch_red || !e || !r || !S || !T || n_patch < 0) return CUTCELL_E_ARG;
    if (n_patch == 0) return CUTCELL_OK;
    PatchMap pm{n_patch, patch_red, nullptr, nullptr, nullptr};
    patch_targets_kernel<<<ceil_div((long)n_patch * 64, 256), 256, 0, (cudaStream_t)stream>>>(pm, e, r, c->dinv, S, T);
    CK(cudaGetLastError());
    return CUTCELL_OK;
}

int cutcell_pcg_set_block_inverses(cutcell_ctx* c, const double* binv) {
    if (!c || c->kind != KIND_TILES || c->pmap.n_patch <= 0) return CUTCELL_E_ARG;
    if (!binv) {
        c->pmap.binv = nullptr;
        c->pmap.slot = nullptr;
        return CUTCELL_OK;
    }
    if (!c->pslot_all) {
        std::vector<int> id(c->pmap.n_patch);
        for (int k = 0; k < c->pmap.n_patch; ++k) id[k] = k;
        CK(cudaMalloc(&c->pslot_all, id.size() * sizeof(int)));
        CK(cudaMemcpy(c->pslot_all, id.data(), id.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    c->pmap.binv = binv;
    c->pmap.slot = c->pslot_all;
    return CUTCELL_OK;
}

int cutcell_pcg_set_patch_blocks(cutcell_ctx* c, const int32_t* patch_red, int32_t n_patch, const int32_t* slot,
                                 const double* binv) {
    if (!c || c->kind != KIND_TILES) return CUTCELL_E_ARG;
    if (!binv) {
        c->pmap.binv = nullptr;
        c->pmap.slot = nullptr;
        return CUTCELL_OK;
    }
    if (!patch_red || !slot || n_patch <= 0) return CUTCELL_E_ARG;
    if (c->mlp && (c->pmap.red != patch_red || c->pmap.n_patch != n_patch)) {
        g_last_error = "patch blocks must use the layout of the attached network";
        return CUTCELL_E_ARG;
    }
    if (!c->mlp) {
        c->pmap.red = patch_red;
        c->pmap.n_patch = n_patch;
        c->pmap.gamma = nullptr;
    }
    c->pmap.binv = binv;
    c->pmap.slot = slot;
    if (!c->zl) {
        CK(cudaMalloc(&c->zl, (size_t)c->n * sizeof(double)));
        CK(cudaMalloc(&c->rold, (size_t)c->n * sizeof(double)));
    }
    return CUTCELL_OK;
}

int cutcell_pcg_set_coarse(cutcell_ctx* c, const CutcellCoarseDesc* d) {
    if (!c || c->kind != KIND_TILES) return CUTCELL_E_ARG;
    if (!d) {
        c->has_coarse = false;
        return CUTCELL_OK;
    }
    const int nb = c->td.n + c->td.p;
    if (d->nb != nb || d->nbc < 1 || d->nbc > nb || d->pw != c->td.p + 1 || d->pw > d->nbc || d->rw < 1 || d->rw > nb ||
        !d->plo || !d->pval || !d->rlo || !d->rval || !d->minv) {
        g_last_error = "coarse level: fine DOFs per axis must be n + p, prolongation bands p + 1 wide, restriction "
                       "bands within the grid, all tables set";
        return CUTCELL_E_ARG;
    }
    const long long ncg = (long long)d->nbc * d->nbc * d->nbc;
    if (ncg > 16384) {
        g_last_error = "coarse level: at most 16384 coarse DOFs (the dense inverse is read every iteration)";
        return CUTCELL_E_SHAPE;
    }
    if (c->cwork) cudaFree(c->cwork);
    c->cwork = nullptr;
    const size_t nt1 = (size_t)nb * nb * d->nbc;
    CK(cudaMalloc(&c->cwork, (nt1 + 2 * (size_t)ncg + 2 * (size_t)c->n) * sizeof(double)));
    CoarseDev& cd = c->coarse;
    cd.nb = nb;
    cd.nbc = d->nbc;
    cd.ncg = (int)ncg;
    cd.pw = d->pw;
    cd.rw = d->rw;
    cd.plo = d->plo;
    cd.pval = d->pval;
    cd.rlo = d->rlo;
    cd.rval = d->rval;
    cd.minv = d->minv;
    cd.t1 = c->cwork;
    cd.rc = cd.t1 + nt1;
    cd.yc = cd.rc + ncg;
    cd.zc = cd.yc + ncg;
    cd.azc = cd.zc + c->n;
    if (!c->zl) {
        CK(cudaMalloc(&c->zl, (size_t)c->n * sizeof(double)));
        CK(cudaMalloc(&c->rold, (size_t)c->n * sizeof(double)));
    }
    c->has_coarse = true;
    return CUTCELL_OK;
}

int cutcell_pcg_set_twolevel_blocks(cutcell_ctx* c, const uint16_t* binv0, int32_t n_extra,
                                    const int32_t* const* patch_red, const int32_t* n_patch,
                                    const uint16_t* const* binv, double omega) {
    if (!c || c->kind != KIND_TILES) return CUTCELL_E_ARG;
    CoarseDev& cd = c->coarse;
    if (n_extra < 0 || n_extra > ZSUM_MAX || (n_extra > 0 && (!patch_red || !n_patch || !binv)) ||
        (n_extra > 0 && !(omega > 0.0 && omega <= 1.0))) {
        g_last_error = "two-level blocks: at most 3 extra tilings, each with a layout and inverses; weight in (0, 1]";
        return CUTCELL_E_ARG;
    }
    for (int i = 0; i < n_extra; ++i)
        if (!patch_red[i] || !binv[i] || n_patch[i] <= 0) {
            g_last_error = "two-level blocks: an extra tiling without layout or inverses";
            return CUTCELL_E_ARG;
        }
    for (int i = 0; i < n_extra; ++i)
        if (!c->czx[i]) CK(cudaMalloc(&c->czx[i], (size_t)c->n * sizeof(double)));
    cd.binv0h = reinterpret_cast<const __nv_bfloat16*>(binv0);
    cd.n_extra = n_extra;
    for (int i = 0; i < ZSUM_MAX; ++i) {
        const bool on = i < n_extra;
        cd.n_patch_x[i] = on ? n_patch[i] : 0;
        cd.red_x[i] = on ? patch_red[i] : nullptr;
        cd.binv_x[i] = on ? reinterpret_cast<const __nv_bfloat16*>(binv[i]) : nullptr;
        cd.zx[i] = c->czx[i];
    }
    cd.omega = n_extra > 0 ? omega : 1.0;
    return CUTCELL_OK;
}

int cutcell_pcg_set_learned(cutcell_ctx* c, cutcell_mlp* m, const int32_t* patch_red, const float* patch_gamma,
                            int32_t n_patch) {
    if (!c || c->kind != KIND_TILES) return CUTCELL_E_ARG;
    if (m && (!patch_red || !patch_gamma || n_patch <= 0)) return CUTCELL_E_ARG;
    c->mlp = m;
    // patch blocks set for the same layout stay attached
    const bool keep = c->pmap.binv && c->pmap.red == patch_red && c->pmap.n_patch == n_patch;
    c->pmap = PatchMap{n_patch, patch_red, patch_gamma, keep ? c->pmap.binv : nullptr, keep ? c->pmap.slot : nullptr};
    if (m && !c->zl) {
        CK(cudaMalloc(&c->zl, (size_t)c->n * sizeof(double)));
        CK(cudaMalloc(&c->rold, (size_t)c->n * sizeof(double)));
    }
    return CUTCELL_OK;
}

// ---------------------------------------------------------------------------
// periodic-hill fast diagonalisation
// ---------------------------------------------------------------------------

__global__ void fd_transpose_kernel(int n, const double* A, double* AT) {
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < (long)n * n; t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t / n), j = (int)(t % n);
        AT[(size_t)j * n + i] = A[t];
    }
}

int cutcell_fastdiag_create(int32_t nr, int32_t nz, const double* M2, const double* Qx2, const double* Qy2,
                            const double* mu, const double* kap, const double* Ainv, const double* Sinv,
                            cutcell_fastdiag** out) {
    if (!out || nr <= 0 || nz <= 0 || !M2 || !Qx2 || !Qy2 || !mu || !kap || !Ainv || !Sinv) return CUTCELL_E_ARG;
    if ((size_t)6 * nr * sizeof(double) > 200 * 1024) return CUTCELL_E_SHAPE;  // per-mode vectors staged in shared memory
    cutcell_fastdiag* f = new cutcell_fastdiag();
    CK(cudaGetDevice(&f->device));
    const size_t vec = (size_t)nz * nr * sizeof(double);
    CK(cudaMalloc(&f->X, 6 * vec));
    CK(cudaMalloc(&f->T, 6 * vec));
    CK(cudaMalloc(&f->UT, 6 * vec));
    CK(cudaMalloc(&f->G, 6 * vec));
    CK(cudaMalloc(&f->U, 6 * vec));
    CK(cudaMalloc(&f->S2, 2 * vec * 8));  // Gx Gy Gz DIV P Hx Hy Hz
    CK(cudaMalloc(&f->part, (size_t)FD_KSPLIT * 6 * vec));  // split-K partial products
    CK(cudaMalloc(&f->QxT, (size_t)nr * nr * sizeof(double)));
    CK(cudaMalloc(&f->QyT, (size_t)nr * nr * sizeof(double)));
    CK(cudaMalloc(&f->cosT, (size_t)nz * nz * sizeof(double)));
    CK(cudaMalloc(&f->sinT, (size_t)nz * nz * sizeof(double)));
    std::vector<double> ct((size_t)nz * nz), st((size_t)nz * nz);
    for (int a = 0; a < nz; ++a)
        for (int b = 0; b < nz; ++b) {
            // reduce a*b mod nz first so the angle stays in [0, 2 pi)
            const double ang = 2.0 * M_PI * (double)((a * b) % nz) / nz;
            ct[(size_t)a * nz + b] = std::cos(ang);
            st[(size_t)a * nz + b] = std::sin(ang);
        }
    CK(cudaMemcpy(f->cosT, ct.data(), ct.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(f->sinT, st.data(), st.size() * sizeof(double), cudaMemcpyHostToDevice));
    fd_transpose_kernel<<<ceil_div((long)nr * nr, 256), 256>>>(nr, Qx2, f->QxT);
    fd_transpose_kernel<<<ceil_div((long)nr * nr, 256), 256>>>(nr, Qy2, f->QyT);
    FastDiagDev& d = f->d;
    d.nr = nr;
    d.nz = nz;
    d.M2 = M2;
    d.Qx2 = Qx2;
    d.Qy2 = Qy2;
    d.Qx2T = f->QxT;
    d.Qy2T = f->QyT;
    d.mu = mu;
    d.kap = kap;
    d.Ainv = Ainv;
    d.Sinv = Sinv;
    d.cosT = f->cosT;
    d.sinT = f->sinT;
    const int smem6 = (int)(6 * nr * sizeof(double)), smem2 = (int)(2 * nr * sizeof(double));
    CK(cudaFuncSetAttribute(fd_mode_mv_kernel<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem6));
    CK(cudaFuncSetAttribute(fd_mode_mv_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem2));
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    *out = f;
    return CUTCELL_OK;
}

// Ypart[z][v][r] = sum_{k in kslice(z)} A[r][k] X_v[k] on the FP64 tensor cores
// (dmma_tile: M = nr rows of the shared operator, N = the nvec vectors, split
// over K by blockIdx.z); fd_sum_ksplit_kernel adds the slices in order.
__global__ void __launch_bounds__(256) fd_dmma_kernel(int nr, const double* A, const double* X, VecSel sx,
                                                      double* Ypart, int nvec) {
    const int kch = (nr + gridDim.z - 1) / gridDim.z;
    const int kb = blockIdx.z * kch, ke = min(nr, kb + kch);
    double* Yz = Ypart + (size_t)blockIdx.z * nvec * nr;
    dmma_tile(
        nr, nvec, kb, ke, blockIdx.y * DG_BM, blockIdx.x * DG_BN,
        [&](int m, int k) { return __ldg(A + (size_t)m * nr + k); },
        [&](int v, int k) { return __ldg(X + vec_off(sx, v, nr) + k); },
        [&](int m, int v, double val) { Yz[(size_t)v * nr + m] = val; });
}

static void fd_gemm(cudaStream_t s, int nr, const double* A, const double* X, VecSel sx, double* Y, VecSel sy,
                    int nvec, double* part) {
    dim3 grid(ceil_div(nvec, DG_BN), ceil_div(nr, DG_BM), FD_KSPLIT);
    fd_dmma_kernel<<<grid, 256, 0, s>>>(nr, A, X, sx, part, nvec);
    fd_sum_ksplit_kernel<<<ceil_div((long)nvec * nr, 256), 256, 0, s>>>(nr, nvec, FD_KSPLIT, part, Y, sy);
}

int cutcell_fastdiag_solve(cutcell_fastdiag* f, const double* ux, const double* uy, const double* uz, double* ox,
                           double* oy, double* oz, void* stream) {
    if (!f || !ux || !uy || !uz || !ox || !oy || !oz) return CUTCELL_E_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const FastDiagDev& d = f->d;
    const int nr = d.nr, nz = d.nz;
    const size_t v2 = (size_t)2 * nz * nr;
    double* Gx = f->S2;
    double* Gy = Gx + v2;
    double* Gz = Gy + v2;
    double* DIV = Gz + v2;
    double* P = DIV + v2;
    double* Hx = P + v2;
    double* Hy = Hx + v2;
    double* Hz = Hy + v2;
    const int ew = ceil_div((long)nz * nr * 3, 256);
    const int rows = nr >= 1024 ? 128 : 32;
    dim3 mv_grid(ceil_div(nr, rows), nz);
    fd_dft_kernel<<<ew, 256, 0, s>>>(d, ux, uy, uz, f->X);
    fd_gemm(s, nr, d.M2, f->X, VecSel{6, 0, 6}, f->T, VecSel{6, 0, 6}, 6 * nz, f->part);
    fd_scale_mu_kernel<<<ceil_div((long)nz * 6 * nr, 256), 256, 0, s>>>(d, f->T);
    fd_mode_mv_kernel<6><<<mv_grid, FD_MV_THREADS, 6 * nr * sizeof(double), s>>>(nr, d.Ainv, f->T, f->UT, nullptr, rows);
    fd_gemm(s, nr, d.Qx2, f->UT, VecSel{2, 0, 6}, Gx, VecSel{2, 0, 2}, 2 * nz, f->part);
    fd_gemm(s, nr, d.Qy2, f->UT, VecSel{2, 2, 6}, Gy, VecSel{2, 0, 2}, 2 * nz, f->part);
    fd_gemm(s, nr, d.M2, f->UT, VecSel{2, 4, 6}, Gz, VecSel{2, 0, 2}, 2 * nz, f->part);
    fd_div_kernel<<<ceil_div((long)nz * nr, 256), 256, 0, s>>>(d, Gx, Gy, Gz, DIV);
    fd_mode_mv_kernel<2><<<mv_grid, FD_MV_THREADS, 2 * nr * sizeof(double), s>>>(nr, d.Sinv, DIV, P, nullptr, rows);
    fd_gemm(s, nr, d.Qx2T, P, VecSel{2, 0, 2}, Hx, VecSel{2, 0, 2}, 2 * nz, f->part);
    fd_gemm(s, nr, d.Qy2T, P, VecSel{2, 0, 2}, Hy, VecSel{2, 0, 2}, 2 * nz, f->part);
    fd_gemm(s, nr, d.M2, P, VecSel{2, 0, 2}, Hz, VecSel{2, 0, 2}, 2 * nz, f->part);
    fd_grad_kernel<<<ceil_div((long)nz * nr, 256), 256, 0, s>>>(d, Hx, Hy, Hz, f->G);
    fd_mode_mv_kernel<6><<<mv_grid, FD_MV_THREADS, 6 * nr * sizeof(double), s>>>(nr, d.Ainv, f->G, f->U, f->UT, rows);
    fd_idft_kernel<<<ew, 256, 0, s>>>(d, f->U, ox, oy, oz);
    CK(cudaGetLastError());
    return CUTCELL_OK;
}

int cutcell_fastdiag_destroy(cutcell_fastdiag* f) {
    if (!f) return CUTCELL_E_ARG;
    cudaSetDevice(f->device);  // cudaFree below waits for the work that may still use the buffers
    void* bufs[] = {f->X, f->T, f->UT, f->G, f->U, f->S2, f->QxT, f->QyT, f->cosT, f->sinT, f->part};
    for (void* b : bufs)
        if (b) cudaFree(b);
    delete f;
    return CUTCELL_OK;
}

}  // extern "C"
