// Allocation-free Jacobi-PCG on a CSR matrix.
//
// Some callers cannot allocate device memory at the moment they need a
// solve: code running while a framework's caching allocator has reserved the
// whole device, latency-critical loops that must not take the implicit
// device-wide synchronisation of cudaMalloc / cudaFree, or hosts whose memory
// budget is fixed when they start.  For them this file provides one entry
// point whose working memory is a file-scope __device__ array of fixed size:
// the caller passes the matrix, b and x; everything else (Jacobi inverse,
// r, p, Ap, reduction partials, barrier words, result) lives in the array.
//
// The array exists once per GPU that loads the library and is held until
// the process exits.  Every call on a device shares it and it keeps the last
// call's contents, so the words that must start at zero are cleared on every
// call; two calls that overlap on the GPU (different streams, or different
// host threads) race on it and must be serialised by the caller.
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "pcg.cuh"

#define CUTCELL_NOALLOC_MAX_N 65536
#define CUTCELL_NOALLOC_MAX_BLOCKS 1024
#define CUTCELL_NOALLOC_CTRL_WORDS 256  // barrier / error words (unsigned), one 128-byte line each

namespace {

// layout in doubles: dinv | r | p | Ap | part[8][MAX_BLOCKS] | result | control words
constexpr size_t kVec = CUTCELL_NOALLOC_MAX_N;
constexpr size_t kOffDinv = 0;
constexpr size_t kOffR = kOffDinv + kVec;
constexpr size_t kOffP = kOffR + kVec;
constexpr size_t kOffAp = kOffP + kVec;
constexpr size_t kOffPart = kOffAp + kVec;
constexpr size_t kOffRes = kOffPart + 8 * (size_t)CUTCELL_NOALLOC_MAX_BLOCKS;
constexpr size_t kOffCtrl = kOffRes + 8;  // DevResult is 32 bytes; 64 reserved
constexpr size_t kTotalDoubles = kOffCtrl + CUTCELL_NOALLOC_CTRL_WORDS / 2;

}  // namespace

static __device__ __align__(256) double g_noalloc_scratch[kTotalDoubles];

namespace {

struct DeviceSetup {
    double* base = nullptr;  // device address of g_noalloc_scratch
    int blocks = 0;
    bool ready = false;
};

constexpr int kMaxDevices = 64;
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mu;
thread_local std::string g_noalloc_error;

// Skipped entirely when the structure check of the same call flagged the CSR
// (the row offsets could then point anywhere).
__global__ void noalloc_dinv_kernel(int n, const int* ptr, const int* idx, const double* val, int jacobi,
                                    double* dinv, const int* bad) {
    if (*((volatile const int*)bad)) return;
    for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
        double d = 0.0;
        if (jacobi)
            for (int k = ptr[row]; k < ptr[row + 1]; ++k)
                if (idx[k] == row) d += val[k];
        dinv[row] = (jacobi && fabs(d) > 0.0) ? 1.0 / d : 1.0;
    }
}

__global__ void __launch_bounds__(CUTCELL_BLOCK, 2) noalloc_pcg_kernel(CsrOp<double> op, SolveArgs a, const int* bad) {
    extern __shared__ double sm[];
    __shared__ double sh[CUTCELL_WARPS + 1];
    // a malformed CSR (flagged by the structure check before this launch) is
    // reported without reading it; every block sees the same flag and leaves
    if (*((volatile const int*)bad)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            a.res->status = CUTCELL_E_SHAPE;
            a.res->iterations = 0;
            a.res->outer = 0;
            a.res->rel = -1.0;
            a.res->true_rel = -1.0;
        }
        return;
    }
    int iters = 0;
    double rel = 1.0;
    int status = pcg_core(op, a.B, a.b, a.x, a.tol, a.maxiter, a.gs, sm, sh, 0.0, &iters, &rel);
    double true_rel = -1.0;
    if (status != CUTCELL_E_BARRIER && !grid_error(a.gs)) {
        const double bn = norm_of(a.b, a.B.n, a.B.part, a.gs, sh, 6);
        true_rel = true_residual(op, a.B, a.b, a.x, bn == 0.0 ? 1.0 : bn, a.gs, sm, sh, nullptr);
    }
    if (grid_error(a.gs)) status = CUTCELL_E_BARRIER;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.res->status = status;
        a.res->iterations = iters;
        a.res->outer = 1;
        a.res->rel = rel;
        a.res->true_rel = true_rel;
    }
}

int fail(cudaError_t e, const char* what) {
    g_noalloc_error = std::string(what) + ": " + cudaGetErrorString(e);
    return CUTCELL_E_CUDA;
}

// Once per device, with that device current: resolve the array's device
// address (the host-side name is only a stand-in) and the grid size.
int setup_device(int dev, DeviceSetup** out) {
    if (dev < 0 || dev >= kMaxDevices) {
        g_noalloc_error = "device ordinal beyond the library's fixed table of 64 devices";
        return CUTCELL_E_ARG;
    }
    std::lock_guard<std::mutex> lock(g_setup_mu);
    DeviceSetup& s = g_setup[dev];
    if (!s.ready) {
        cudaError_t e = cudaGetSymbolAddress((void**)&s.base, g_noalloc_scratch);
        if (e != cudaSuccess) return fail(e, "cudaGetSymbolAddress");
        int sms = 0, per = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return fail(e, "cudaDeviceGetAttribute");
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, noalloc_pcg_kernel, CUTCELL_BLOCK, 0);
        if (e != cudaSuccess) return fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        s.blocks = sms * per;
        if (s.blocks < 1 || s.blocks > CUTCELL_NOALLOC_MAX_BLOCKS) {
            g_noalloc_error = "grid does not fit the fixed reduction scratch";
            return CUTCELL_E_CUDA;
        }
        s.ready = true;
    }
    *out = &s;
    return CUTCELL_OK;
}

}  // namespace

extern "C" {

int cutcell_pcg_solve_csr_noalloc(int32_t n, int32_t nnz, const int32_t* indptr, const int32_t* indices,
                                  const double* data, const double* b, double* x, double tol, int32_t maxiter,
                                  int32_t precond, CutcellReport* report, void* stream) {
    g_noalloc_error.clear();
    if (n <= 0 || nnz < 0 || !indptr || (nnz > 0 && (!indices || !data)) || !b || !x || maxiter < 0 ||
        !(tol >= 0.0)) {
        g_noalloc_error = "invalid argument: n > 0, nnz >= 0, non-null arrays, maxiter >= 0 and tol >= 0 are required";
        return CUTCELL_E_ARG;
    }
    if (precond != CUTCELL_PRECOND_NONE && precond != CUTCELL_PRECOND_JACOBI) {
        g_noalloc_error = "invalid argument: precond must be CUTCELL_PRECOND_NONE or CUTCELL_PRECOND_JACOBI";
        return CUTCELL_E_ARG;
    }
    if (n > CUTCELL_NOALLOC_MAX_N) {
        g_noalloc_error = "n exceeds the fixed scratch (CUTCELL_NOALLOC_MAX_N unknowns)";
        return CUTCELL_E_SHAPE;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(e, "cudaGetDevice");
    DeviceSetup* S = nullptr;
    int st = setup_device(dev, &S);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    double* base = S->base;
    unsigned* ctrl = reinterpret_cast<unsigned*>(base + kOffCtrl);
    // words that must start at zero: barrier arrival, error and CSR-check words
    if ((e = cudaMemsetAsync(ctrl, 0, CUTCELL_NOALLOC_CTRL_WORDS * sizeof(unsigned), s)) != cudaSuccess)
        return fail(e, "cudaMemsetAsync");
    int* bad = reinterpret_cast<int*>(ctrl + 64);
    csr_check_kernel<<<ceil_div(n > nnz ? n : nnz, 256) < 1184 ? ceil_div(n > nnz ? n : nnz, 256) : 1184, 256, 0, s>>>(
        n, nnz, indptr, indices, bad);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "csr_check_kernel launch");
    noalloc_dinv_kernel<<<ceil_div(n, 256), 256, 0, s>>>(n, indptr, indices, data,
                                                        precond == CUTCELL_PRECOND_JACOBI, base + kOffDinv, bad);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "noalloc_dinv_kernel launch");
    const double mean = nnz / (double)n;
    int l2 = 0;
    while ((1 << l2) < 32 && (1 << l2) * 2 <= mean) ++l2;
    CsrOp<double> op{n, l2, indptr, indices, data};
    SolveArgs a;
    memset(&a, 0, sizeof(a));
    a.b = b;
    a.x = x;
    a.tol = tol;
    a.maxiter = maxiter;
    a.res = reinterpret_cast<DevResult*>(base + kOffRes);
    a.gs.count = ctrl;
    a.gs.limit_ns = cutcell_internal_wait_limit_ns();
    a.gs.err = reinterpret_cast<int*>(ctrl + 32);
    a.gs.nblocks = (unsigned)S->blocks;
    a.B.n = n;
    a.B.dinv = base + kOffDinv;
    a.B.r = base + kOffR;
    a.B.p = base + kOffP;
    a.B.Ap = base + kOffAp;
    a.B.part = base + kOffPart;
    const int* badc = bad;
    void* args[] = {(void*)&op, (void*)&a, (void*)&badc};
    e = cudaLaunchCooperativeKernel((const void*)noalloc_pcg_kernel, dim3(S->blocks), dim3(CUTCELL_BLOCK), args, 0, s);
    if (e != cudaSuccess) return fail(e, "cudaLaunchCooperativeKernel");
    DevResult hr;
    if ((e = cudaMemcpyAsync(&hr, a.res, sizeof(hr), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return fail(e, "cudaMemcpyAsync");
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return fail(e, "cudaStreamSynchronize");
    if (report) {
        report->status = hr.status;
        report->iterations = hr.iterations;
        report->outer_iterations = hr.outer;
        report->blocks = S->blocks;
        report->relative_residual = hr.rel;
        report->true_relative_residual = hr.true_rel;
        report->elapsed_ms = 0.0;  // not timed: no events are created on this path
    }
    if (hr.status == CUTCELL_E_SHAPE) {
        g_noalloc_error = "malformed CSR: row offsets must rise from 0 to nnz and columns lie in [0, n)";
        return CUTCELL_E_SHAPE;
    }
    if (hr.status == CUTCELL_E_BARRIER) {
        g_noalloc_error = "a device-wide wait ran out (cutcell_set_wait_limit)";
        return CUTCELL_E_BARRIER;
    }
    return CUTCELL_OK;
}

const char* cutcell_noalloc_last_error(void) { return g_noalloc_error.c_str(); }

}  // extern "C"
