// Batched Jacobi-PCG: many independent CSR systems of uneven size solved in
// one persistent launch.  The reference solves its sweeps one system at a
// time through solve_cpu_cg / solve_gpu_cg (code/fast_solver_workbench.py:
// 169-176, code/fast_solver_backends.py:90-132,194-289); the per-system
// iteration here is the same Jacobi-PCG with the same stopping test as the
// single-system kernel (pcg.cuh, pcg_core).
//
// Work decomposition
//   * A team is one thread-block cluster of C CTAs (C = 1, 2, 4, 8 or 16).  Teams
//     claim problems from a global counter in a host-chosen order (heaviest
//     first), so uneven sizes balance without any grid-wide barrier.
//   * A problem's rows are split into C contiguous slices, one per CTA.  Each
//     CTA keeps x, r, A p and D^-1 of its rows, and full-length copies of z
//     and p, in shared memory; after each r update every CTA stores its slice
//     of z into all C copies of z through distributed shared memory (DSMEM).
//   * A CTA's CSR slice is staged once per problem into shared memory (16-bit
//     column indices) when it fits the configured budget; otherwise it is
//     read from global memory (L2-resident for these sizes) every iteration.
//   * Dot products: a deterministic block sum, each CTA's partial stored into
//     every CTA's slot array, one hardware cluster barrier, then every CTA adds
//     the C partials in rank order -- all CTAs hold the same bits and take the
//     same branches, so the cluster barriers are always matched.
// Two cluster barriers per iteration: p.Ap, and r.r / r.z together with the
// gather of z = D^-1 r; every CTA then forms the whole p = z + beta p itself.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

namespace cg = cooperative_groups;

void cutcell_internal_set_error(const std::string& what);

#define BATCH_MAX_THREADS 512
#define BATCH_MAX_CLUSTER 16  // 16 is a non-portable cluster size (allowed on B200)
#define BATCH_MAX_N 16384  // per system: the full copy of p must sit in shared memory

namespace {

struct BatchProblem {
    int n, nnz;
    int ptr_off;       // first of the problem's n + 1 row offsets (values 0 .. nnz)
    int vec_off;       // first entry of the problem's b / x
    long long nz_off;  // first nonzero of the problem in indices / data
    int tpr_log2;      // lanes per row (log2)
    int pad;
};

struct BatchResult {
    int status, iterations;
    double rel, true_rel;
    unsigned long long t0, t1;  // %globaltimer (ns) when the team took / finished the system
    int team, pad;
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

struct BatchArgs {
    const BatchProblem* prob;
    const int* order;
    int n_prob;
    const int* indptr;
    const int* indices;
    const double* data;
    const double* b;
    double* x;
    double tol;
    int maxiter;
    int jacobi;
    BatchResult* res;
    unsigned* queue;
    int n_max;      // largest n in the batch
    int rows_max;   // ceil(n_max / C)
    int mat_bytes;  // shared-memory budget for a staged CSR slice (multiple of 16)
};

// Dynamic shared-memory layout (byte offsets, each 16-byte aligned).
struct BatchSmem {
    int pfull, zfull, x, r, q, d, slots, mat, total;
    __host__ __device__ static int vec_bytes(int n) { return 8 * ((n + 1) & ~1); }
    __host__ __device__ BatchSmem(int n_max, int rows_max, int mat_bytes) {
        pfull = 0;
        zfull = pfull + vec_bytes(n_max);
        x = zfull + vec_bytes(n_max);
        r = x + vec_bytes(rows_max);
        q = r + vec_bytes(rows_max);
        d = q + vec_bytes(rows_max);
        slots = d + vec_bytes(rows_max);
        mat = slots + 8 * 5 * 3 * BATCH_MAX_CLUSTER;  // 5 reduction groups x 3 values x 16 ranks
        total = mat + mat_bytes;
    }
};

// slot groups: one per reduction site, so a slot is never rewritten before
// every CTA has read it (at least one cluster barrier separates the two)
enum { SLOT_CHECK = 0, SLOT_INIT = 1, SLOT_PAP = 2, SLOT_RR = 3, SLOT_TRUE = 4 };

struct Team {
    cg::cluster_group cl;
    unsigned C, rank;
    __device__ Team() : cl(cg::this_cluster()) {
        C = cl.num_blocks();
        rank = cl.block_rank();
    }
    __device__ __forceinline__ void sync() const {
        if (C == 1)
            __syncthreads();
        else
            cl.sync();  // barrier.cluster arrive (release) + wait (acquire)
    }
    template <typename T>
    __device__ __forceinline__ T* at(T* p, unsigned c) const {
        return C == 1 ? p : cl.map_shared_rank(p, c);
    }
};

// Team-wide sums of NV per-thread values; every CTA ends with identical bits.
// Warp partials -> warp 0 (fixed shuffle tree) -> lane c stores the CTA's
// partial into rank c's slot -> one team barrier -> rank-ordered sum.
template <int NV>
__device__ __forceinline__ void team_sum(double (&v)[NV], double* sh, double* slots, int group, const Team& t) {
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = warp_sum(v[q]);
    if (l == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) sh[q * 16 + w] = v[q];
    }
    __syncthreads();
    double* gs = slots + group * 3 * BATCH_MAX_CLUSTER;
    if (w == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double s = (l < nw) ? sh[q * 16 + l] : 0.0;
            s = warp_sum(s);
            if (l < (int)t.C) *t.at(gs + q * BATCH_MAX_CLUSTER + t.rank, (unsigned)l) = s;
        }
    }
    t.sync();
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double s = 0.0;
        for (unsigned c = 0; c < t.C; ++c) s += gs[q * BATCH_MAX_CLUSTER + c];
        v[q] = s;
    }
}

// q[i] = sum_k val[k] pin[col[k]] over the CTA's rows, tpr lanes per row; returns
// this thread's share of sum_i pdot[i] q[i] (pdot may be null).  The row loop has
// the same trip count on every lane, so the group shuffles are always full-warp.
// Each lane keeps four independent accumulators so that its loads overlap.
template <typename ColT, bool LDG>
__device__ __forceinline__ double spmv_rows(int nown, int tl, const int* rp, int rp_base, const ColT* col,
                                            const double* val, const double* pin, double* qout,
                                            const double* pdot) {
    const int tpr = 1 << tl;
    const int groups = blockDim.x >> tl;
    const int g = threadIdx.x >> tl, lane = threadIdx.x & (tpr - 1);
    double dot = 0.0;
    for (int base = 0; base < nown; base += groups) {
        const int i = base + g;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        if (i < nown) {
            const int kb = (LDG ? __ldg(rp + i) : rp[i]) - rp_base;
            const int ke = (LDG ? __ldg(rp + i + 1) : rp[i + 1]) - rp_base;
            int k = kb + lane;
            for (; k + 3 * tpr < ke; k += 4 * tpr) {
                int c[4];
                double v[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    c[u] = LDG ? (int)__ldg(col + k + u * tpr) : (int)col[k + u * tpr];
                    v[u] = LDG ? __ldg(val + k + u * tpr) : val[k + u * tpr];
                }
                s0 = fma(v[0], pin[c[0]], s0);
                s1 = fma(v[1], pin[c[1]], s1);
                s2 = fma(v[2], pin[c[2]], s2);
                s3 = fma(v[3], pin[c[3]], s3);
            }
            for (; k < ke; k += tpr) {
                const int c = LDG ? (int)__ldg(col + k) : (int)col[k];
                const double v = LDG ? __ldg(val + k) : val[k];
                s0 = fma(v, pin[c], s0);
            }
        }
        double s = (s0 + s1) + (s2 + s3);
        for (int o = tpr >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (i < nown && lane == 0) {
            qout[i] = s;
            if (pdot) dot = fma(pdot[i], s, dot);
        }
    }
    return dot;
}

__global__ void __launch_bounds__(BATCH_MAX_THREADS) batch_pcg_kernel(BatchArgs a) {
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ double sh[3 * 16];
    __shared__ int s_job;
    const Team t;
    const BatchSmem L(a.n_max, a.rows_max, a.mat_bytes);
    double* pfull = reinterpret_cast<double*>(smraw + L.pfull);  // p, full length, updated locally
    double* zfull = reinterpret_cast<double*>(smraw + L.zfull);  // z = D^-1 r, full length, gathered
    double* xo = reinterpret_cast<double*>(smraw + L.x);
    double* ro = reinterpret_cast<double*>(smraw + L.r);
    double* qo = reinterpret_cast<double*>(smraw + L.q);
    double* dio = reinterpret_cast<double*>(smraw + L.d);
    double* slots = reinterpret_cast<double*>(smraw + L.slots);
    unsigned char* mat = smraw + L.mat;

    for (;;) {
        if (t.rank == 0 && threadIdx.x == 0) {
            const int j = (int)atomicAdd(a.queue, 1u);
            for (unsigned c = 0; c < t.C; ++c) *t.at(&s_job, c) = j;
        }
        t.sync();
        const int j = s_job;
        if (j >= a.n_prob) break;
        const int pid = a.order[j];
        const BatchProblem P = a.prob[pid];
        const unsigned long long t_begin = global_ns();
        const int n = P.n;
        const int r0 = (int)(((long long)n * t.rank) / t.C);
        const int r1 = (int)(((long long)n * (t.rank + 1)) / t.C);
        const int nown = r1 - r0;
        const int* gptr = a.indptr + P.ptr_off;
        const int* gcol = a.indices + P.nz_off;
        const double* gval = a.data + P.nz_off;
        const double* b = a.b + P.vec_off;

        // ---- validate the slice and stage it when it fits -------------------
        double bad = 0.0;
        if (threadIdx.x == 0 && (gptr[0] != 0 || gptr[n] != P.nnz)) bad = 1.0;
        int kb0 = gptr[r0], ke0 = gptr[r1];
        kb0 = min(max(kb0, 0), P.nnz);
        ke0 = min(max(ke0, kb0), P.nnz);
        const int snnz = ke0 - kb0;
        const bool staged = 10LL * snnz + 4LL * (nown + 1) + 16 <= (long long)a.mat_bytes;
        double* sval = reinterpret_cast<double*>(mat);
        uint16_t* scol = reinterpret_cast<uint16_t*>(mat + 8 * (size_t)snnz);
        int* srp = reinterpret_cast<int*>(mat + ((10 * (size_t)snnz + 3) & ~(size_t)3));
        for (int i = threadIdx.x; i < nown; i += blockDim.x) {
            const int lo = gptr[r0 + i], hi = gptr[r0 + i + 1];
            if (lo > hi || lo < kb0 || hi > ke0) bad = 1.0;
            if (staged) srp[i] = lo - kb0;
        }
        if (staged && threadIdx.x == 0) srp[nown] = snnz;
        for (int k = threadIdx.x; k < snnz; k += blockDim.x) {
            const int c = gcol[kb0 + k];
            if (c < 0 || c >= n) bad = 1.0;
            if (staged) {
                scol[k] = (uint16_t)min(max(c, 0), n - 1);
                sval[k] = gval[kb0 + k];
            }
        }
        {
            double v[1] = {bad};
            team_sum<1>(v, sh, slots, SLOT_CHECK, t);
            bad = v[0];
        }
        if (bad > 0.0) {
            if (t.rank == 0 && threadIdx.x == 0) {
                BatchResult R;
                R.status = CUTCELL_E_SHAPE;
                R.iterations = 0;
                R.rel = -1.0;
                R.true_rel = -1.0;
                R.t0 = t_begin;
                R.t1 = global_ns();
                R.team = blockIdx.x / t.C;
                R.pad = 0;
                a.res[pid] = R;
            }
            t.sync();
            continue;
        }
        // the row offsets seen through the chosen source
        const int* rp = staged ? srp : gptr + r0;
        const int rp_base = staged ? 0 : kb0;

        // ---- x = 0, r = b, z = D^-1 r (published to every CTA), p = z -------
        double init[2] = {0.0, 0.0};
        for (int i = threadIdx.x; i < nown; i += blockDim.x) {
            const int row = r0 + i;
            double dg = 0.0;
            const int kb = rp[i] - rp_base, ke = rp[i + 1] - rp_base;
            for (int k = kb; k < ke; ++k) {
                const int c = staged ? (int)scol[k] : gcol[kb0 + k];
                if (c == row) dg += staged ? sval[k] : gval[kb0 + k];
            }
            const double di = (a.jacobi && fabs(dg) > 0.0) ? 1.0 / dg : 1.0;
            dio[i] = di;
            const double bi = b[row];
            xo[i] = 0.0;
            ro[i] = bi;
            const double zi = di * bi;
            for (unsigned c = 0; c < t.C; ++c) t.at(zfull, c)[row] = zi;
            init[0] += bi * zi;
            init[1] += bi * bi;
        }
        team_sum<2>(init, sh, slots, SLOT_INIT, t);  // its barrier also publishes z
        for (int i = threadIdx.x; i < n; i += blockDim.x) pfull[i] = zfull[i];
        __syncthreads();
        double rz = init[0];
        double bnorm = sqrt(init[1]);
        if (bnorm == 0.0) bnorm = 1.0;

        const int* lcol_g = gcol + kb0;
        const double* lval_g = gval + kb0;
        int status = CUTCELL_E_NOCONV;
        int k = 1;
        double rel = 1.0;
        for (k = 1; k <= a.maxiter; ++k) {
            double v1[1];
            v1[0] = staged ? spmv_rows<uint16_t, false>(nown, P.tpr_log2, rp, 0, scol, sval, pfull, qo, pfull + r0)
                           : spmv_rows<int, true>(nown, P.tpr_log2, rp, rp_base, lcol_g, lval_g, pfull, qo, pfull + r0);
            team_sum<1>(v1, sh, slots, SLOT_PAP, t);  // its barriers also complete q
            const double pap = v1[0];
            if (!(pap > 0.0) || !isfinite(pap)) {
                status = CUTCELL_E_BREAKDOWN;
                break;
            }
            const double alpha = rz / pap;
            double v2[2] = {0.0, 0.0};
            for (int i = threadIdx.x; i < nown; i += blockDim.x) {
                xo[i] += alpha * pfull[r0 + i];
                const double ri = ro[i] - alpha * qo[i];
                ro[i] = ri;
                const double zi = dio[i] * ri;
                for (unsigned c = 0; c < t.C; ++c) t.at(zfull, c)[r0 + i] = zi;
                v2[0] += ri * ri;
                v2[1] += ri * zi;
            }
            team_sum<2>(v2, sh, slots, SLOT_RR, t);  // its barrier also publishes z
            rel = sqrt(v2[0]) / bnorm;
            if (!isfinite(rel)) {
                status = CUTCELL_E_NAN;
                break;
            }
            if (rel <= a.tol) {
                status = CUTCELL_OK;
                break;
            }
            const double beta = v2[1] / rz;
            rz = v2[1];
            // every CTA forms the whole new p from the gathered z: identical bits
            // in all copies, and no third barrier for publishing p
            for (int i = threadIdx.x; i < n; i += blockDim.x) pfull[i] = zfull[i] + beta * pfull[i];
            __syncthreads();
        }
        const int iters = (k > a.maxiter) ? a.maxiter : k;

        // ---- true residual ||b - A x|| / ||b|| in FP64 ------------------------
        t.sync();  // every CTA is done reading z before x overwrites it
        for (int i = threadIdx.x; i < nown; i += blockDim.x)
            for (unsigned c = 0; c < t.C; ++c) t.at(zfull, c)[r0 + i] = xo[i];
        t.sync();
        if (staged)
            spmv_rows<uint16_t, false>(nown, P.tpr_log2, rp, 0, scol, sval, zfull, qo, nullptr);
        else
            spmv_rows<int, true>(nown, P.tpr_log2, rp, rp_base, lcol_g, lval_g, zfull, qo, nullptr);
        __syncthreads();
        double v3[1] = {0.0};
        double* x = a.x + P.vec_off;
        for (int i = threadIdx.x; i < nown; i += blockDim.x) {
            const double e = b[r0 + i] - qo[i];
            v3[0] += e * e;
            x[r0 + i] = xo[i];
        }
        team_sum<1>(v3, sh, slots, SLOT_TRUE, t);
        if (t.rank == 0 && threadIdx.x == 0) {
            BatchResult R;
            R.status = status;
            R.iterations = iters;
            R.rel = rel;
            R.true_rel = sqrt(v3[0]) / bnorm;
            R.t0 = t_begin;
            R.t1 = global_ns();
            R.team = blockIdx.x / t.C;
            R.pad = 0;
            a.res[pid] = R;
        }
        t.sync();  // shared vectors, slots and s_job are reused by the next problem
    }
}

// Makes the context's device current for one call and restores the caller's.
struct DeviceGuard {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit DeviceGuard(int dev) {
        err = cudaGetDevice(&prev);
        if (err == cudaSuccess && prev != dev) err = cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

int fail(cudaError_t e, const char* what) {
    cutcell_internal_set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return CUTCELL_E_CUDA;
}

int arg_error(const std::string& what, int code = CUTCELL_E_ARG) {
    cutcell_internal_set_error(what);
    return code;
}

#define BCK(call)                                         \
    do {                                                  \
        cudaError_t _e = (call);                          \
        if (_e != cudaSuccess) return fail(_e, #call);    \
    } while (0)

}  // namespace

struct cutcell_batch {
    int device = 0;
    int n_prob = 0;
    std::vector<int> n, nnz;
    std::vector<int> ptr_off, vec_off;
    std::vector<long long> nz_off;
    int n_max = 0;
    long long vec_total = 0;
    const int* indptr = nullptr;
    const int* indices = nullptr;
    const double* data = nullptr;
    BatchProblem* d_prob = nullptr;
    int* d_order = nullptr;
    BatchResult* d_res = nullptr;
    BatchResult* h_res = nullptr;  // pinned
    unsigned* d_queue = nullptr;
    cudaStream_t cap = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // configuration
    bool configured = false;
    int cluster = 1, threads = 256, mat_bytes = 0, teams = 0, smem = 0;
    int version = 0;
    // captured graph and the arguments it was captured with
    cudaGraphExec_t exec = nullptr;
    int g_version = -1;
    const double* g_b = nullptr;
    double* g_x = nullptr;
    double g_tol = 0.0;
    int g_maxiter = -1, g_pre = -1;

    ~cutcell_batch() {
        if (exec) cudaGraphExecDestroy(exec);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (cap) cudaStreamDestroy(cap);
        cudaFree(d_prob);
        cudaFree(d_order);
        cudaFree(d_res);
        cudaFree(d_queue);
        if (h_res) cudaFreeHost(h_res);
    }
};

namespace {

int capture(cutcell_batch* B, const double* rhs, double* x, double tol, int maxiter, int pre) {
    if (B->exec) {
        cudaGraphExecDestroy(B->exec);
        B->exec = nullptr;
    }
    BatchArgs a;
    memset(&a, 0, sizeof(a));
    a.prob = B->d_prob;
    a.order = B->d_order;
    a.n_prob = B->n_prob;
    a.indptr = B->indptr;
    a.indices = B->indices;
    a.data = B->data;
    a.b = rhs;
    a.x = x;
    a.tol = tol;
    a.maxiter = maxiter;
    a.jacobi = pre == CUTCELL_PRECOND_JACOBI;
    a.res = B->d_res;
    a.queue = B->d_queue;
    a.n_max = B->n_max;
    a.rows_max = (B->n_max + B->cluster - 1) / B->cluster;
    a.mat_bytes = B->mat_bytes;

    cudaLaunchConfig_t cfg;
    memset(&cfg, 0, sizeof(cfg));
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = B->cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(B->teams * B->cluster);
    cfg.blockDim = dim3(B->threads);
    cfg.dynamicSmemBytes = B->smem;
    cfg.stream = B->cap;
    cfg.attrs = attr;
    cfg.numAttrs = 1;

    cudaGraph_t g = nullptr;
    BCK(cudaStreamBeginCapture(B->cap, cudaStreamCaptureModeThreadLocal));
    cudaError_t e1 = cudaMemsetAsync(B->d_queue, 0, sizeof(unsigned), B->cap);
    cudaError_t e2 = e1 == cudaSuccess ? cudaLaunchKernelEx(&cfg, batch_pcg_kernel, a) : e1;
    cudaError_t e3 = e2 == cudaSuccess ? cudaMemcpyAsync(B->h_res, B->d_res, sizeof(BatchResult) * B->n_prob,
                                                         cudaMemcpyDeviceToHost, B->cap)
                                       : e2;
    cudaError_t e4 = cudaStreamEndCapture(B->cap, &g);
    if (e3 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return fail(e3, "batch graph capture");
    }
    if (e4 != cudaSuccess) return fail(e4, "cudaStreamEndCapture");
    cudaError_t e5 = cudaGraphInstantiate(&B->exec, g, 0);
    cudaGraphDestroy(g);
    if (e5 != cudaSuccess) {
        B->exec = nullptr;
        return fail(e5, "cudaGraphInstantiate");
    }
    B->g_version = B->version;
    B->g_b = rhs;
    B->g_x = x;
    B->g_tol = tol;
    B->g_maxiter = maxiter;
    B->g_pre = pre;
    return CUTCELL_OK;
}

}  // namespace

extern "C" {

int cutcell_batch_create(int32_t n_problems, const int32_t* n, const int32_t* nnz, const int32_t* indptr,
                         const int32_t* indices, const double* data, cutcell_batch** out) {
    if (!out) return CUTCELL_E_ARG;
    *out = nullptr;
    if (n_problems <= 0 || !n || !nnz || !indptr) return arg_error("batch: empty batch or null sizes");
    cutcell_batch* B = new cutcell_batch();
    B->n_prob = n_problems;
    long long ptr_total = 0, nz_total = 0;
    for (int i = 0; i < n_problems; ++i) {
        if (n[i] < 1 || n[i] > BATCH_MAX_N || nnz[i] < 0) {
            delete B;
            return arg_error("batch: system " + std::to_string(i) + " has n outside [1, 16384] or nnz < 0",
                             CUTCELL_E_SHAPE);
        }
        B->n.push_back(n[i]);
        B->nnz.push_back(nnz[i]);
        B->ptr_off.push_back((int)ptr_total);
        B->vec_off.push_back((int)B->vec_total);
        B->nz_off.push_back(nz_total);
        ptr_total += n[i] + 1;
        B->vec_total += n[i];
        nz_total += nnz[i];
        B->n_max = std::max(B->n_max, n[i]);
    }
    if (ptr_total > 0x7fffffffLL || B->vec_total > 0x7fffffffLL) {
        delete B;
        return arg_error("batch: packed row offsets exceed 2^31", CUTCELL_E_SHAPE);
    }
    if (nz_total > 0 && (!indices || !data)) {
        delete B;
        return arg_error("batch: null indices / data");
    }
    B->indptr = indptr;
    B->indices = indices;
    B->data = data;
    int st = CUTCELL_OK;
    cudaError_t e = cudaGetDevice(&B->device);
    if (e == cudaSuccess) e = cudaMalloc(&B->d_prob, sizeof(BatchProblem) * n_problems);
    if (e == cudaSuccess) e = cudaMalloc(&B->d_order, sizeof(int) * n_problems);
    if (e == cudaSuccess) e = cudaMalloc(&B->d_res, sizeof(BatchResult) * n_problems);
    if (e == cudaSuccess) e = cudaMalloc(&B->d_queue, 128);
    if (e == cudaSuccess) e = cudaMallocHost(&B->h_res, sizeof(BatchResult) * n_problems);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&B->cap, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&B->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&B->ev1);
    if (e != cudaSuccess) st = fail(e, "cutcell_batch_create");
    if (st) {
        delete B;
        return st;
    }
    *out = B;
    return CUTCELL_OK;
}

int cutcell_batch_configure(cutcell_batch* B, const CutcellBatchConfig* cfg, const int32_t* lanes_per_row,
                            const int32_t* order) {
    if (!B || !cfg || !lanes_per_row || !order) return CUTCELL_E_ARG;
    const int C = cfg->cluster, T = cfg->threads;
    if (!(C == 1 || C == 2 || C == 4 || C == 8 || C == 16))
        return arg_error("batch: cluster must be 1, 2, 4, 8 or 16");
    if (T < 32 || T > BATCH_MAX_THREADS || (T % 32) != 0) return arg_error("batch: threads must be 32..512, x32");
    if (cfg->smem_matrix < 0 || (cfg->smem_matrix % 16) != 0)
        return arg_error("batch: smem_matrix must be a non-negative multiple of 16");
    if (cfg->teams < 0) return arg_error("batch: teams must be >= 0");
    std::vector<int> seen(B->n_prob, 0);
    std::vector<BatchProblem> hp(B->n_prob);
    for (int i = 0; i < B->n_prob; ++i) {
        const int o = order[i];
        if (o < 0 || o >= B->n_prob || seen[o]++) return arg_error("batch: order is not a permutation");
        const int l = lanes_per_row[i];
        if (l < 1 || l > 32 || (l & (l - 1)) != 0 || l > T)
            return arg_error("batch: lanes_per_row must be a power of two in [1, min(32, threads)]");
        int tl = 0;
        while ((1 << tl) < l) ++tl;
        hp[i].n = B->n[i];
        hp[i].nnz = B->nnz[i];
        hp[i].ptr_off = B->ptr_off[i];
        hp[i].vec_off = B->vec_off[i];
        hp[i].nz_off = B->nz_off[i];
        hp[i].tpr_log2 = tl;
        hp[i].pad = 0;
    }
    const int rows_max = (B->n_max + C - 1) / C;
    const BatchSmem L(B->n_max, rows_max, cfg->smem_matrix);
    int optin = 0;
    DeviceGuard dg(B->device);
    BCK(dg.err);
    BCK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, B->device));
    const int static_bytes = (int)(sizeof(double) * 3 * 16 + sizeof(int));
    if (L.total + static_bytes > optin)
        return arg_error("batch: shared memory " + std::to_string(L.total) + " B exceeds the per-block limit " +
                             std::to_string(optin - static_bytes),
                         CUTCELL_E_SHAPE);
    BCK(cudaFuncSetAttribute(batch_pcg_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, L.total));
    if (C > 8) BCK(cudaFuncSetAttribute(batch_pcg_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));

    cudaLaunchConfig_t lc;
    memset(&lc, 0, sizeof(lc));
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    lc.gridDim = dim3(C * B->n_prob);
    lc.blockDim = dim3(T);
    lc.dynamicSmemBytes = L.total;
    lc.attrs = attr;
    lc.numAttrs = 1;
    int max_clusters = 0;
    BCK(cudaOccupancyMaxActiveClusters(&max_clusters, batch_pcg_kernel, &lc));
    if (max_clusters < 1) return arg_error("batch: configuration does not fit on the device", CUTCELL_E_SHAPE);
    int teams = std::min(max_clusters, B->n_prob);
    if (cfg->teams > 0) teams = std::min(teams, cfg->teams);

    std::vector<int> ord(order, order + B->n_prob);
    BCK(cudaMemcpy(B->d_prob, hp.data(), sizeof(BatchProblem) * B->n_prob, cudaMemcpyHostToDevice));
    BCK(cudaMemcpy(B->d_order, ord.data(), sizeof(int) * B->n_prob, cudaMemcpyHostToDevice));
    B->cluster = C;
    B->threads = T;
    B->mat_bytes = cfg->smem_matrix;
    B->teams = teams;
    B->smem = L.total;
    B->configured = true;
    ++B->version;
    return CUTCELL_OK;
}

int cutcell_batch_info(const cutcell_batch* B, int32_t* teams, int32_t* smem_bytes) {
    if (!B || !B->configured) return CUTCELL_E_ARG;
    if (teams) *teams = B->teams;
    if (smem_bytes) *smem_bytes = B->smem;
    return CUTCELL_OK;
}

int cutcell_batch_solve(cutcell_batch* B, const double* rhs, double* x, double tol, int32_t maxiter,
                        int32_t precond, CutcellReport* reports, void* stream) {
    if (!B || !rhs || !x || !reports || maxiter < 0 || !(tol >= 0.0)) return CUTCELL_E_ARG;
    if (!B->configured) return arg_error("batch: cutcell_batch_configure has not been called");
    if (precond != CUTCELL_PRECOND_NONE && precond != CUTCELL_PRECOND_JACOBI)
        return arg_error("batch: preconditioner must be none or jacobi");
    DeviceGuard dg(B->device);
    BCK(dg.err);
    if (!B->exec || B->g_version != B->version || B->g_b != rhs || B->g_x != x || B->g_tol != tol ||
        B->g_maxiter != maxiter || B->g_pre != precond) {
        const int st = capture(B, rhs, x, tol, maxiter, precond);
        if (st) return st;
    }
    cudaStream_t s = (cudaStream_t)stream;
    BCK(cudaEventRecord(B->ev0, s));
    BCK(cudaGraphLaunch(B->exec, s));
    BCK(cudaEventRecord(B->ev1, s));
    BCK(cudaEventSynchronize(B->ev1));
    float ms = 0.0f;
    BCK(cudaEventElapsedTime(&ms, B->ev0, B->ev1));
    int worst = CUTCELL_OK;
    for (int i = 0; i < B->n_prob; ++i) {
        const BatchResult& R = B->h_res[i];
        CutcellReport& r = reports[i];
        r.status = R.status;
        r.iterations = R.iterations;
        r.outer_iterations = 1;
        r.blocks = B->cluster;
        r.relative_residual = R.rel;
        r.true_relative_residual = R.true_rel;
        r.elapsed_ms = ms;
        if (R.status == CUTCELL_E_SHAPE) worst = CUTCELL_E_SHAPE;
    }
    return worst;
}

int cutcell_batch_timeline(const cutcell_batch* B, double* start_us, double* end_us, int32_t* team) {
    if (!B || !B->exec) return arg_error("batch: no solve has run");
    unsigned long long t_min = ~0ULL;
    for (int i = 0; i < B->n_prob; ++i) t_min = std::min(t_min, B->h_res[i].t0);
    for (int i = 0; i < B->n_prob; ++i) {
        const BatchResult& R = B->h_res[i];
        if (start_us) start_us[i] = 1e-3 * (double)(R.t0 - t_min);
        if (end_us) end_us[i] = 1e-3 * (double)(R.t1 - t_min);
        if (team) team[i] = R.team;
    }
    return CUTCELL_OK;
}

int cutcell_batch_destroy(cutcell_batch* B) {
    if (!B) return CUTCELL_E_ARG;
    DeviceGuard dg(B->device);
    delete B;
    return CUTCELL_OK;
}

}  // extern "C"
