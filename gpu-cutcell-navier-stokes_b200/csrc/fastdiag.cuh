// Periodic-hill fast-diagonalisation solve on the device: the algorithm of
// FastDiagHill::solve (cpp/include/cut/hill_fastdiag.h:47-79).
//
// Spectral layout: mode-major, component, real/imag part, 2D mode:
//   V[((k * NC + c) * 2 + part) * nr + m]
// so the 2*NC vectors of one Fourier mode are contiguous.  Stages:
//   1. DFT in z of (ux, uy, uz) -> X               (twiddle table, exact)
//   2. T  = mu_k M2 X                               (shared operator GEMM)
//   3. UT = Ainv_k T                                (per-mode streamed matvec, 6 rhs)
//   4. DIV = mu_k (Qx2 UTx + Qy2 UTy) + i kap_k M2 UTz   (3 shared GEMMs + combine)
//   5. P  = Sinv_k DIV                              (per-mode streamed matvec, 2 rhs)
//   6. G  = (mu_k Qx2^T P, mu_k Qy2^T P, -i kap_k M2 P)  (3 shared GEMMs + combine)
//   7. U  = UT - Ainv_k G                           (per-mode streamed matvec, 6 rhs)
//   8. inverse DFT with the 1/nz factor -> (ox, oy, oz)
// The per-mode inverses dominate the traffic: 3 nz nr^2 doubles per solve.
#pragma once

#include "common.cuh"

struct FastDiagDev {
    int nr, nz;
    const double* M2;
    const double* Qx2;
    const double* Qy2;
    const double* Qx2T;
    const double* Qy2T;
    const double* mu;
    const double* kap;
    const double* Ainv;  // [nz][nr][nr]
    const double* Sinv;  // [nz][nr][nr]
    const double* cosT;  // [nz][nz] cos(2 pi a b / nz)
    const double* sinT;  // [nz][nz] sin(2 pi a b / nz)
};

// 1. X[k][c][0/1][m] = sum_iz f_c(m, iz) (cos, -sin)(2 pi iz k / nz)
__global__ void fd_dft_kernel(FastDiagDev d, const double* ux, const double* uy, const double* uz, double* X) {
    const int nr = d.nr, nz = d.nz;
    const long total = (long)nr * nz * 3;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        const int m = (int)(t % nr);
        const int k = (int)((t / nr) % nz);
        const int c = (int)(t / ((long)nr * nz));
        const double* f = c == 0 ? ux : (c == 1 ? uy : uz);
        double re = 0.0, im = 0.0;
        for (int iz = 0; iz < nz; ++iz) {
            const double v = f[(size_t)m * nz + iz];
            re += v * d.cosT[iz * nz + k];
            im -= v * d.sinT[iz * nz + k];
        }
        X[(((size_t)k * 3 + c) * 2 + 0) * nr + m] = re;
        X[(((size_t)k * 3 + c) * 2 + 1) * nr + m] = im;
    }
}

// 8. o_c(m, iz) = (1/nz) sum_k (Re U cos - Im U sin)(2 pi iz k / nz)
__global__ void fd_idft_kernel(FastDiagDev d, const double* U, double* ox, double* oy, double* oz) {
    const int nr = d.nr, nz = d.nz;
    const long total = (long)nr * nz * 3;
    const double inv = 1.0 / nz;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        const int iz = (int)(t % nz);
        const int m = (int)((t / nz) % nr);
        const int c = (int)(t / ((long)nr * nz));
        double s = 0.0;
        for (int k = 0; k < nz; ++k) {
            s += U[(((size_t)k * 3 + c) * 2 + 0) * nr + m] * d.cosT[iz * nz + k] -
                 U[(((size_t)k * 3 + c) * 2 + 1) * nr + m] * d.sinT[iz * nz + k];
        }
        double* o = c == 0 ? ox : (c == 1 ? oy : oz);
        o[(size_t)m * nz + iz] = s * inv;
    }
}

// Shared operator on many vectors: Y[v] = A X[v] for vectors v of a strided
// set (vector v at X + vsel(v) * nr).  Tiled FP64 GEMM: a block computes 64
// rows x 16 vectors, K staged through shared memory in chunks of 32.
struct VecSel {
    int per_mode;  // vectors taken from each mode
    int first;     // first vector slot within the mode (slot = (c*2 + part))
    int slots;     // slots per mode in the source layout (6 for 3 components, 2 for one)
};

__device__ __forceinline__ size_t vec_off(const VecSel& s, int v, int nr) {
    const int k = v / s.per_mode, q = v % s.per_mode;
    return ((size_t)k * s.slots + s.first + q) * nr;
}

// Shared-operator products Y_v = A X_v of the solve split the inner dimension
// into FD_KSPLIT slices (fd_dmma_kernel, the FP64 tensor-core tile of
// dgemm.cuh); slice z of vector v sits at Ypart + (z * nvec + v) * nr and
// fd_sum_ksplit_kernel adds the slices in order (deterministic, no atomics).
#define FD_KSPLIT 4

// Y[sel(v)] = sum_z Ypart[z][v]  (slices added in order)
__global__ void fd_sum_ksplit_kernel(int nr, int nvec, int ks, const double* Ypart, double* Y, VecSel sy) {
    const long total = (long)nvec * nr;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        const int v = (int)(t / nr), r = (int)(t % nr);
        double s = 0.0;
        for (int z = 0; z < ks; ++z) s += Ypart[(size_t)z * total + t];
        Y[vec_off(sy, v, nr) + r] = s;
    }
}

// Per-mode dense matvec with NV right-hand sides, streaming B_k once:
// Y_k[v] = B_k X_k[v], or Y_k[v] = Ysub_k[v] - B_k X_k[v] when Ysub != 0.
// grid (row chunks, modes); X_k staged in shared memory; each warp streams
// 4 rows at a time (4 independent loads per column step) for memory-level
// parallelism.
#define FD_MV_THREADS 512
template <int NV>
__global__ void __launch_bounds__(FD_MV_THREADS) fd_mode_mv_kernel(int nr, const double* B, const double* X, double* Y,
                                                                  const double* Ysub, int rows_per_block) {
    extern __shared__ double xs[];  // NV * nr
    const int k = blockIdx.y;
    const double* Xk = X + (size_t)k * NV * nr;
    for (int e = threadIdx.x; e < NV * nr; e += blockDim.x) xs[e] = Xk[e];
    __syncthreads();
    const double* Bk = B + (size_t)k * nr * nr;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int r_begin = blockIdx.x * rows_per_block;
    const int r_end = min(nr, r_begin + rows_per_block);
    for (int r = r_begin + 4 * warp; r < r_end; r += 4 * nw) {
        double acc[4][NV];
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int v = 0; v < NV; ++v) acc[q][v] = 0.0;
        const double* row[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) row[q] = Bk + (size_t)min(r + q, nr - 1) * nr;
#pragma unroll 2
        for (int j = lane; j < nr; j += 32) {
            double b[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) b[q] = __ldg(row[q] + j);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                const double xv = xs[v * nr + j];
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[q][v] += b[q] * xv;
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int v = 0; v < NV; ++v) acc[q][v] = warp_sum(acc[q][v]);
        if (lane == 0) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (r + q >= r_end) continue;
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    const size_t o = ((size_t)k * NV + v) * nr + r + q;
                    Y[o] = Ysub ? Ysub[o] - acc[q][v] : acc[q][v];
                }
            }
        }
    }
}

// T = mu_k * (M2 X): scale the 6 vectors of each mode by mu_k (in place).
__global__ void fd_scale_mu_kernel(FastDiagDev d, double* T) {
    const long total = (long)d.nz * 6 * d.nr;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        const int k = (int)(t / (6L * d.nr));
        T[t] *= d.mu[k];
    }
}

// DIV_k (re, im) from Gx = Qx2 UTx, Gy = Qy2 UTy, Gz = M2 UTz (each [k][re/im][m]):
// re = mu (Gx_r + Gy_r) - kap Gz_i ; im = mu (Gx_i + Gy_i) + kap Gz_r
__global__ void fd_div_kernel(FastDiagDev d, const double* Gx, const double* Gy, const double* Gz, double* DIV) {
    const int nr = d.nr;
    const long total = (long)d.nz * nr;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        const int k = (int)(t / nr), m = (int)(t % nr);
        const size_t re = ((size_t)k * 2 + 0) * nr + m, im = ((size_t)k * 2 + 1) * nr + m;
        const double mu = d.mu[k], kap = d.kap[k];
        DIV[re] = mu * (Gx[re] + Gy[re]) - kap * Gz[im];
        DIV[im] = mu * (Gx[im] + Gy[im]) + kap * Gz[re];
    }
}

// G (6 vectors per mode) from Hx = Qx2^T P, Hy = Qy2^T P, Hz = M2 P:
// Gx = mu Hx, Gy = mu Hy, Gz = (kap Hz_i, -kap Hz_r)
__global__ void fd_grad_kernel(FastDiagDev d, const double* Hx, const double* Hy, const double* Hz, double* G) {
    const int nr = d.nr;
    const long total = (long)d.nz * nr;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        const int k = (int)(t / nr), m = (int)(t % nr);
        const size_t re = ((size_t)k * 2 + 0) * nr + m, im = ((size_t)k * 2 + 1) * nr + m;
        const double mu = d.mu[k], kap = d.kap[k];
        double* g = G + (size_t)k * 6 * nr;
        g[0 * nr + m] = mu * Hx[re];
        g[1 * nr + m] = mu * Hx[im];
        g[2 * nr + m] = mu * Hy[re];
        g[3 * nr + m] = mu * Hy[im];
        g[4 * nr + m] = kap * Hz[im];
        g[5 * nr + m] = -kap * Hz[re];
    }
}
