// Batched FP64 "NT" GEMM on the FP64 tensor cores (mma.sync.m8n8k4.f64):
//
//   C_b = A_b diag(s_b) B_b^T  (+ beta C_b),   b = blockIdx.z
//
// A_b is M x K and B_b is N x K, both row-major (leading dimensions lda, ldb),
// s_b an optional K-vector folded into the A tile as it is staged; a zero
// batch stride shares an operand across the batch.  This is the dense work of
// the periodic-hill fast-diagonalisation build through a shared generalised
// eigenbasis (A_k^{-1} = Phi diag(d_k) Phi^T, S_k = G diag(w_k) G^T with
// G = [Qx2 Phi | Qy2 Phi | M2 Phi]), and of the shared-operator products of
// the solve.
//
// Tiling: a 256-thread block computes a 64 x 64 tile of C; its 8 warps are
// arranged 2 (M) x 4 (N), each owning 32 x 16 = 4 x 2 mma tiles of 8 x 8.  K is
// staged in chunks of 16 through shared memory as it lies in global memory
// (row m, k contiguous), rows padded to 20 doubles: a half-warp's staging
// store (16 consecutive k of one row) and a half-warp's fragment read (lane
// 4g + t reads row g, column k0 + t, g < 4) then fall in 16 distinct 8-byte
// bank pairs.  The next chunk is loaded into registers while the current one
// is multiplied.
#pragma once

#include "common.cuh"

#define DG_BM 64
#define DG_BN 64
#define DG_BK 16
#define DG_KS (DG_BK + 4)  // padded row of a staged chunk

struct DgemmArgs {
    int M, N, K;
    const double* A;
    long long lda, sA;
    const double* B;
    long long ldb, sB;
    const double* s;  // optional
    long long sS;
    double beta;
    double* C;
    long long ldc, sC;
};

__device__ __forceinline__ void dg_mma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// One 64 x 64 tile of C = A B^T over k in [kb, ke) by a 256-thread block:
// a(m, k) and b(n, k) return the operand entries (callers return 0 outside
// their ranges), store(m, n, v) receives every entry of the tile inside M x N.
template <class AL, class BL, class CS>
__device__ __forceinline__ void dmma_tile(int M, int N, int kb, int ke, int m0, int n0, const AL& a, const BL& b,
                                          const CS& store) {
    __shared__ double As[DG_BM][DG_KS];
    __shared__ double Bs[DG_BN][DG_KS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gq = lane >> 2, t4 = lane & 3;
    const int wm = (warp >> 2) * 32, wn = (warp & 3) * 16;
    double acc[4][2][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    // staging: 64 x 16 entries of each operand, 4 per thread; thread e loads
    // row e / 16, column e % 16 (consecutive threads, consecutive k)
    double ra[4], rb[4];
    auto load = [&](int k0) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = threadIdx.x + 256 * u;
            const int r = e >> 4, c = e & 15;
            const int k = k0 + c;
            const bool kin = k < ke;
            ra[u] = (kin && m0 + r < M) ? a(m0 + r, k) : 0.0;
            rb[u] = (kin && n0 + r < N) ? b(n0 + r, k) : 0.0;
        }
    };
    load(kb);
    for (int k0 = kb; k0 < ke; k0 += DG_BK) {
        __syncthreads();  // the previous chunk's fragments have been read
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = threadIdx.x + 256 * u;
            const int r = e >> 4, c = e & 15;
            As[r][c] = ra[u];
            Bs[r][c] = rb[u];
        }
        __syncthreads();
        if (k0 + DG_BK < ke) load(k0 + DG_BK);  // next chunk in flight during the products
#pragma unroll
        for (int ks = 0; ks < DG_BK; ks += 4) {
            double af[4], bf[2];
#pragma unroll
            for (int i = 0; i < 4; ++i) af[i] = As[wm + 8 * i + gq][ks + t4];
#pragma unroll
            for (int j = 0; j < 2; ++j) bf[j] = Bs[wn + 8 * j + gq][ks + t4];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) dg_mma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
        }
    }
    // C fragment of lane 4g + t: rows g, columns 2t and 2t + 1 of each 8 x 8 tile
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int m = m0 + wm + 8 * i + gq;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int n = n0 + wn + 8 * j + 2 * t4 + h;
                if (n < N) store(m, n, acc[i][j][h]);
            }
        }
    }
}

static __global__ void __launch_bounds__(256) dgemm_nt_kernel(DgemmArgs g) {
    const int bz = blockIdx.z;
    const double* A = g.A + (size_t)bz * g.sA;
    const double* B = g.B + (size_t)bz * g.sB;
    const double* S = g.s ? g.s + (size_t)bz * g.sS : nullptr;
    double* C = g.C + (size_t)bz * g.sC;
    const long long lda = g.lda, ldb = g.ldb, ldc = g.ldc;
    const double beta = g.beta;
    dmma_tile(
        g.M, g.N, 0, g.K, blockIdx.y * DG_BM, blockIdx.x * DG_BN,
        [&](int m, int k) { return S ? __ldg(A + (size_t)m * lda + k) * __ldg(S + k) : __ldg(A + (size_t)m * lda + k); },
        [&](int n, int k) { return __ldg(B + (size_t)n * ldb + k); },
        [&](int m, int n, double v) {
            double* cp = C + (size_t)m * ldc + n;
            *cp = (beta != 0.0 ? beta * *cp : 0.0) + v;
        });
}
