// Tensor-core kernels of the patch network (128 -> 64 -> 64 -> 64): batched
// forward, forward + backward, and the weight gradients, on the BF16 tensor
// cores (mma.sync.m16n8k16, FP32 accumulation).
//
// Weights are BF16 (the network's storage).  Activations, deltas and inputs
// are FP32: each operand that is not a weight is split into two BF16 planes,
// v = hi + lo with hi = bf16(v), lo = bf16(v - hi), and multiplied as
// hi * W + lo * W (weight products) or hi * g_hi + hi * g_lo + lo * g_hi
// (gradient products of two FP32 operands), so the products carry about 16
// bits of each FP32 operand.  Every sum runs in a fixed order, so results are
// bit-reproducible.
//
// Fragment layouts of m16n8k16 (g = lane / 4, t = lane % 4):
//   A (16 x 16, row): reg q holds row g + 8 (q & 1), columns k0 + 2t + 8 (q >> 1) and + 1
//   B (16 x 8, col):  reg q holds rows (k) 2t + 8 q and + 1 of column (n) g
//   C (16 x 8):       c0, c1 row g, columns 2t, 2t + 1; c2, c3 row g + 8
// A pair of BF16 values sits in one 32-bit register, the lower index in the
// low half.
#pragma once

#include <cuda_bf16.h>

#define MLPT_WARPS 4
#define MLPT_LD128 136  // padded FP32 / BF16 row of a 128-wide tile (conflict-free fragment access)
#define MLPT_LD64 72    // padded row of a 64-wide tile

__device__ __forceinline__ void mma_bf16(float (&d)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ unsigned bf16_pair(__nv_bfloat16 lo_idx, __nv_bfloat16 hi_idx) {
    return (unsigned)__bfloat16_as_ushort(lo_idx) | ((unsigned)__bfloat16_as_ushort(hi_idx) << 16);
}

// two-plane split of a pair of FP32 values into (hi pair, lo pair)
__device__ __forceinline__ void split_pair(float v0, float v1, unsigned& hi, unsigned& lo) {
    const __nv_bfloat16 h0 = __float2bfloat16_rn(v0), h1 = __float2bfloat16_rn(v1);
    hi = bf16_pair(h0, h1);
    lo = bf16_pair(__float2bfloat16_rn(v0 - __bfloat162float(h0)), __float2bfloat16_rn(v1 - __bfloat162float(h1)));
}

// A fragments (both planes) of the 16-row FP32 tile S (row stride ld) at
// columns k0..k0+15; act >= 0 applies the hidden activation on load.
__device__ __forceinline__ void tc_load_a(const float* S, int ld, int k0, int act, unsigned (&ah)[4], unsigned (&al)[4]) {
    const int l = threadIdx.x & 31, g = l >> 2, t = l & 3;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float2 v = *reinterpret_cast<const float2*>(S + (g + 8 * (q & 1)) * ld + k0 + 2 * t + 8 * (q >> 1));
        float v0 = v.x, v1 = v.y;
        if (act >= 0) {
            v0 = mlp_act(v0, act);
            v1 = mlp_act(v1, act);
        }
        split_pair(v0, v1, ah[q], al[q]);
    }
}

// acc[j] (16 x 8, columns 8 j ..) = bias + A (16 x K, FP32 smem) W (K x 64),
// W given n-major in shared memory (Wn[n * ldw + k], BF16).
template <int K>
__device__ __forceinline__ void tc_layer(const float* A, int lda, int act_a, const __nv_bfloat16* Wn, int ldw,
                                         const float* bias, float (&acc)[8][4]) {
    const int l = threadIdx.x & 31, g = l >> 2, t = l & 3;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const float b0 = bias ? bias[8 * j + 2 * t] : 0.f, b1 = bias ? bias[8 * j + 2 * t + 1] : 0.f;
        acc[j][0] = b0;
        acc[j][1] = b1;
        acc[j][2] = b0;
        acc[j][3] = b1;
    }
#pragma unroll
    for (int k0 = 0; k0 < K; k0 += 16) {
        unsigned ah[4], al[4];
        tc_load_a(A, lda, k0, act_a, ah, al);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const __nv_bfloat16* w = Wn + (8 * j + g) * ldw + k0 + 2 * t;
            const unsigned b[2] = {*reinterpret_cast<const unsigned*>(w), *reinterpret_cast<const unsigned*>(w + 8)};
            mma_bf16(acc[j], ah, b);
            mma_bf16(acc[j], al, b);
        }
    }
}

// store a 16 x 64 accumulator tile into FP32 shared memory (row stride ld)
__device__ __forceinline__ void tc_store(float* O, int ld, const float (&acc)[8][4]) {
    const int l = threadIdx.x & 31, g = l >> 2, t = l & 3;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        *reinterpret_cast<float2*>(O + g * ld + 8 * j + 2 * t) = make_float2(acc[j][0], acc[j][1]);
        *reinterpret_cast<float2*>(O + (g + 8) * ld + 8 * j + 2 * t) = make_float2(acc[j][2], acc[j][3]);
    }
}

// Shared-memory image for the tile kernels: the three weight matrices n-major
// (forward operands), W2 and W3 as stored ([in][out], the backward operands),
// the biases, then MLPT_WARPS per-warp work tiles.
struct MlpTcSmem {
    __nv_bfloat16 *w1n, *w2n, *w3n, *w2r, *w3r;
    float* b;
    float* warp_base;
    __host__ __device__ static constexpr size_t weights_bytes() {
        return sizeof(__nv_bfloat16) * (size_t)(64 * MLPT_LD128 + 4 * 64 * MLPT_LD64) + 3 * 64 * sizeof(float);
    }
    // per warp: X (16 x 136), Z1, Z2, D (16 x 72 each), FP32
    __host__ __device__ static constexpr size_t warp_floats() { return 16 * MLPT_LD128 + 3 * 16 * MLPT_LD64; }
    __host__ __device__ static constexpr size_t bytes() { return weights_bytes() + MLPT_WARPS * warp_floats() * sizeof(float); }
};

__device__ __forceinline__ MlpTcSmem mlp_tc_load(const MlpWeights& W, char* base) {
    MlpTcSmem s;
    s.w1n = reinterpret_cast<__nv_bfloat16*>(base);
    s.w2n = s.w1n + 64 * MLPT_LD128;
    s.w3n = s.w2n + 64 * MLPT_LD64;
    s.w2r = s.w3n + 64 * MLPT_LD64;
    s.w3r = s.w2r + 64 * MLPT_LD64;
    s.b = reinterpret_cast<float*>(s.w3r + 64 * MLPT_LD64);
    s.warp_base = s.b + 3 * 64;
    const __nv_bfloat16* W1 = W.w;
    const __nv_bfloat16* W2 = W1 + MLP_IN * MLP_H;
    const __nv_bfloat16* W3 = W2 + MLP_H * MLP_H;
    for (int e = threadIdx.x; e < MLP_IN * MLP_H; e += blockDim.x) {  // W1[i][o] -> w1n[o][i]
        const int i = e / MLP_H, o = e % MLP_H;
        s.w1n[o * MLPT_LD128 + i] = W1[e];
    }
    for (int e = threadIdx.x; e < MLP_H * MLP_H; e += blockDim.x) {
        const int i = e / MLP_H, o = e % MLP_H;
        s.w2n[o * MLPT_LD64 + i] = W2[e];
        s.w3n[o * MLPT_LD64 + i] = W3[e];
        s.w2r[i * MLPT_LD64 + o] = W2[e];
        s.w3r[i * MLPT_LD64 + o] = W3[e];
    }
    for (int k = threadIdx.x; k < 64; k += blockDim.x) {
        s.b[k] = W.theta[MLP_OFF_B1 + k];
        s.b[64 + k] = W.theta[MLP_OFF_B2 + k];
        s.b[128 + k] = W.theta[MLP_OFF_B3 + k];
    }
    return s;
}

// rows r0 .. r0 + 15 of X (zero beyond batch) into the warp's X tile
__device__ __forceinline__ void tc_load_rows(const float* X, int batch, int r0, float* Xs) {
    const int l = threadIdx.x & 31;
    for (int e = l; e < 16 * MLP_IN; e += 32) {
        const int r = e / MLP_IN, c = e % MLP_IN;
        Xs[r * MLPT_LD128 + c] = (r0 + r < batch) ? X[(size_t)(r0 + r) * MLP_IN + c] : 0.f;
    }
    __syncwarp();
}

// Forward of the warp's 16-row tile: Z1, Z2 (pre-activations) in shared
// memory, the output in acc.
__device__ __forceinline__ void tc_forward(const MlpTcSmem& S, int act, const float* Xs, float* Z1, float* Z2,
                                           float (&acc)[8][4]) {
    tc_layer<MLP_IN>(Xs, MLPT_LD128, -1, S.w1n, MLPT_LD128, S.b, acc);
    tc_store(Z1, MLPT_LD64, acc);
    __syncwarp();
    tc_layer<MLP_H>(Z1, MLPT_LD64, act, S.w2n, MLPT_LD64, S.b + 64, acc);
    tc_store(Z2, MLPT_LD64, acc);
    __syncwarp();
    tc_layer<MLP_H>(Z2, MLPT_LD64, act, S.w3n, MLPT_LD64, S.b + 128, acc);
}

// Batched inference, one 16-sample tile per warp.
__global__ void __launch_bounds__(MLPT_WARPS * 32) mlp_forward_tc_kernel(MlpWeights W, const float* X, int batch, float* Y) {
    extern __shared__ __align__(16) char smem[];
    const MlpTcSmem S = mlp_tc_load(W, smem);
    __syncthreads();
    const int warp = threadIdx.x >> 5, l = threadIdx.x & 31, g = l >> 2, t = l & 3;
    float* Xs = S.warp_base + warp * MlpTcSmem::warp_floats();
    float* Z1 = Xs + 16 * MLPT_LD128;
    float* Z2 = Z1 + 16 * MLPT_LD64;
    const int ntile = (batch + 15) / 16;
    for (int tile = blockIdx.x * MLPT_WARPS + warp; tile < ntile; tile += gridDim.x * MLPT_WARPS) {
        const int r0 = 16 * tile;
        tc_load_rows(X, batch, r0, Xs);
        float acc[8][4];
        tc_forward(S, W.act, Xs, Z1, Z2, acc);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int c = 8 * j + 2 * t;
            if (r0 + g < batch) *reinterpret_cast<float2*>(Y + (size_t)(r0 + g) * MLP_OUT + c) = make_float2(acc[j][0], acc[j][1]);
            if (r0 + g + 8 < batch)
                *reinterpret_cast<float2*>(Y + (size_t)(r0 + g + 8) * MLP_OUT + c) = make_float2(acc[j][2], acc[j][3]);
        }
        __syncwarp();
    }
}

// Forward + backward of one 16-sample tile per warp (mean-squared loss over
// batch x 64 outputs): writes Y, DY = dL/dy, H2 = act(z2), D2 = dL/dz2,
// H1 = act(z1), D1 = dL/dz1 and the per-sample squared error, for the
// weight-gradient kernel.
__global__ void __launch_bounds__(MLPT_WARPS * 32) mlp_fwd_bwd_tc_kernel(MlpWeights W, const float* X, const float* Tgt,
                                                                    int batch, float* H1, float* H2, float* D1,
                                                                    float* D2, float* DY, float* Y, float* sample_loss) {
    extern __shared__ __align__(16) char smem[];
    const MlpTcSmem S = mlp_tc_load(W, smem);
    __syncthreads();
    const int warp = threadIdx.x >> 5, l = threadIdx.x & 31, g = l >> 2, t = l & 3;
    float* Xs = S.warp_base + warp * MlpTcSmem::warp_floats();
    float* Z1 = Xs + 16 * MLPT_LD128;
    float* Z2 = Z1 + 16 * MLPT_LD64;
    float* Ds = Z2 + 16 * MLPT_LD64;
    const float scale = 2.0f / (float)((long)batch * MLP_OUT);
    const int act = W.act;
    const int ntile = (batch + 15) / 16;
    for (int tile = blockIdx.x * MLPT_WARPS + warp; tile < ntile; tile += gridDim.x * MLPT_WARPS) {
        const int r0 = 16 * tile;
        const bool in0 = r0 + g < batch, in1 = r0 + g + 8 < batch;
        tc_load_rows(X, batch, r0, Xs);
        float acc[8][4];
        tc_forward(S, act, Xs, Z1, Z2, acc);
        // dy = scale (y - t); rows past the batch carry zero deltas
        float l0 = 0.f, l1 = 0.f;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int c = 8 * j + 2 * t;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const float e0 = in0 ? acc[j][h] - Tgt[(size_t)(r0 + g) * MLP_OUT + c + h] : 0.f;
                const float e1 = in1 ? acc[j][2 + h] - Tgt[(size_t)(r0 + g + 8) * MLP_OUT + c + h] : 0.f;
                l0 += e0 * e0;
                l1 += e1 * e1;
                Ds[g * MLPT_LD64 + c + h] = scale * e0;
                Ds[(g + 8) * MLPT_LD64 + c + h] = scale * e1;
                if (in0) {
                    Y[(size_t)(r0 + g) * MLP_OUT + c + h] = acc[j][h];
                    DY[(size_t)(r0 + g) * MLP_OUT + c + h] = scale * e0;
                }
                if (in1) {
                    Y[(size_t)(r0 + g + 8) * MLP_OUT + c + h] = acc[j][2 + h];
                    DY[(size_t)(r0 + g + 8) * MLP_OUT + c + h] = scale * e1;
                }
            }
        }
        l0 += __shfl_xor_sync(0xffffffffu, l0, 1);
        l0 += __shfl_xor_sync(0xffffffffu, l0, 2);
        l1 += __shfl_xor_sync(0xffffffffu, l1, 1);
        l1 += __shfl_xor_sync(0xffffffffu, l1, 2);
        if (t == 0) {
            if (in0) sample_loss[r0 + g] = l0;
            if (in1) sample_loss[r0 + g + 8] = l1;
        }
        __syncwarp();
        // dz2 = (dy W3^T) * act'(z2): B[k = o][n = h] = W3[h][o], the stored row-major W3
        tc_layer<MLP_OUT>(Ds, MLPT_LD64, -1, S.w3r, MLPT_LD64, nullptr, acc);
        __syncwarp();  // every lane has read dy before it is overwritten
#pragma unroll
        for (int j = 0; j < 8; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int r = g + 8 * (q >> 1), c = 8 * j + 2 * t + (q & 1);
                acc[j][q] *= mlp_dact(Z2[r * MLPT_LD64 + c], act);
            }
        tc_store(Ds, MLPT_LD64, acc);
        __syncwarp();
        for (int e = l; e < 16 * 64; e += 32) {
            const int r = e / 64, c = e % 64;
            if (r0 + r < batch) {
                D2[(size_t)(r0 + r) * 64 + c] = Ds[r * MLPT_LD64 + c];
                H2[(size_t)(r0 + r) * 64 + c] = mlp_act(Z2[r * MLPT_LD64 + c], act);
            }
        }
        // dz1 = (dz2 W2^T) * act'(z1)
        tc_layer<MLP_H>(Ds, MLPT_LD64, -1, S.w2r, MLPT_LD64, nullptr, acc);
        __syncwarp();
#pragma unroll
        for (int j = 0; j < 8; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int r = g + 8 * (q >> 1), c = 8 * j + 2 * t + (q & 1);
                acc[j][q] *= mlp_dact(Z1[r * MLPT_LD64 + c], act);
            }
        tc_store(Ds, MLPT_LD64, acc);
        __syncwarp();
        for (int e = l; e < 16 * 64; e += 32) {
            const int r = e / 64, c = e % 64;
            if (r0 + r < batch) {
                D1[(size_t)(r0 + r) * 64 + c] = Ds[r * MLPT_LD64 + c];
                H1[(size_t)(r0 + r) * 64 + c] = mlp_act(Z1[r * MLPT_LD64 + c], act);
            }
        }
        __syncwarp();
    }
}

// Weight gradients dW = A^T G summed over the batch in order (A = X, H1, H2;
// G = D1, D2, DY), one warp per 16-row slice of a weight matrix: 8 slices of
// W1 and 4 each of W2 and W3.  The batch is contracted 16 samples per MMA step;
// both operands are FP32 and are split into two planes (hi g_hi + hi g_lo +
// lo g_hi).
__global__ void __launch_bounds__(128) mlp_wgrad_tc_kernel(const float* X, const float* H1, const float* H2,
                                                           const float* D1, const float* D2, const float* DY, int batch,
                                                           float* grad) {
    const int w = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (w >= 16) return;
    const int l = threadIdx.x & 31, g = l >> 2, t = l & 3;
    const float* A;
    const float* G;
    int lda, m0, off;
    if (w < 8) {
        A = X; lda = MLP_IN; G = D1; m0 = 16 * w; off = MLP_OFF_W1;
    } else if (w < 12) {
        A = H1; lda = 64; G = D2; m0 = 16 * (w - 8); off = MLP_OFF_W2;
    } else {
        A = H2; lda = 64; G = DY; m0 = 16 * (w - 12); off = MLP_OFF_W3;
    }
    float acc[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
    auto at = [&](const float* M, int ld, int b, int c) { return b < batch ? M[(size_t)b * ld + c] : 0.f; };
    for (int b0 = 0; b0 < batch; b0 += 16) {
        // A^T fragment: element (m, k) = A[b0 + k][m0 + m]
        unsigned ah[4], al[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int m = m0 + g + 8 * (q & 1), k = b0 + 2 * t + 8 * (q >> 1);
            split_pair(at(A, lda, k, m), at(A, lda, k + 1, m), ah[q], al[q]);
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            // G fragment: element (k, n) = G[b0 + k][8 j + n]
            unsigned bh[2], bl[2];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int k = b0 + 2 * t + 8 * q, n = 8 * j + g;
                split_pair(at(G, 64, k, n), at(G, 64, k + 1, n), bh[q], bl[q]);
            }
            mma_bf16(acc[j], ah, bh);
            mma_bf16(acc[j], ah, bl);
            mma_bf16(acc[j], al, bh);
        }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int c = 8 * j + 2 * t;
        grad[off + (m0 + g) * 64 + c] = acc[j][0];
        grad[off + (m0 + g) * 64 + c + 1] = acc[j][1];
        grad[off + (m0 + g + 8) * 64 + c] = acc[j][2];
        grad[off + (m0 + g + 8) * 64 + c + 1] = acc[j][3];
    }
}

// Bias gradients: column sums of D1, D2, DY over the batch in order.
__global__ void mlp_bgrad_kernel(const float* D1, const float* D2, const float* DY, int batch, float* grad) {
    const int k = threadIdx.x;
    if (k >= 192) return;
    const float* G = k < 64 ? D1 : (k < 128 ? D2 : DY);
    const int o = k % 64;
    const int off = k < 64 ? MLP_OFF_B1 : (k < 128 ? MLP_OFF_B2 : MLP_OFF_B3);
    float s = 0.f;
    for (int b = 0; b < batch; ++b) s += G[(size_t)b * 64 + o];
    grad[off + o] = s;
}
