// Learned preconditioner: a patch-wise MLP (128 -> 64 -> 64 -> 64, ReLU) with
// BF16 weights and FP32 accumulation, its training kernels (forward /
// backward / Adam), and the flexible PCG that applies it after Jacobi.
//
// Features of one 4x4x4 DOF patch: u = D^{-1} r on the patch's 64 DOFs,
// s = ||u|| + 1e-300, input x = [u / s, gamma * u / s] (gamma = fluid-mass
// ratio of each DOF, 0 off the fluid).  The correction is
// z = D^{-1} r + s * (y(x) - y(-x)) / 2.
// Every reduced DOF belongs to exactly one patch, so z is written once.
#pragma once

#include "ops.cuh"

#define MLP_IN 128
#define MLP_H 64
#define MLP_OUT 64
#define MLP_PATCH 64
// FP32 parameter vector layout: W1[128][64], b1[64], W2[64][64], b2[64], W3[64][64], b3[64]
#define MLP_OFF_W1 0
#define MLP_OFF_B1 (MLP_IN * MLP_H)
#define MLP_OFF_W2 (MLP_OFF_B1 + MLP_H)
#define MLP_OFF_B2 (MLP_OFF_W2 + MLP_H * MLP_H)
#define MLP_OFF_W3 (MLP_OFF_B2 + MLP_H)
#define MLP_OFF_B3 (MLP_OFF_W3 + MLP_H * MLP_OUT)
#define MLP_NPARAM (MLP_OFF_B3 + MLP_OUT)
#define MLP_NW (MLP_IN * MLP_H + MLP_H * MLP_H + MLP_H * MLP_OUT)  // weights only

struct MlpWeights {
    const __nv_bfloat16* w;  // BF16 weights W1|W2|W3 (row-major [in][out])
    const float* theta;      // FP32 parameters (biases read from here)
    int act;                 // hidden activation: 0 ReLU, 1 identity (a linear network)
};

__device__ __forceinline__ float mlp_act(float v, int act) { return act ? v : fmaxf(v, 0.f); }
__device__ __forceinline__ float mlp_dact(float z, int act) { return act ? 1.f : (z > 0.f ? 1.f : 0.f); }

// Shared-memory image of the network: BF16 weights + FP32 biases.
struct MlpSmem {
    __nv_bfloat16* w;  // MLP_NW
    float* b;          // 3 * 64
    int act;
    __host__ __device__ static constexpr size_t bytes() { return MLP_NW * sizeof(__nv_bfloat16) + 3 * 64 * sizeof(float); }
};

__device__ __forceinline__ MlpSmem mlp_load_smem(const MlpWeights& W, char* base) {
    MlpSmem s;
    s.w = reinterpret_cast<__nv_bfloat16*>(base);
    s.b = reinterpret_cast<float*>(base + MLP_NW * sizeof(__nv_bfloat16));
    s.act = W.act;
    for (int k = threadIdx.x; k < MLP_NW; k += blockDim.x) s.w[k] = W.w[k];
    for (int k = threadIdx.x; k < 64; k += blockDim.x) {
        s.b[k] = W.theta[MLP_OFF_B1 + k];
        s.b[64 + k] = W.theta[MLP_OFF_B2 + k];
        s.b[128 + k] = W.theta[MLP_OFF_B3 + k];
    }
    return s;
}

// One sample per warp. x (128 floats) and h (2 x 64 floats) are the warp's
// shared scratch; on return y[0..63] (in h2 storage) holds the output, and
// z1/z2 (pre-activations) are written when non-null.  Lane l owns outputs l
// and l + 32 of every layer.
__device__ __forceinline__ void mlp_forward_warp(const MlpSmem& S, const float* x, float* h1, float* h2, float* y,
                                                 float* z1, float* z2) {
    const int l = threadIdx.x & 31;
    const __nv_bfloat16* W1 = S.w;
    const __nv_bfloat16* W2 = S.w + MLP_IN * MLP_H;
    const __nv_bfloat16* W3 = W2 + MLP_H * MLP_H;
    float a0 = S.b[l], a1 = S.b[l + 32];
#pragma unroll 8
    for (int i = 0; i < MLP_IN; ++i) {
        const float xi = x[i];
        a0 = fmaf(xi, __bfloat162float(W1[i * MLP_H + l]), a0);
        a1 = fmaf(xi, __bfloat162float(W1[i * MLP_H + l + 32]), a1);
    }
    if (z1) {
        z1[l] = a0;
        z1[l + 32] = a1;
    }
    h1[l] = mlp_act(a0, S.act);
    h1[l + 32] = mlp_act(a1, S.act);
    __syncwarp();
    a0 = S.b[64 + l];
    a1 = S.b[64 + l + 32];
#pragma unroll 8
    for (int i = 0; i < MLP_H; ++i) {
        const float hi = h1[i];
        a0 = fmaf(hi, __bfloat162float(W2[i * MLP_H + l]), a0);
        a1 = fmaf(hi, __bfloat162float(W2[i * MLP_H + l + 32]), a1);
    }
    if (z2) {
        z2[l] = a0;
        z2[l + 32] = a1;
    }
    h2[l] = mlp_act(a0, S.act);
    h2[l + 32] = mlp_act(a1, S.act);
    __syncwarp();
    a0 = S.b[128 + l];
    a1 = S.b[128 + l + 32];
#pragma unroll 8
    for (int i = 0; i < MLP_H; ++i) {
        const float hi = h2[i];
        a0 = fmaf(hi, __bfloat162float(W3[i * MLP_OUT + l]), a0);
        a1 = fmaf(hi, __bfloat162float(W3[i * MLP_OUT + l + 32]), a1);
    }
    __syncwarp();
    y[l] = a0;
    y[l + 32] = a1;
    __syncwarp();
}

// ---------------------------------------------------------------------------
// Training and batched inference on the BF16 tensor cores: mlp_tc.cuh.
// (mlp_forward_warp above, one sample per warp, serves the patch inference
// inside the flexible PCG, where each warp holds one patch.)
// ---------------------------------------------------------------------------

#include "mlp_tc.cuh"

// Adam step on the FP32 parameters and refresh of the BF16 weights.
__global__ void mlp_adam_kernel(float* theta, float* m, float* v, const float* grad, __nv_bfloat16* wbf, float lr,
                                float b1, float b2, float eps, float c1, float c2) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= MLP_NPARAM) return;
    const float g = grad[k];
    const float mk = b1 * m[k] + (1.f - b1) * g;
    const float vk = b2 * v[k] + (1.f - b2) * g * g;
    m[k] = mk;
    v[k] = vk;
    const float p = theta[k] - lr * (mk / c1) / (sqrtf(vk / c2) + eps);
    theta[k] = p;
    // W1 | b1 | W2 | b2 | W3 | b3  ->  W1 | W2 | W3 in the BF16 image
    int w = -1;
    if (k < MLP_OFF_B1) w = k;
    else if (k >= MLP_OFF_W2 && k < MLP_OFF_B2) w = MLP_IN * MLP_H + (k - MLP_OFF_W2);
    else if (k >= MLP_OFF_W3 && k < MLP_OFF_B3) w = MLP_IN * MLP_H + MLP_H * MLP_H + (k - MLP_OFF_W3);
    if (w >= 0) wbf[w] = __float2bfloat16(p);
}

__global__ void mlp_refresh_bf16_kernel(const float* theta, __nv_bfloat16* wbf) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= MLP_NPARAM) return;
    int w = -1;
    if (k < MLP_OFF_B1) w = k;
    else if (k >= MLP_OFF_W2 && k < MLP_OFF_B2) w = MLP_IN * MLP_H + (k - MLP_OFF_W2);
    else if (k >= MLP_OFF_W3 && k < MLP_OFF_B3) w = MLP_IN * MLP_H + MLP_H * MLP_H + (k - MLP_OFF_W3);
    if (w >= 0) wbf[w] = __float2bfloat16(theta[k]);
}

// ---------------------------------------------------------------------------
// Patch features from a reduced residual (dataset generation and tests).
// X[k] = [u/s, gamma], S[k] = s with u = dinv * r on the patch.
// ---------------------------------------------------------------------------
struct PatchMap {
    int n_patch;
    const int* red;      // [n_patch][64] reduced index or -1
    const float* gamma;  // [n_patch][64]
    const double* binv;  // optional exact patch inverses [n_blocks][64][64], symmetric
    const int* slot;     // optional [n_patch]: block of the patch in binv, or -1 (network / Jacobi)
};

__device__ __forceinline__ float patch_features_warp(const PatchMap& pm, int k, const double* r, const double* dinv,
                                                     float* x) {
    const int l = threadIdx.x & 31;
    double u0 = 0.0, u1 = 0.0;
    const int j0 = __ldg(pm.red + (size_t)k * 64 + l), j1 = __ldg(pm.red + (size_t)k * 64 + l + 32);
    if (j0 >= 0) u0 = __ldg(dinv + j0) * __ldcg(r + j0);
    if (j1 >= 0) u1 = __ldg(dinv + j1) * __ldcg(r + j1);
    double ss = u0 * u0 + u1 * u1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    const double s = sqrt(ss) + 1e-300;
    x[l] = (float)(u0 / s);
    x[l + 32] = (float)(u1 / s);
    x[64 + l] = __ldg(pm.gamma + (size_t)k * 64 + l) * (float)(u0 / s);
    x[64 + l + 32] = __ldg(pm.gamma + (size_t)k * 64 + l + 32) * (float)(u1 / s);
    __syncwarp();
    return (float)s;
}

__global__ void patch_features_kernel(PatchMap pm, const double* r, const double* dinv, float* X, float* Sc) {
    __shared__ float xs[8][MLP_IN];
    const int warp = threadIdx.x >> 5, l = threadIdx.x & 31;
    const int gw = blockIdx.x * (blockDim.x >> 5) + warp, nw = gridDim.x * (blockDim.x >> 5);
    for (int k = gw; k < pm.n_patch; k += nw) {
        const float s = patch_features_warp(pm, k, r, dinv, xs[warp]);
        for (int i = l; i < MLP_IN; i += 32) X[(size_t)k * MLP_IN + i] = xs[warp][i];
        if (l == 0) Sc[k] = s;
        __syncwarp();
    }
}

// Training targets: T[k][q] = (e_j - dinv_j r_j) / s_k on the patch DOFs.
__global__ void patch_targets_kernel(PatchMap pm, const double* e, const double* r, const double* dinv, const float* Sc,
                                     float* T) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < pm.n_patch * 64; t += gridDim.x * blockDim.x) {
        const int k = t >> 6;
        const int j = __ldg(pm.red + t);
        float v = 0.f;
        if (j >= 0) v = (float)((e[j] - dinv[j] * r[j]) / (double)Sc[k]);
        T[t] = v;
    }
}

// ---------------------------------------------------------------------------
// Flexible PCG with the patch preconditioner z = M(r): exact patch blocks
// where given, the network z = D^{-1} r + s * mlp(x) or Jacobi on the other
// patches (Polak-Ribiere beta).
// ---------------------------------------------------------------------------
// Patch preconditioner modes (LearnedArgs::use_mlp):
//   1: patches with an exact block use it, the others the network;
//   2: patches with an exact block use it, the others Jacobi (block Jacobi,
//      the method without the network).
struct LearnedArgs {
    MlpWeights W;
    PatchMap pm;
    double* z;      // [n] preconditioned residual
    double* rold;   // [n]
    int use_mlp;
    const double* ones;  // [n] ones: the fused p update p = 1 * z + beta p_old
};

// One patch of the fused residual / preconditioner phase, by one warp: the
// iterate and residual updates of the patch's DOFs (alpha = 0 at the start),
// then z_P = M_P(r_P), and this lane's shares of r.z, r.r and r_old.z.
template <bool kNet>
__device__ __forceinline__ void patch_step(const LearnedArgs& L, const PcgBufs& B, int k, double alpha,
                                           const double* pk, double* x, const MlpSmem& S, float* xs, double& rz,
                                           double& rr, double& roz) {
    const int l = threadIdx.x & 31;
    const int j0 = __ldg(L.pm.red + (size_t)k * 64 + l), j1 = __ldg(L.pm.red + (size_t)k * 64 + l + 32);
    double ro0 = 0.0, ro1 = 0.0, r0 = 0.0, r1 = 0.0;
    if (j0 >= 0) {
        ro0 = B.r[j0];
        r0 = ro0;
        if (alpha != 0.0) {
            x[j0] += alpha * __ldcg(pk + j0);
            r0 = ro0 - alpha * __ldcg(B.Ap + j0);
            B.r[j0] = r0;
        }
    }
    if (j1 >= 0) {
        ro1 = B.r[j1];
        r1 = ro1;
        if (alpha != 0.0) {
            x[j1] += alpha * __ldcg(pk + j1);
            r1 = ro1 - alpha * __ldcg(B.Ap + j1);
            B.r[j1] = r1;
        }
    }
    const int slot = (L.pm.binv && L.pm.slot) ? __ldg(L.pm.slot + k) : -1;
    double z0, z1;
    if (slot >= 0) {  // exact block solve, columns read coalesced (the inverse is symmetric)
        const double* Bk = L.pm.binv + (size_t)slot * 4096;
        z0 = 0.0;
        z1 = 0.0;
#pragma unroll 8
        for (int q = 0; q < 64; ++q) {
            const double rq = __shfl_sync(0xffffffffu, q < 32 ? r0 : r1, q & 31);
            z0 += __ldg(Bk + q * 64 + l) * rq;
            z1 += __ldg(Bk + q * 64 + l + 32) * rq;
        }
    } else {
        z0 = j0 >= 0 ? B.dinv[j0] * r0 : 0.0;
        z1 = j1 >= 0 ? B.dinv[j1] * r1 : 0.0;
        if constexpr (kNet) {
            // network correction z += s (mlp(x) - mlp(-x)) / 2 from the features
            // of the updated residual (the warp's own writes, ordered by syncwarp)
            __syncwarp();
            float* h1 = xs + MLP_IN;
            float* h2 = h1 + 64;
            float* y = h2 + 64;
            const float s = patch_features_warp(L.pm, k, B.r, B.dinv, xs);
            mlp_forward_warp(S, xs, h1, h2, y, nullptr, nullptr);
            const float yp0 = y[l], yp1 = y[l + 32];
            __syncwarp();
            xs[l] = -xs[l];
            xs[l + 32] = -xs[l + 32];
            xs[64 + l] = -xs[64 + l];
            xs[64 + l + 32] = -xs[64 + l + 32];
            __syncwarp();
            mlp_forward_warp(S, xs, h1, h2, y, nullptr, nullptr);
            z0 += (double)s * (double)(0.5f * (yp0 - y[l]));
            z1 += (double)s * (double)(0.5f * (yp1 - y[l + 32]));
            __syncwarp();
        }
    }
    if (j0 >= 0) {
        L.z[j0] = z0;
        rz += r0 * z0;
        rr += r0 * r0;
        roz += ro0 * z0;
    }
    if (j1 >= 0) {
        L.z[j1] = z1;
        rz += r1 * z1;
        rr += r1 * r1;
        roz += ro1 * z1;
    }
}

// Patch-preconditioned flexible PCG (Polak-Ribiere beta) with the operator's
// fused p update: per iteration
//   apply:  p = z + beta p_old (phase 0 of the operator, z in place of D^-1 r
//           and ones as the scale), A p, p.A p        (the operator's barriers)
//   barrier, alpha = r.z / p.A p
//   patch phase (one warp per patch): x += alpha p, r -= alpha A p,
//           z = M(r) on the patch, partials of r.z, r.r, r_old.z
//   barrier, rel = ||r|| / ||b||, beta = (r.z - r_old.z) / r.z_old
// so an iteration takes the barriers of plain PCG.  Every reduced DOF lies in
// exactly one patch.
template <class Op, bool kNet>
__global__ void __launch_bounds__(CUTCELL_BLOCK, 2) ppcg_kernel(Op op, SolveArgs a, LearnedArgs L, size_t op_smem) {
    static_assert(Op::kFusedP, "the patch PCG forms p inside the operator's first phase");
    extern __shared__ __align__(16) double sm[];
    __shared__ double sh[CUTCELL_WARPS + 1];
    char* smem_mlp = reinterpret_cast<char*>(sm) + op_smem;
    float* scratch = reinterpret_cast<float*>(smem_mlp + MlpSmem::bytes());
    const PcgBufs& B = a.B;
    const int n = B.n, nb = gridDim.x;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gstride = gridDim.x * blockDim.x;
    const int warp = threadIdx.x >> 5;
    const int gw = blockIdx.x * (blockDim.x >> 5) + warp, nw = gridDim.x * (blockDim.x >> 5);
    float* xs = scratch + warp * (MLP_IN + 3 * 64);
    double* part = B.part;
    const GridSync& gs = a.gs;
    MlpSmem S;
    if constexpr (kNet) S = mlp_load_smem(L.W, smem_mlp);
    // x = 0, r = b, ||b||
    double bb = 0.0;
    for (int i = gtid; i < n; i += gstride) {
        a.x[i] = 0.0;
        B.r[i] = a.b[i];
        bb += a.b[i] * a.b[i];
    }
    bb = block_sum(bb, sh);
    if (threadIdx.x == 0) part[1 * nb + blockIdx.x] = bb;
    int status = CUTCELL_E_NOCONV, k = 0;
    double rel = 1.0;
    if (!grid_sync(gs)) status = CUTCELL_E_BARRIER;
    double bnorm = sqrt(grid_reduce(part + 1 * nb, nb, sh));
    if (bnorm == 0.0) bnorm = 1.0;
    // z = M(b), p = z, rz
    double rz = 0.0, rr = 0.0, roz = 0.0;
    for (int q = gw; q < L.pm.n_patch; q += nw) patch_step<kNet>(L, B, q, 0.0, B.p, a.x, S, xs, rz, rr, roz);
    rz = block_sum(rz, sh);
    if (threadIdx.x == 0) part[0 * nb + blockIdx.x] = rz;
    if (!grid_sync(gs)) status = CUTCELL_E_BARRIER;
    rz = grid_reduce(part + 0 * nb, nb, sh);
    for (int i = gtid; i < n; i += gstride) B.p[i] = __ldcg(L.z + i);
    if (!grid_sync(gs)) status = CUTCELL_E_BARRIER;
    double* P[2] = {B.p, B.p2};
    double beta = 0.0;
    for (k = 1; k <= a.maxiter && status != CUTCELL_E_BARRIER; ++k) {
        double* pk = P[(k - 1) & 1];
        double pap = (k > 1) ? op.apply_next(P[k & 1], pk, L.z, L.ones, beta, B.Ap, gs, sm) : op.apply(pk, B.Ap, gs, sm);
        if (grid_error(gs)) {
            status = CUTCELL_E_BARRIER;
            break;
        }
        pap = block_sum(pap, sh);
        if (threadIdx.x == 0) part[2 * nb + blockIdx.x] = pap;
        if (!grid_sync(gs)) {
            status = CUTCELL_E_BARRIER;
            break;
        }
        pap = grid_reduce(part + 2 * nb, nb, sh);
        if (!(pap > 0.0) || !isfinite(pap)) {
            status = CUTCELL_E_BREAKDOWN;
            break;
        }
        const double alpha = rz / pap;
        double d0 = 0.0, d1 = 0.0, d2 = 0.0;
        for (int q = gw; q < L.pm.n_patch; q += nw) patch_step<kNet>(L, B, q, alpha, pk, a.x, S, xs, d0, d1, d2);
        d0 = block_sum(d0, sh);
        d1 = block_sum(d1, sh);
        d2 = block_sum(d2, sh);
        if (threadIdx.x == 0) {
            part[3 * nb + blockIdx.x] = d0;
            part[4 * nb + blockIdx.x] = d1;
            part[5 * nb + blockIdx.x] = d2;
        }
        if (!grid_sync(gs)) {
            status = CUTCELL_E_BARRIER;
            break;
        }
        const double rzn = grid_reduce(part + 3 * nb, nb, sh);
        rel = sqrt(grid_reduce(part + 4 * nb, nb, sh)) / bnorm;
        const double roz_n = grid_reduce(part + 5 * nb, nb, sh);
        if (!isfinite(rel)) {
            status = CUTCELL_E_NAN;
            break;
        }
        if (rel <= a.tol) {
            status = CUTCELL_OK;
            break;
        }
        beta = (rzn - roz_n) / rz;
        rz = rzn;
    }
    const int iters = k > a.maxiter ? a.maxiter : k;
    double true_rel = -1.0;
    if (status != CUTCELL_E_BARRIER && !grid_error(gs))
        true_rel = true_residual(op, B, a.b, a.x, bnorm, gs, sm, sh, nullptr);
    if (grid_error(gs)) status = CUTCELL_E_BARRIER;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.res->status = status;
        a.res->iterations = iters;
        a.res->outer = 1;
        a.res->rel = rel;
        a.res->true_rel = true_rel;
    }
}

