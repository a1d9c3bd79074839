// Periodic-hill advection and fast step on the device:
//   hill_skew_conv (cpp/include/cut/hill3d.h:519-538) for the three velocity
//   components at once, and hill_fastdiag_step (cpp/include/cut/hill_fastdiag.h:
//   83-95): SSP-RK3 of -skew_conv, + dt fx on u_x, then the fast-diagonalisation
//   solve (cutcell_fastdiag_solve).
//
// The reference samples every field to the (n2q x nzq) quadrature grid,
// forms the products there and loads them back, materialising a dozen
// quadrature-grid arrays per stage (hill3d.h:245-312).  Here one warp owns a
// segment of consecutive 2D quadrature points that share one sparse row
// pattern (the reduced modes a 2D cell touches) and does, per point, without
// leaving the SM:
//   (a) 2D sample: lanes = z modes, T[9][iz] = (phi, dphi/dx, dphi/dy) rows
//       times the staged coefficient rows of u_x, u_y, u_z;
//   (b) z expand, products, z contract: lanes = z elements; each element's
//       (p+6) z points see p+1 basis functions (a periodic band), so every
//       value, gradient and weak-form integrand is a 4-term sum in registers;
//   (c) band scatter of the per-element integrals to z modes in p+1 conflict-
//       free rounds (element e writes mode (e - s + j) mod nz in round j);
//   (d) 2D load: lanes = z modes, accumulate w2 (phi P + dpx X + dpy Y) into
//       the segment's per-mode accumulators (registers).
// Segment partials are summed per reduced mode in a fixed order (no atomics,
// bit-reproducible), then the separable mass solve applies Mz^-1 per mode and
// M2^-1 by a split-K FP64 GEMM.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "dgemm.cuh"

void cutcell_internal_set_error(const std::string& what);

#define HILL_WARPS 4
#define HILL_NZB 4       // z band width: p + 1 with p = 3
#define HILL_MAX_NZ 32   // z modes held one per lane
#define HILL_MAX_QPE 16  // z quadrature points per z element

namespace {

struct HillAdvDev {
    int nr, nz, qpe, n_seg, lmax;
    const int* seg_q0;    // [n_seg] first 2D point
    const int* seg_q1;    // [n_seg] one past the last
    const int* seg_pat;   // [n_seg] offset of the pattern in pat_idx (also the partial row offset)
    const int* seg_len;   // [n_seg] modes in the pattern
    const int* pat_idx;   // reduced modes of each segment's pattern
    const int* sp_ptr;    // [n2q + 1] row offsets of the sparse sample rows
    const double* phi;    // sample values, derivative values (physical x, y)
    const double* dpx;
    const double* dpy;
    const double* w2;     // [n2q]
    const int* zb;        // [nz][HILL_NZB] z modes seen by element e, in periodic order
    const double* Vl;     // [nz][qpe][HILL_NZB] basis values at the element's points
    const double* dVl;    // derivatives
    const double* wzl;    // [nz][qpe] z weights
    const int* g_ptr;     // [nr + 1] gather: partial rows of each mode, in segment order
    const int* g_ent;
    const double* Mzinv;  // [nz][nz]
    const double* M2inv;  // [nr][nr]
};

// One CTA (HILL_WARPS warps) per segment.  Each round, warp w takes point
// q0 + HILL_WARPS*r + w through (a)-(c); after a CTA barrier every warp adds
// all the round's points into the modes it owns (a = w + HILL_WARPS t) in (d).
// Dynamic shared memory: the segment's coefficient rows C[a][comp][iz]
// (lmax x 3 x nz), per warp two 9 x nz buffers, and the z tables (basis
// values, derivatives, weights of every z element, laid out lane-contiguous).
// CTA b takes segment seg_list[b]: segments are launched in two groups, the
// ones of at most 16 modes with LMAX = 16 (a smaller CTA, four per SM) and
// the longer ones with the next LMAX.
template <int LMAX>
__global__ void __launch_bounds__(HILL_WARPS * 32, 4) hill_segment_kernel(HillAdvDev d, const int* seg_list,
                                                                      const double* ux, const double* uy,
                                                                      const double* uz, double* part) {
    constexpr int LW = (LMAX + HILL_WARPS - 1) / HILL_WARPS;  // modes owned per warp
    extern __shared__ double hs[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = __ldg(seg_list + blockIdx.x);
    const int nz = d.nz;
    double* Cs = hs;
    double* Tw = Cs + LMAX * 3 * nz + w * 18 * nz;
    double* PXYall = Cs + LMAX * 3 * nz + 9 * nz;  // warp w' buffer at PXYall + w' * 18 nz
    double* PXY = PXYall + w * 18 * nz;
    // z tables, lane-contiguous: V[(k * NZB + j) * nz + e], wz[k * nz + e]
    const int qpe = d.qpe;
    double* zV = Cs + LMAX * 3 * nz + HILL_WARPS * 18 * nz;
    double* zD = zV + qpe * HILL_NZB * nz;
    double* zW = zD + qpe * HILL_NZB * nz;
    for (int e = threadIdx.x; e < nz * qpe * HILL_NZB; e += blockDim.x) {
        const int el_ = e / (qpe * HILL_NZB), k = (e / HILL_NZB) % qpe, j = e % HILL_NZB;
        zV[(k * HILL_NZB + j) * nz + el_] = __ldg(d.Vl + e);
        zD[(k * HILL_NZB + j) * nz + el_] = __ldg(d.dVl + e);
    }
    for (int e = threadIdx.x; e < nz * qpe; e += blockDim.x) zW[(e % qpe) * nz + e / qpe] = __ldg(d.wzl + e);
    const int L = d.seg_len[s];
    const int* pat = d.pat_idx + d.seg_pat[s];
    const double* U[3] = {ux, uy, uz};
    for (int e = threadIdx.x; e < L * 3 * nz; e += blockDim.x) {
        const int a = e / (3 * nz), r = e % (3 * nz), c = r / nz, iz = r % nz;
        Cs[e] = U[c][(size_t)pat[a] * nz + iz];
    }
    double acc[LW][3];
#pragma unroll
    for (int t = 0; t < LW; ++t) acc[t][0] = acc[t][1] = acc[t][2] = 0.0;
    int zb[HILL_NZB];
    const bool el = lane < nz;
#pragma unroll
    for (int j = 0; j < HILL_NZB; ++j) zb[j] = el ? d.zb[lane * HILL_NZB + j] : 0;
    __syncthreads();

    const int q0 = d.seg_q0[s], q1 = d.seg_q1[s];
    for (int qr = q0; qr < q1; qr += HILL_WARPS) {
        const int q = qr + w;
        if (q < q1) {  // warp-uniform
            const int base = d.sp_ptr[q];
            // (a) 2D sample of u_x, u_y, u_z and their x, y derivatives; lane = iz
            if (lane < nz) {
                double T[9];
#pragma unroll
                for (int k = 0; k < 9; ++k) T[k] = 0.0;
#pragma unroll 4
                for (int a = 0; a < L; ++a) {
                    const double ph = __ldg(d.phi + base + a), gx = __ldg(d.dpx + base + a),
                                 gy = __ldg(d.dpy + base + a);
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const double cv = Cs[(a * 3 + c) * nz + lane];
                        T[c * 3 + 0] = fma(ph, cv, T[c * 3 + 0]);
                        T[c * 3 + 1] = fma(gx, cv, T[c * 3 + 1]);
                        T[c * 3 + 2] = fma(gy, cv, T[c * 3 + 2]);
                    }
                }
#pragma unroll
                for (int k = 0; k < 9; ++k) {
                    Tw[k * nz + lane] = T[k];
                    PXY[k * nz + lane] = 0.0;
                }
            }
            __syncwarp();
            // (b) lane = z element: expand, products, contract against the band;
            // one component c at a time, its band integrals scattered in (c)
            // before the next component starts
            if (el) {
                double Tv[3][HILL_NZB];  // values of u_x, u_y, u_z on the band
#pragma unroll
                for (int k = 0; k < 3; ++k)
#pragma unroll
                    for (int j = 0; j < HILL_NZB; ++j) Tv[k][j] = Tw[(k * 3) * nz + zb[j]];
#pragma unroll 1
                for (int c = 0; c < 3; ++c) {
                    double Tx[HILL_NZB], Ty[HILL_NZB];
#pragma unroll
                    for (int j = 0; j < HILL_NZB; ++j) {
                        Tx[j] = Tw[(c * 3 + 1) * nz + zb[j]];
                        Ty[j] = Tw[(c * 3 + 2) * nz + zb[j]];
                    }
                    double Pl[HILL_NZB], Xl[HILL_NZB], Yl[HILL_NZB];
#pragma unroll
                    for (int j = 0; j < HILL_NZB; ++j) Pl[j] = Xl[j] = Yl[j] = 0.0;
                    for (int k = 0; k < qpe; ++k) {
                        double vl[HILL_NZB], dvl[HILL_NZB];
#pragma unroll
                        for (int j = 0; j < HILL_NZB; ++j) {
                            vl[j] = zV[(k * HILL_NZB + j) * nz + lane];
                            dvl[j] = zD[(k * HILL_NZB + j) * nz + lane];
                        }
                        const double wk = zW[k * nz + lane];
                        double u[3] = {0.0, 0.0, 0.0};
                        double gx = 0.0, gy = 0.0, gz = 0.0;
#pragma unroll
                        for (int j = 0; j < HILL_NZB; ++j) {
#pragma unroll
                            for (int v = 0; v < 3; ++v) u[v] = fma(vl[j], Tv[v][j], u[v]);
                            gx = fma(vl[j], Tx[j], gx);
                            gy = fma(vl[j], Ty[j], gy);
                        }
#pragma unroll
                        for (int j = 0; j < HILL_NZB; ++j) {
                            const double tc = c == 0 ? Tv[0][j] : (c == 1 ? Tv[1][j] : Tv[2][j]);
                            gz = fma(dvl[j], tc, gz);
                        }
                        const double uc = c == 0 ? u[0] : (c == 1 ? u[1] : u[2]);
                        // w = u (the field advects itself): w.grad u_c and w u_c
                        const double conv = u[0] * gx + u[1] * gy + u[2] * gz;
                        const double hw = 0.5 * wk;
                        const double fx = hw * u[0] * uc, fy = hw * u[1] * uc, fz = hw * u[2] * uc;
                        const double cw = hw * conv;
#pragma unroll
                        for (int j = 0; j < HILL_NZB; ++j) {
                            Pl[j] += vl[j] * cw - dvl[j] * fz;
                            Xl[j] -= vl[j] * fx;
                            Yl[j] -= vl[j] * fy;
                        }
                    }
                    // (c) band scatter: round j writes mode zb[j], distinct across lanes
#pragma unroll
                    for (int j = 0; j < HILL_NZB; ++j) {
                        const int m = zb[j];
                        PXY[(c * 3 + 0) * nz + m] += Pl[j];
                        PXY[(c * 3 + 1) * nz + m] += Xl[j];
                        PXY[(c * 3 + 2) * nz + m] += Yl[j];
                        __syncwarp(__activemask());
                    }
                }
            }
        }
        __syncthreads();
        // (d) 2D load of the round's points into the modes this warp owns; lane = iz
        if (lane < nz) {
            for (int w2i = 0; w2i < HILL_WARPS; ++w2i) {
                const int qq = qr + w2i;
                if (qq >= q1) break;
                const int base = d.sp_ptr[qq];
                const double wq = __ldg(d.w2 + qq);
                const double* B = PXYall + w2i * 18 * nz;
                double P[3], X[3], Y[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    P[c] = wq * B[(c * 3 + 0) * nz + lane];
                    X[c] = wq * B[(c * 3 + 1) * nz + lane];
                    Y[c] = wq * B[(c * 3 + 2) * nz + lane];
                }
#pragma unroll
                for (int t = 0; t < LW; ++t) {
                    const int a = w + HILL_WARPS * t;
                    if (a < L) {
                        const double ph = __ldg(d.phi + base + a), gx = __ldg(d.dpx + base + a),
                                     gy = __ldg(d.dpy + base + a);
#pragma unroll
                        for (int c = 0; c < 3; ++c) acc[t][c] += ph * P[c] + gx * X[c] + gy * Y[c];
                    }
                }
            }
        }
        __syncthreads();
    }
    if (lane < nz) {
        double* out = part + (size_t)d.seg_pat[s] * 3 * nz;
#pragma unroll
        for (int t = 0; t < LW; ++t) {
            const int a = w + HILL_WARPS * t;
            if (a < L) {
#pragma unroll
                for (int c = 0; c < 3; ++c) out[((size_t)a * 3 + c) * nz + lane] = acc[t][c];
            }
        }
    }
}

// Per reduced mode (one warp, lane = iz): sum its segment partials in segment
// order, then apply Mz^-1 along z; writes T[m][c*nz + iz].
__global__ void hill_gather_kernel(HillAdvDev d, const double* part, double* T) {
    const int lane = threadIdx.x & 31;
    const int m = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (m >= d.nr) return;
    const int nz = d.nz;
    double r[3] = {0.0, 0.0, 0.0};
    if (lane < nz)
        for (int k = d.g_ptr[m]; k < d.g_ptr[m + 1]; ++k) {
            const double* p = part + (size_t)d.g_ent[k] * 3 * nz;
#pragma unroll
            for (int c = 0; c < 3; ++c) r[c] += p[c * nz + lane];
        }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double t = 0.0;
        for (int jz = 0; jz < nz; ++jz) {
            const double rj = __shfl_sync(0xffffffffu, r[c], jz);
            if (lane < nz) t = fma(d.Mzinv[lane * nz + jz], rj, t);
        }
        if (lane < nz) T[(size_t)(c * nz + lane) * d.nr + m] = t;
    }
}

// C_part[z] = A[:, kslice(z)] B[kslice(z), :] for row-major A (n x n) and B
// given transposed (BT: ncol x n, row col = column col of B), on the FP64
// tensor cores (dmma_tile, 64 x 64 tiles, split over K by blockIdx.z).
__global__ void __launch_bounds__(256) hill_gemm_kernel(int n, int ncol, const double* A, const double* BT, double* Cp) {
    const int kch = (n + gridDim.z - 1) / gridDim.z;
    const int kb = blockIdx.z * kch, ke = min(n, kb + kch);
    double* Cz = Cp + (size_t)blockIdx.z * n * ncol;
    dmma_tile(
        n, ncol, kb, ke, blockIdx.y * DG_BM, blockIdx.x * DG_BN,
        [&](int m, int k) { return __ldg(A + (size_t)m * n + k); },
        [&](int c, int k) { return __ldg(BT + (size_t)c * n + k); },
        [&](int m, int c, double v) { Cz[(size_t)m * ncol + c] = v; });
}

// out_c[m*nz + iz] = scale * sum_z Cp[z][m][c*nz + iz]  (slices in order)
__global__ void hill_sum_kernel(int nr, int nz, int ks, const double* Cp, double scale, double* ox, double* oy,
                                double* oz) {
    const int ncol = 3 * nz;
    const long total = (long)nr * ncol;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int z = 0; z < ks; ++z) s += Cp[(size_t)z * total + t];
        const int m = (int)(t / ncol), r = (int)(t % ncol), c = r / nz, iz = r % nz;
        double* o = c == 0 ? ox : (c == 1 ? oy : oz);
        o[(size_t)m * nz + iz] = scale * s;
    }
}

// y = a x + b (y + dt L)  over n entries, for three components (SSP-RK3 stages)
__global__ void hill_rk_kernel(long n, double a, const double* x0, const double* x1, const double* x2, double b,
                               double dt, const double* L0, const double* L1, const double* L2, const double* v0,
                               const double* v1, const double* v2, double* y0, double* y1, double* y2) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        y0[i] = a * x0[i] + b * (v0[i] + dt * L0[i]);
        y1[i] = a * x1[i] + b * (v1[i] + dt * L1[i]);
        y2[i] = a * x2[i] + b * (v2[i] + dt * L2[i]);
    }
}

__global__ void hill_add_kernel(long n, double c, double* y) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) y[i] += c;
}

int hfail(cudaError_t e, const char* what) {
    cutcell_internal_set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return CUTCELL_E_CUDA;
}

int harg(const std::string& what, int code = CUTCELL_E_ARG) {
    cutcell_internal_set_error(what);
    return code;
}

#define HCK(call)                                       \
    do {                                                \
        cudaError_t _e = (call);                        \
        if (_e != cudaSuccess) return hfail(_e, #call); \
    } while (0)

constexpr int HILL_KSPLIT = 4;

}  // namespace

struct cutcell_hill {
    int device = 0;
    HillAdvDev d;
    int n_part = 0;      // partial rows (sum of segment lengths)
    double* part = nullptr;
    double* T = nullptr;     // [nr][3 nz]
    double* Cp = nullptr;    // [KSPLIT][nr][3 nz]
    double* work = nullptr;  // 3 stage fields x 3 comps + 3 operator outputs: 12 x nr x nz
    int* seg_list = nullptr;  // segments of <= 16 modes, then the longer ones
    int n_short = 0;
    int lm_long = 16;         // LMAX of the longer group
    size_t smem_short = 0;    // dynamic shared memory of the LMAX = 16 group
    size_t smem = 0;          // ... and of the longer group
};

namespace {

int advect(cutcell_hill* H, const double* ux, const double* uy, const double* uz, double scale, double* ox,
           double* oy, double* oz, cudaStream_t s) {
    const HillAdvDev& d = H->d;
    const int n_long = d.n_seg - H->n_short;
    const int* longs = H->seg_list + H->n_short;
    if (H->n_short > 0)
        hill_segment_kernel<16><<<H->n_short, HILL_WARPS * 32, H->smem_short, s>>>(d, H->seg_list, ux, uy, uz, H->part);
    if (n_long > 0) {
        if (H->lm_long <= 24)
            hill_segment_kernel<24><<<n_long, HILL_WARPS * 32, H->smem, s>>>(d, longs, ux, uy, uz, H->part);
        else
            hill_segment_kernel<32><<<n_long, HILL_WARPS * 32, H->smem, s>>>(d, longs, ux, uy, uz, H->part);
    }
    HCK(cudaGetLastError());
    hill_gather_kernel<<<(d.nr + 7) / 8, 256, 0, s>>>(d, H->part, H->T);
    HCK(cudaGetLastError());
    const int ncol = 3 * d.nz;
    dim3 g((ncol + DG_BN - 1) / DG_BN, (d.nr + DG_BM - 1) / DG_BM, HILL_KSPLIT);
    hill_gemm_kernel<<<g, 256, 0, s>>>(d.nr, ncol, d.M2inv, H->T, H->Cp);
    HCK(cudaGetLastError());
    hill_sum_kernel<<<296, 256, 0, s>>>(d.nr, d.nz, HILL_KSPLIT, H->Cp, scale, ox, oy, oz);
    HCK(cudaGetLastError());
    return CUTCELL_OK;
}

template <int LMAX>
int set_smem(size_t bytes) {
    return (int)cudaFuncSetAttribute(hill_segment_kernel<LMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)bytes);
}

}  // namespace

extern "C" {

int cutcell_fastdiag_solve(cutcell_fastdiag* fd, const double* ux, const double* uy, const double* uz, double* ox,
                           double* oy, double* oz, void* stream);

int cutcell_hill_create(const CutcellHillDesc* desc, cutcell_hill** out) {
    if (!out || !desc) return CUTCELL_E_ARG;
    *out = nullptr;
    const CutcellHillDesc& h = *desc;
    if (h.nr < 1 || h.nz < 1 || h.n_seg < 1 || h.n_part < 1) return harg("hill: empty sizes", CUTCELL_E_SHAPE);
    if (h.nz > HILL_MAX_NZ) return harg("hill: nz above 32 is not supported", CUTCELL_E_SHAPE);
    if (h.qpe < 1 || h.qpe > HILL_MAX_QPE) return harg("hill: z points per element outside [1, 16]", CUTCELL_E_SHAPE);
    if (h.nzb != HILL_NZB) return harg("hill: z band width must be 4 (degree 3)", CUTCELL_E_SHAPE);
    if (h.lmax < 1 || h.lmax > 32) return harg("hill: more than 32 modes in a 2D row pattern", CUTCELL_E_SHAPE);
    cutcell_hill* H = new cutcell_hill();
    HillAdvDev& d = H->d;
    d.nr = h.nr;
    d.nz = h.nz;
    d.qpe = h.qpe;
    d.n_seg = h.n_seg;
    d.lmax = h.lmax;
    d.seg_q0 = h.seg_q0;
    d.seg_q1 = h.seg_q1;
    d.seg_pat = h.seg_pat;
    d.seg_len = h.seg_len;
    d.pat_idx = h.pat_idx;
    d.sp_ptr = h.sp_ptr;
    d.phi = h.phi;
    d.dpx = h.dpx;
    d.dpy = h.dpy;
    d.w2 = h.w2;
    d.zb = h.zb;
    d.Vl = h.Vl;
    d.dVl = h.dVl;
    d.wzl = h.wzl;
    d.g_ptr = h.g_ptr;
    d.g_ent = h.g_ent;
    d.Mzinv = h.Mzinv;
    d.M2inv = h.M2inv;
    H->n_part = h.n_part;
    auto smem_for = [&](int lm) {
        return sizeof(double) * ((size_t)lm * 3 * h.nz + (size_t)HILL_WARPS * 18 * h.nz +
                                 (size_t)h.nz * h.qpe * (2 * HILL_NZB + 1));
    };
    const size_t fld = (size_t)h.nr * h.nz;
    cudaError_t e = cudaGetDevice(&H->device);
    // segment groups by pattern length (host copy of seg_len)
    std::vector<int> len(h.n_seg), order;
    if (e == cudaSuccess) e = cudaMemcpy(len.data(), h.seg_len, sizeof(int) * h.n_seg, cudaMemcpyDeviceToHost);
    int lmax_long = 0;
    for (int i = 0; i < h.n_seg && e == cudaSuccess; ++i)
        if (len[i] <= 16) order.push_back(i);
    H->n_short = (int)order.size();
    for (int i = 0; i < h.n_seg && e == cudaSuccess; ++i)
        if (len[i] > 16) {
            order.push_back(i);
            lmax_long = std::max(lmax_long, len[i]);
        }
    if (e == cudaSuccess && (int)order.size() != h.n_seg) e = cudaErrorInvalidValue;
    if (e == cudaSuccess && lmax_long > h.lmax) {
        delete H;
        return harg("hill: a segment pattern is longer than lmax", CUTCELL_E_SHAPE);
    }
    H->lm_long = lmax_long <= 24 ? 24 : 32;
    H->smem_short = smem_for(16);
    H->smem = smem_for(H->lm_long);
    if (e == cudaSuccess) e = cudaMalloc(&H->seg_list, sizeof(int) * h.n_seg);
    if (e == cudaSuccess) e = cudaMemcpy(H->seg_list, order.data(), sizeof(int) * h.n_seg, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&H->part, sizeof(double) * (size_t)h.n_part * 3 * h.nz);
    if (e == cudaSuccess) e = cudaMalloc(&H->T, sizeof(double) * fld * 3);
    if (e == cudaSuccess) e = cudaMalloc(&H->Cp, sizeof(double) * fld * 3 * HILL_KSPLIT);
    if (e == cudaSuccess) e = cudaMalloc(&H->work, sizeof(double) * fld * 12);
    if (e == cudaSuccess && H->smem_short > 48 * 1024) e = (cudaError_t)set_smem<16>(H->smem_short);
    if (e == cudaSuccess && H->smem > 48 * 1024)
        e = (cudaError_t)(H->lm_long == 24 ? set_smem<24>(H->smem) : set_smem<32>(H->smem));
    if (e != cudaSuccess) {
        const int st = hfail(e, "cutcell_hill_create");
        cutcell_hill_destroy(H);
        return st;
    }
    *out = H;
    return CUTCELL_OK;
}

int cutcell_hill_skew_conv(cutcell_hill* H, const double* ux, const double* uy, const double* uz, double* cx,
                           double* cy, double* cz, void* stream) {
    if (!H || !ux || !uy || !uz || !cx || !cy || !cz) return CUTCELL_E_ARG;
    return advect(H, ux, uy, uz, 1.0, cx, cy, cz, (cudaStream_t)stream);
}

int cutcell_hill_step(cutcell_hill* H, cutcell_fastdiag* fd, double* ux, double* uy, double* uz, double dt,
                      double fx, void* stream) {
    if (!H || !fd || !ux || !uy || !uz) return CUTCELL_E_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const long n = (long)H->d.nr * H->d.nz;
    double* W = H->work;
    double* L[3] = {W, W + n, W + 2 * n};
    double* A[3] = {W + 3 * n, W + 4 * n, W + 5 * n};  // u1, then u2
    double* B[3] = {W + 6 * n, W + 7 * n, W + 8 * n};  // u*
    const int g = 592, t = 256;
    int st;
    // u1 = u + dt L(u)
    if ((st = advect(H, ux, uy, uz, -1.0, L[0], L[1], L[2], s))) return st;
    hill_rk_kernel<<<g, t, 0, s>>>(n, 0.0, ux, uy, uz, 1.0, dt, L[0], L[1], L[2], ux, uy, uz, A[0], A[1], A[2]);
    // u2 = 3/4 u + 1/4 (u1 + dt L(u1))
    if ((st = advect(H, A[0], A[1], A[2], -1.0, L[0], L[1], L[2], s))) return st;
    hill_rk_kernel<<<g, t, 0, s>>>(n, 0.75, ux, uy, uz, 0.25, dt, L[0], L[1], L[2], A[0], A[1], A[2], A[0], A[1],
                                   A[2]);
    // u* = 1/3 u + 2/3 (u2 + dt L(u2))
    if ((st = advect(H, A[0], A[1], A[2], -1.0, L[0], L[1], L[2], s))) return st;
    hill_rk_kernel<<<g, t, 0, s>>>(n, 1.0 / 3.0, ux, uy, uz, 2.0 / 3.0, dt, L[0], L[1], L[2], A[0], A[1], A[2], B[0],
                                   B[1], B[2]);
    if (fx != 0.0) hill_add_kernel<<<g, t, 0, s>>>(n, dt * fx, B[0]);
    HCK(cudaGetLastError());
    return cutcell_fastdiag_solve(fd, B[0], B[1], B[2], ux, uy, uz, stream);
}

int cutcell_hill_destroy(cutcell_hill* H) {
    if (!H) return CUTCELL_E_ARG;
    cudaFree(H->part);
    cudaFree(H->T);
    cudaFree(H->Cp);
    cudaFree(H->work);
    cudaFree(H->seg_list);
    delete H;
    return CUTCELL_OK;
}

}  // extern "C"
