// Operator applies used inside the persistent Krylov kernels.
//
//  * CsrOp   : y = A p for an assembled reduced matrix (E^T A E in CSR), the
//              drop-in for ``solve_spd(A, b)`` (code/fast_solver_backends.py:194-289).
//  * TileOp  : matrix-free y = E^T A E p on the structured background grid:
//              E gather fused into the tile load, sum-factorised full tiles,
//              element-by-element mixed tiles (dense cut-element blocks), and
//              a deterministic cross-tile reduction fused with the E^T scatter.
//
// Vectors shared between blocks are read with __ldcg (L2 only) because they
// are rewritten inside the same launch; operator data is read-only and uses
// the non-coherent path.
#pragma once

#include "common.cuh"

// ---------------------------------------------------------------------------
// CSR operator
// ---------------------------------------------------------------------------

template <typename V>
struct CsrOp {
    int n;
    int tpr_log2;  // threads per row = 1 << tpr_log2 (1..32)
    const int* __restrict__ ptr;
    const int* __restrict__ idx;
    const V* __restrict__ val;

    // y = A p over the whole grid; returns this thread's share of p.y.
    __device__ __forceinline__ double apply(const double* p, double* y, const GridSync&, double*) const {
        typedef typename Conv<V>::acc acc_t;
        const int tpr = 1 << tpr_log2;
        const int lane = threadIdx.x & 31;
        const int sub = lane & (tpr - 1);
        const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        const int nwarps = (gridDim.x * blockDim.x) >> 5;
        const int rows_per_warp = 32 >> tpr_log2;
        double part = 0.0;
        for (int base = gwarp * rows_per_warp; base < n; base += nwarps * rows_per_warp) {
            const int row = base + (lane >> tpr_log2);
            acc_t s = 0;
            if (row < n) {
                const int k1 = __ldg(ptr + row + 1);
                for (int k = __ldg(ptr + row) + sub; k < k1; k += tpr)
                    s += Conv<V>::ld(val + k) * (acc_t)__ldcg(p + __ldg(idx + k));
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
                if (o < tpr) s += __shfl_down_sync(0xffffffffu, s, o, tpr);
            if (row < n && sub == 0) {
                const double yr = (double)s;
                y[row] = yr;
                part += __ldcg(p + row) * yr;
            }
        }
        return part;
    }
};

// ---------------------------------------------------------------------------
// Aggregation extension E (n_full x n_red): identity rows + small rows.
// ---------------------------------------------------------------------------

struct ExtDev {
    int n_full, n_red, n_small;
    const int* __restrict__ red_of_full;   // [n_full] reduced column of identity rows, -1 otherwise
    const int* __restrict__ small_slot;    // [n_full] slot in the small-row CSR, -1 otherwise
    const int* __restrict__ small_ptr;     // [n_small+1]
    const int* __restrict__ small_idx;     // reduced columns
    const double* __restrict__ small_val;
    const int* __restrict__ full_of_red;   // [n_red]
    const int* __restrict__ smallT_ptr;    // [n_red+1]  E_small^T rows
    const int* __restrict__ smallT_row;    // full index of the contributing small row
    const double* __restrict__ smallT_val;

    // (E x)_i
    __device__ __forceinline__ double gather(const double* x, int i) const {
        const int r = __ldg(red_of_full + i);
        if (r >= 0) return __ldcg(x + r);
        const int s = __ldg(small_slot + i);
        if (s < 0) return 0.0;
        double acc = 0.0;
        const int k1 = __ldg(small_ptr + s + 1);
        for (int k = __ldg(small_ptr + s); k < k1; ++k) acc += __ldg(small_val + k) * __ldcg(x + __ldg(small_idx + k));
        return acc;
    }
};

// ---------------------------------------------------------------------------
// Matrix-free tile operator
// ---------------------------------------------------------------------------

enum { TILE_EMPTY = 0, TILE_FULL = 1, TILE_MIXED = 2 };

template <typename CT>
struct TileOp {
    int n;      // elements per axis
    int p;      // degree
    int P1;     // p + 1
    int P;      // (p+1)^3
    int T;      // elements per tile edge
    int D;      // T + p, DOFs per tile edge
    int nta;    // tiles per axis
    int nb;     // DOFs per axis (n + p)
    int ntile_list;
    double a_mass;
    const int* __restrict__ tile_list;   // nonempty linear tile ids (work order)
    const int* __restrict__ tile_kind;   // per linear tile
    const int* __restrict__ tile_eptr;   // per linear tile, element range (mixed tiles)
    const int* __restrict__ tile_elem;   // local element id (ez*T+ey)*T+ex
    const int* __restrict__ tile_ecut;   // cut block index, -1 for a full element
    const double* __restrict__ M1;       // [n][P1*P1]
    const double* __restrict__ Kt1;      // [3][n][P1*P1]
    const double* __restrict__ TM;       // [nta][D*D]
    const double* __restrict__ TA;       // [nta][D*D]  a_mass*TM + TK_x
    const double* __restrict__ TK;       // [3][nta][D*D]
    const CT* __restrict__ cut_mats;     // [ncut][P*P]
    ExtDev ext;
    double* ypart;                       // [nta^3][D^3]

    __device__ __forceinline__ int D3() const { return D * D * D; }

    // ---- phase 1: one tile -> ypart ---------------------------------------
    __device__ void tile_apply(const double* pred, int tile, double* sm) const {
        typedef typename Conv<CT>::acc acc_t;
        const int d3 = D3();
        const int tx = tile % nta, ty = (tile / nta) % nta, tz = tile / (nta * nta);
        double* xs = sm;               // D^3
        double* out = ypart + (size_t)tile * d3;
        for (int k = threadIdx.x; k < d3; k += blockDim.x) {
            const int dx = k % D, dy = (k / D) % D, dz = k / (D * D);
            const int gx = tx * T + dx, gy = ty * T + dy, gz = tz * T + dz;
            double v = 0.0;
            if (gx < nb && gy < nb && gz < nb) v = ext.gather(pred, (gz * nb + gy) * nb + gx);
            xs[k] = v;
        }
        __syncthreads();
        const int kind = __ldg(tile_kind + tile);
        if (kind == TILE_FULL) {
            double* u1 = xs + d3;
            double* u2 = u1 + d3;
            double* v1 = u2 + d3;
            double* v2 = v1 + d3;
            const double* Mx = TM + (size_t)tx * D * D;
            const double* Ax = TA + (size_t)tx * D * D;
            const double* My = TM + (size_t)ty * D * D;
            const double* Ky = TK + ((size_t)1 * nta + ty) * D * D;
            const double* Mz = TM + (size_t)tz * D * D;
            const double* Kz = TK + ((size_t)2 * nta + tz) * D * D;
            // x passes
            for (int k = threadIdx.x; k < d3; k += blockDim.x) {
                const int i = k % D, row = k - i;
                const int j0 = max(0, i - p), j1 = min(D - 1, i + p);
                double s1 = 0.0, s2 = 0.0;
                for (int j = j0; j <= j1; ++j) {
                    const double xv = xs[row + j];
                    s1 += __ldg(Mx + i * D + j) * xv;
                    s2 += __ldg(Ax + i * D + j) * xv;
                }
                u1[k] = s1;
                u2[k] = s2;
            }
            __syncthreads();
            // y passes: v1 = My u1, v2 = My u2 + Ky u1
            for (int k = threadIdx.x; k < d3; k += blockDim.x) {
                const int x = k % D, i = (k / D) % D, z = k / (D * D);
                const int j0 = max(0, i - p), j1 = min(D - 1, i + p);
                double s1 = 0.0, s2 = 0.0;
                for (int j = j0; j <= j1; ++j) {
                    const int o = (z * D + j) * D + x;
                    const double m = __ldg(My + i * D + j);
                    s1 += m * u1[o];
                    s2 += m * u2[o] + __ldg(Ky + i * D + j) * u1[o];
                }
                v1[k] = s1;
                v2[k] = s2;
            }
            __syncthreads();
            // z passes: out = Mz v2 + Kz v1
            for (int k = threadIdx.x; k < d3; k += blockDim.x) {
                const int xy = k % (D * D), i = k / (D * D);
                const int j0 = max(0, i - p), j1 = min(D - 1, i + p);
                double s = 0.0;
                for (int j = j0; j <= j1; ++j) {
                    const int o = j * D * D + xy;
                    s += __ldg(Mz + i * D + j) * v2[o] + __ldg(Kz + i * D + j) * v1[o];
                }
                out[k] = s;
            }
            __syncthreads();
            return;
        }
        // ---- mixed tile: element by element, one warp per element --------
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int nw = blockDim.x >> 5;
        double* acc = xs + d3 + (size_t)warp * d3;            // per-warp accumulator
        double* e0 = xs + d3 + (size_t)nw * d3 + (size_t)warp * 4 * P;
        double* e1 = e0 + P;
        double* e2 = e1 + P;
        double* e3 = e2 + P;
        for (int k = lane; k < d3; k += 32) acc[k] = 0.0;
        const int eb = __ldg(tile_eptr + tile), ee = __ldg(tile_eptr + tile + 1);
        const int P1sq = P1 * P1;
        for (int it = eb + warp; it < ee; it += nw) {
            const int le = __ldg(tile_elem + it);
            const int lx = le % T, ly = (le / T) % T, lz = le / (T * T);
            const int cut = __ldg(tile_ecut + it);
            __syncwarp();
            for (int k = lane; k < P; k += 32) {
                const int a = k % P1, b = (k / P1) % P1, c = k / P1sq;
                e0[k] = xs[((lz + c) * D + (ly + b)) * D + (lx + a)];
            }
            __syncwarp();
            if (cut >= 0) {
                const CT* A = cut_mats + (size_t)cut * P * P;
                for (int r0 = 0; r0 < P; r0 += 32) {
                    const int r = r0 + lane;
                    acc_t s = 0;
                    if (r < P) {
                        for (int c = 0; c < P; ++c) s += Conv<CT>::ld(A + (size_t)c * P + r) * (acc_t)e0[c];
                        const int a = r % P1, b = (r / P1) % P1, cc = r / P1sq;
                        acc[((lz + cc) * D + (ly + b)) * D + (lx + a)] += (double)s;
                    }
                }
            } else {
                const int ex = tx * T + lx, ey = ty * T + ly, ez = tz * T + lz;
                const double* Mx = M1 + (size_t)ex * P1sq;
                const double* Kx = Kt1 + (size_t)ex * P1sq;
                const double* My = M1 + (size_t)ey * P1sq;
                const double* Ky = Kt1 + ((size_t)n + ey) * P1sq;
                const double* Mz = M1 + (size_t)ez * P1sq;
                const double* Kz = Kt1 + ((size_t)2 * n + ez) * P1sq;
                for (int k = lane; k < P; k += 32) {
                    const int i = k % P1, row = k - i;
                    double s1 = 0.0, s2 = 0.0;
                    for (int j = 0; j < P1; ++j) {
                        const double m = __ldg(Mx + i * P1 + j);
                        s1 += m * e0[row + j];
                        s2 += (a_mass * m + __ldg(Kx + i * P1 + j)) * e0[row + j];
                    }
                    e1[k] = s1;
                    e2[k] = s2;
                }
                __syncwarp();
                for (int k = lane; k < P; k += 32) {
                    const int x = k % P1, i = (k / P1) % P1, z = k / P1sq;
                    double s1 = 0.0, s2 = 0.0;
                    for (int j = 0; j < P1; ++j) {
                        const int o = (z * P1 + j) * P1 + x;
                        const double m = __ldg(My + i * P1 + j);
                        s1 += m * e1[o];
                        s2 += m * e2[o] + __ldg(Ky + i * P1 + j) * e1[o];
                    }
                    e3[k] = s1;
                    e0[k] = s2;  // e0 no longer needed as input
                }
                __syncwarp();
                for (int k = lane; k < P; k += 32) {
                    const int xy = k % P1sq, i = k / P1sq;
                    double s = 0.0;
                    for (int j = 0; j < P1; ++j) {
                        const int o = j * P1sq + xy;
                        s += __ldg(Mz + i * P1 + j) * e0[o] + __ldg(Kz + i * P1 + j) * e3[o];
                    }
                    const int a = xy % P1, b = xy / P1;
                    acc[((lz + i) * D + (ly + b)) * D + (lx + a)] += s;
                }
            }
        }
        __syncthreads();
        double* acc0 = xs + d3;
        for (int k = threadIdx.x; k < d3; k += blockDim.x) {
            double s = 0.0;
            for (int w = 0; w < nw; ++w) s += acc0[(size_t)w * d3 + k];
            out[k] = s;
        }
        __syncthreads();
    }

    // ---- phase 2 helpers ---------------------------------------------------
    __device__ __forceinline__ double yfull(int i) const {
        const int ix = i % nb, iy = (i / nb) % nb, iz = i / (nb * nb);
        int t1x = min(ix / T, nta - 1), t1y = min(iy / T, nta - 1), t1z = min(iz / T, nta - 1);
        const int d3 = D3();
        double s = 0.0;
        for (int tz = t1z - 1; tz <= t1z; ++tz) {
            if (tz < 0 || iz - tz * T >= D) continue;
            for (int ty = t1y - 1; ty <= t1y; ++ty) {
                if (ty < 0 || iy - ty * T >= D) continue;
                for (int tx = t1x - 1; tx <= t1x; ++tx) {
                    if (tx < 0 || ix - tx * T >= D) continue;
                    const int tile = (tz * nta + ty) * nta + tx;
                    s += __ldcg(ypart + (size_t)tile * d3 + ((iz - tz * T) * D + (iy - ty * T)) * D + (ix - tx * T));
                }
            }
        }
        return s;
    }

    __device__ __forceinline__ double scatter_row(int j) const {
        double y = yfull(__ldg(ext.full_of_red + j));
        const int k1 = __ldg(ext.smallT_ptr + j + 1);
        for (int k = __ldg(ext.smallT_ptr + j); k < k1; ++k)
            y += __ldg(ext.smallT_val + k) * yfull(__ldg(ext.smallT_row + k));
        return y;
    }

    __device__ __forceinline__ double apply(const double* p, double* y, const GridSync& gs, double* sm) const {
        for (int li = blockIdx.x; li < ntile_list; li += gridDim.x) tile_apply(p, __ldg(tile_list + li), sm);
        if (!grid_sync(gs)) return 0.0;
        double part = 0.0;
        for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < ext.n_red; j += gridDim.x * blockDim.x) {
            const double yj = scatter_row(j);
            y[j] = yj;
            part += __ldcg(p + j) * yj;
        }
        return part;
    }

    static size_t smem_bytes(int D, int P, int nwarps) {
        const size_t d3 = (size_t)D * D * D;
        size_t full = 5 * d3;
        size_t mixed = d3 + (size_t)nwarps * d3 + (size_t)nwarps * 4 * P;
        return (full > mixed ? full : mixed) * sizeof(double);
    }
};
