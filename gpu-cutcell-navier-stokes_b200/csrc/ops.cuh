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
    static constexpr bool kFusedP = false;
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

// CSR structure check: row offsets start at 0, end at nnz and never decrease;
// every column index lies in [0, n).  Reads only ptr[0..n] and idx[0..nnz), so
// it is safe on any input of the stated sizes; *bad receives 1 on a violation.
static __global__ void csr_check_kernel(int n, int nnz, const int* ptr, const int* idx, int* bad) {
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
    int b = 0;
    if (gtid == 0 && (ptr[0] != 0 || ptr[n] != nnz)) b = 1;
    for (int i = gtid; i < n; i += gs)
        if (ptr[i + 1] < ptr[i]) b = 1;
    for (int k = gtid; k < nnz; k += gs) {
        const int j = idx[k];
        if (j < 0 || j >= n) b = 1;
    }
    if (b) atomicExch(bad, 1);
}

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
    double* psmall;                        // [n_small] (E x) on the small rows, refreshed per apply

    // warp-cooperative values of the small rows: psmall[s] = E[small s, :] x
    __device__ __forceinline__ void small_rows(const double* x) const {
        const int lane = threadIdx.x & 31;
        const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        const int nw = (gridDim.x * blockDim.x) >> 5;
        for (int s = gw; s < n_small; s += nw) {
            double acc = 0.0;
            const int k1 = __ldg(small_ptr + s + 1);
            for (int k = __ldg(small_ptr + s) + lane; k < k1; k += 32) acc += __ldg(small_val + k) * __ldcg(x + __ldg(small_idx + k));
            acc = warp_sum(acc);
            if (lane == 0) psmall[s] = acc;
        }
    }

    // psmall[s] = E[small s, :] p_new with p_new = D^-1 r + beta p_old formed
    // on the fly (the stored p_new is being written concurrently)
    __device__ __forceinline__ void small_rows_next(const double* pold, const double* r, const double* dinv,
                                                    double beta) const {
        const int lane = threadIdx.x & 31;
        const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        const int nw = (gridDim.x * blockDim.x) >> 5;
        for (int s = gw; s < n_small; s += nw) {
            double acc = 0.0;
            const int k1 = __ldg(small_ptr + s + 1);
            for (int k = __ldg(small_ptr + s) + lane; k < k1; k += 32) {
                const int j = __ldg(small_idx + k);
                acc += __ldg(small_val + k) * p_next(__ldg(dinv + j), __ldcg(r + j), beta, __ldcg(pold + j));
            }
            acc = warp_sum(acc);
            if (lane == 0) psmall[s] = acc;
        }
    }

    // psmall[s] = E[small s, :] p_new with p_new = z + beta p_old formed on
    // the fly (p_next_sum)
    __device__ __forceinline__ void small_rows_next_sum(const double* pold, const ZSum& z, double beta) const {
        const int lane = threadIdx.x & 31;
        const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        const int nw = (gridDim.x * blockDim.x) >> 5;
        for (int s = gw; s < n_small; s += nw) {
            double acc = 0.0;
            const int k1 = __ldg(small_ptr + s + 1);
            for (int k = __ldg(small_ptr + s) + lane; k < k1; k += 32) {
                const int j = __ldg(small_idx + k);
                acc += __ldg(small_val + k) * p_next_sum(z, j, beta, __ldcg(pold + j));
            }
            acc = warp_sum(acc);
            if (lane == 0) psmall[s] = acc;
        }
    }

    // (E x)_i once small_rows(x) has completed grid-wide
    __device__ __forceinline__ double gather_fast(const double* x, int i) const {
        const int r = __ldg(red_of_full + i);
        if (r >= 0) return __ldcg(x + r);
        const int s = __ldg(small_slot + i);
        return s >= 0 ? __ldcg(psmall + s) : 0.0;
    }

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
//
// y = E^T A E p in two phases separated by one grid barrier:
//
//  phase 1 (work items, claimed dynamically through one atomic counter):
//    - FULL tile (tile^3 uncut fluid elements): E-gather of the
//      (tile+p)^3 DOF window into shared memory, then the Kronecker sum with
//      tile-assembled 1D factors, 7 banded passes -> ypart[tile];
//    - MIXED tile: the same window, its uncut elements one per warp (7 passes
//      of (p+1)-wide 1D factors cached in shared memory), per-warp
//      accumulators summed in warp order -> ypart[tile];
//    - CUT chunk: dense (p+1)^3 blocks of cut elements, each multiplied by the
//      whole block (4 threads per row, interleaved columns) -> ycut[cut].
//  phase 2 (per reduced DOF j): y_j = sum over E's column j of the full-space
//    values, each full value = fixed-order sum of its <= 8 tile partials and
//    its cut-element partials.  No atomics; results are bit-reproducible.

enum { TILE_EMPTY = 0, TILE_FULL = 1, TILE_MIXED = 2 };

// Non-templated description shared by every precision / degree instance.
struct TileData {
    int n, p, T, nta, nb;
    int n_items;      // tile work items: mixed tiles (heaviest first), then full tiles
    int n_mixed;      // leading mixed-tile items; the rest are full tiles
    int full_warp;    // 1: full tiles are warp-level items (many per SM); 0: block-level
    int lane1;        // 1: one thread per DOF / row in phase 2 (many per thread); 0: groups of 4 lanes
    int n_cut;
    int cut_chunk;    // cut elements per work item
    double a_mass;
    const int* item_list;  // >= 0: tile id; < 0: cut chunk -(k+1)
    const int* tile_kind;
    const int* tile_eptr;
    const int* tile_elem;
    const int* tile_ecut;  // unused by the device (cut elements are separate items)
    const double* M1;
    const double* Kt1;
    const double* TM;
    const double* TA;
    const double* TK;
    const int* cut_base;       // [n_cut] full DOF index of the element's first DOF
    const int* cut_dof_slot;   // [n_full] slot in the DOF -> cut list, -1 if none
    const int* cut_dof_ptr;    // [n_slots + 1]
    const int* cut_dof_ent;    // cut * P + local
    ExtDev ext;
    double* ypart;             // [NS][n_full] tile partials: one plane per covering-tile slot
    double* ycut;              // [n_cut * P] cut partials in DOF-list order (cut_dof_ent order)
    const int* cut_pos;        // [n_cut * P] position of (cut, local row) in ycut
    double* yfv;               // [n_full] full-space values of the needed DOFs
    const int* need;           // [n_need] full DOFs read by the E^T scatter
    int n_need;
    // phase-2 records (built by the host at create): those with a list first,
    // longest first, then those without, in index order
    const int4* need_rec;      // [n_need] {full DOF, row it completes or -1, cut partials [z, w) in ycut}
    const int4* row_rec;       // [n_red] {reduced row, its full DOF, E^T entries [z, w)}
    int n_need_heavy;          // leading records whose lists are long (4 lanes each when lane1)
    int n_row_heavy;
    int n_need_list;           // leading records with a non-empty list
    int n_row_list;
    unsigned* work;            // dynamic tile-item counter (reset in phase 2)
    unsigned* work2;           // dynamic cut-element counter, claimed per warp
};

// Storage of the symmetric 64 x 64 cut-element blocks of degree 3 (2080
// entries, half of the dense block): with A split into 32 x 32 blocks
// [[A00, A01], [A01^T, A11]],
//   [0, 528)      A00 upper triangle, entry (a, b), a <= b, at b(b+1)/2 + a
//   [528, 1040)   A01 columns 0..15 \ entry (a, c) of A01 at
//   [1040, 1552)  A01 columns 16..31 / (c & 15) * 32 + ((a + c) & 31)
//   [1552, 2080)  A11 upper triangle, packed like A00.
// Triangular numbers b(b+1)/2 are distinct modulo 32 for b < 32, and the
// (a + c) & 31 rotation spreads both a row and a column of A01 over all
// banks, so every shared-memory walk below is (nearly) conflict free.  Every
// chunk start and the element stride are multiples of 16 bytes in 8-, 4- and
// 2-byte storage.
constexpr int SYM64_ENTRIES = 2080;
__host__ __device__ constexpr int sym64_index(int i, int j) {
    const int a = i < j ? i : j, b = i < j ? j : i;
    if (b < 32) return b * (b + 1) / 2 + a;
    if (a >= 32) return 1552 + (b - 32) * (b - 31) / 2 + (a - 32);
    const int c = b - 32;
    return 528 + (c >> 4) * 512 + (c & 15) * 32 + ((a + c) & 31);
}

template <typename CT, int P1>
struct TileOp {
    static constexpr bool kFusedP = true;
    static constexpr int kDegree1 = P1;  // p + 1
    static constexpr int P = P1 * P1 * P1;
    static constexpr int PP = P1 * P1;
    static constexpr int T = 4;
    static constexpr int D = T + P1 - 1;
    static constexpr int D3 = D * D * D;
    static constexpr int NW = CUTCELL_WARPS;
    // shared-memory sub-arrays start on 16-byte boundaries (even double counts)
    static constexpr int D3a = (D3 + 1) & ~1;
    static constexpr int Pa = (P + 1) & ~1;
    static constexpr int CTRL = 2;  // doubles reserved for the work-item slot
    // degree 3 stores its cut blocks in the symmetric split layout above
    static constexpr bool kSym = (P1 == 4);
    static constexpr int CUT_ENTRIES = kSym ? SYM64_ENTRIES : P * P;
    // tiles covering one DOF per axis (2 for D <= 2T, 3 for p = 5) and the
    // DOF-major partial slots per DOF
    static constexpr int NC = (D + T - 1) / T;
    static constexpr int NS = NC * NC * NC;
    TileData td;

    // Entry k of the window of tile (tx, ty, tz) is stored in slot plane
    // m = (bz NC + by) NC + bx at its DOF, b = t1 - t per axis with t1 the
    // DOF's last covering tile (min(g / T, nta - 1)); every (DOF, tile) pair
    // has its own slot, slots of absent tiles stay zero, and the gather sums
    // a DOF's NS slots in order.  Entries outside the grid are dropped.  Runs
    // of x-neighbours land in consecutive addresses of one plane, and so do
    // the gather's loads for consecutive DOFs.
    __device__ __forceinline__ void put_partial(int tx, int ty, int tz, int k, double v) const {
        const int dx = k % D, dy = (k / D) % D, dz = k / (D * D);
        const int gx = tx * T + dx, gy = ty * T + dy, gz = tz * T + dz;
        const int nb = td.nb, nta = td.nta;
        if (gx >= nb || gy >= nb || gz >= nb) return;
        const int bx = min(gx / T, nta - 1) - tx, by = min(gy / T, nta - 1) - ty, bz = min(gz / T, nta - 1) - tz;
        td.ypart[(size_t)((bz * NC + by) * NC + bx) * td.ext.n_full + (gz * nb + gy) * nb + gx] = v;
    }
    const CT* __restrict__ cut_mats;

    // per-warp region of a warp-level item: a full tile's window and three
    // pass buffers, or a cut element's gathered values
    static constexpr int WS = (4 * D3a > Pa) ? 4 * D3a : Pa;
    static size_t smem_bytes() {
        const size_t mixed = (size_t)D3a + (size_t)2 * NW * D3a + (size_t)2 * NW * 4 * Pa + 3 * 4 * 2 * PP;
        const size_t full = 5 * (size_t)D3a;
        const size_t warp = (size_t)NW * WS;
        size_t m = mixed > warp ? mixed : warp;
        return (CTRL + (m > full ? m : full)) * sizeof(double);
    }

    __device__ __forceinline__ void gather_window(const double* pred, int tx, int ty, int tz, double* xs) const {
        const int nb = td.nb;
        for (int k = threadIdx.x; k < D3; k += blockDim.x) {
            const int dx = k % D, dy = (k / D) % D, dz = k / (D * D);
            const int gx = tx * T + dx, gy = ty * T + dy, gz = tz * T + dz;
            double v = 0.0;
            if (gx < nb && gy < nb && gz < nb) v = td.ext.gather_fast(pred, (gz * nb + gy) * nb + gx);
            xs[k] = v;
        }
    }

    // A full tile by the whole block (few tiles per block: latency matters).
    __device__ void full_tile(int tx, int ty, int tz, double* xs) const {
        double* u1 = xs + D3a;
        double* u2 = u1 + D3a;
        double* v1 = u2 + D3a;
        double* v2 = v1 + D3a;
        const int nta = td.nta;
        const double* Mx = td.TM + (size_t)tx * D * D;
        const double* Ax = td.TA + (size_t)tx * D * D;
        const double* My = td.TM + (size_t)ty * D * D;
        const double* Ky = td.TK + ((size_t)1 * nta + ty) * D * D;
        const double* Mz = td.TM + (size_t)tz * D * D;
        const double* Kz = td.TK + ((size_t)2 * nta + tz) * D * D;
        constexpr int p = P1 - 1;
        for (int k = threadIdx.x; k < D3; k += blockDim.x) {
            const int i = k % D, row = k - i;
            double s1 = 0.0, s2 = 0.0;
#pragma unroll
            for (int o = -p; o <= p; ++o) {
                const int j = i + o;
                if (j >= 0 && j < D) {
                    const double xv = xs[row + j];
                    s1 += __ldg(Mx + i * D + j) * xv;
                    s2 += __ldg(Ax + i * D + j) * xv;
                }
            }
            u1[k] = s1;
            u2[k] = s2;
        }
        __syncthreads();
        for (int k = threadIdx.x; k < D3; k += blockDim.x) {
            const int x = k % D, i = (k / D) % D, z = k / (D * D);
            double s1 = 0.0, s2 = 0.0;
#pragma unroll
            for (int o = -p; o <= p; ++o) {
                const int j = i + o;
                if (j >= 0 && j < D) {
                    const int q = (z * D + j) * D + x;
                    const double m = __ldg(My + i * D + j);
                    s1 += m * u1[q];
                    s2 += m * u2[q] + __ldg(Ky + i * D + j) * u1[q];
                }
            }
            v1[k] = s1;
            v2[k] = s2;
        }
        __syncthreads();
        for (int k = threadIdx.x; k < D3; k += blockDim.x) {
            const int xy = k % (D * D), i = k / (D * D);
            double s = 0.0;
#pragma unroll
            for (int o = -p; o <= p; ++o) {
                const int j = i + o;
                if (j >= 0 && j < D) {
                    const int q = j * D * D + xy;
                    s += __ldg(Mz + i * D + j) * v2[q] + __ldg(Kz + i * D + j) * v1[q];
                }
            }
            put_partial(tx, ty, tz, k, s);
        }
    }

    // d += a b on the FP64 tensor cores (mma.sync m8n8k4, A 8x4 row-major, B
    // 4x8 column-major).  Fragments of lane = 4 g + t: A(g, t), B(t, g),
    // C(g, 2t) and C(g, 2t + 1).
    __device__ __forceinline__ static void dmma(double& d0, double& d1, double a, double b) {
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                     : "+d"(d0), "+d"(d1)
                     : "d"(a), "d"(b));
    }

    // The three banded passes of a full tile (window in xs, result to out) as
    // batched 1D products on the FP64 tensor cores, for D <= 8.  Each pass is
    // a (D^2 lines x D) by (D x D) product, lines in blocks of 8 (A), the 1D
    // factor transposed in B (its D x D block padded to 8 x 8 with zeros, held
    // in registers), the k dimension in ceil(D/4) steps:
    //   x: u1 = X Mx^T, u2 = X Ax^T            (line = (z, y), k = x)
    //   y: v1 = U1 My^T, v2 = U2 My^T + U1 Ky^T (line = (z, x), k = y)
    //   z: out = V2 Mz^T + V1 Kz^T               (line = (y, x), k = z)
    static constexpr int KS = (D + 3) / 4;
    static constexpr int NLB = (D * D + 7) / 8;
    // B fragments of the tile's six 1D factors, B(k = j, n = i) = F[i][j]:
    // [Mx, Ax, My, Ky, Mz, Kz][k step].  Loaded before the window gather so
    // their latency overlaps it.
    struct TileB {
        double f[6][KS];
    };
    __device__ __forceinline__ TileB tile_bfrags(int tx, int ty, int tz) const {
        const int lane = threadIdx.x & 31;
        const int g = lane >> 2, t4 = lane & 3;
        const int nta = td.nta;
        const double* F[6] = {td.TM + (size_t)tx * D * D, td.TA + (size_t)tx * D * D,
                              td.TM + (size_t)ty * D * D, td.TK + ((size_t)1 * nta + ty) * D * D,
                              td.TM + (size_t)tz * D * D, td.TK + ((size_t)2 * nta + tz) * D * D};
        TileB b;
#pragma unroll
        for (int m = 0; m < 6; ++m)
#pragma unroll
            for (int ks = 0; ks < KS; ++ks) {
                const int i = g, j = 4 * ks + t4;
                b.f[m][ks] = (i < D && j < D) ? __ldg(F[m] + i * D + j) : 0.0;
            }
        return b;
    }

    __device__ void full_tile_passes_mma(const TileB& b, int tile, double* ws) const {
        static_assert(D <= 8, "tensor-core passes need D <= 8");
        const int lane = threadIdx.x & 31;
        const int g = lane >> 2, t4 = lane & 3;
        double* xs = ws;
        double* u1 = ws + D3a;
        double* u2 = u1 + D3a;
        double* v2 = u2 + D3a;
        double* v1 = xs;  // the window is dead after the x pass
        const double* bMx = b.f[0];
        const double* bAx = b.f[1];
        const double* bMy = b.f[2];
        const double* bKy = b.f[3];
        const double* bMz = b.f[4];
        const double* bKz = b.f[5];
        constexpr int L = D * D;
        const int c0 = 2 * t4;  // this lane's two output columns c0, c0 + 1
        // x pass: A(line, j) = xs[line * D + j]
#pragma unroll 1
        for (int mb = 0; mb < NLB; ++mb) {
            const int line = 8 * mb + g;
            double p0 = 0.0, p1 = 0.0, q0 = 0.0, q1 = 0.0;
#pragma unroll
            for (int ks = 0; ks < KS; ++ks) {
                const int j = 4 * ks + t4;
                const double a = (line < L && j < D) ? xs[line * D + j] : 0.0;
                dmma(p0, p1, a, bMx[ks]);
                dmma(q0, q1, a, bAx[ks]);
            }
            if (line < L) {
                if (c0 < D) {
                    u1[line * D + c0] = p0;
                    u2[line * D + c0] = q0;
                }
                if (c0 + 1 < D) {
                    u1[line * D + c0 + 1] = p1;
                    u2[line * D + c0 + 1] = q1;
                }
            }
        }
        __syncwarp();
        // y pass: line = (z, x), A(line, j) = U[(z * D + j) * D + x]
#pragma unroll 1
        for (int mb = 0; mb < NLB; ++mb) {
            const int line = 8 * mb + g;
            const int z = line / D, x = line - z * D;
            double p0 = 0.0, p1 = 0.0, q0 = 0.0, q1 = 0.0;
#pragma unroll
            for (int ks = 0; ks < KS; ++ks) {
                const int j = 4 * ks + t4;
                const bool ok = line < L && j < D;
                const double a1 = ok ? u1[(z * D + j) * D + x] : 0.0;
                const double a2 = ok ? u2[(z * D + j) * D + x] : 0.0;
                dmma(p0, p1, a1, bMy[ks]);
                dmma(q0, q1, a2, bMy[ks]);
                dmma(q0, q1, a1, bKy[ks]);
            }
            if (line < L) {
                if (c0 < D) {
                    v1[(z * D + c0) * D + x] = p0;
                    v2[(z * D + c0) * D + x] = q0;
                }
                if (c0 + 1 < D) {
                    v1[(z * D + c0 + 1) * D + x] = p1;
                    v2[(z * D + c0 + 1) * D + x] = q1;
                }
            }
        }
        __syncwarp();
        // z pass: line = (y, x), A(line, j) = V[j * D * D + line]
        const int nta = td.nta;
        const int tx = tile % nta, ty = (tile / nta) % nta, tz = tile / (nta * nta);
#pragma unroll 1
        for (int mb = 0; mb < NLB; ++mb) {
            const int line = 8 * mb + g;
            double p0 = 0.0, p1 = 0.0;
#pragma unroll
            for (int ks = 0; ks < KS; ++ks) {
                const int j = 4 * ks + t4;
                const bool ok = line < L && j < D;
                const double a2 = ok ? v2[j * L + line] : 0.0;
                const double a1 = ok ? v1[j * L + line] : 0.0;
                dmma(p0, p1, a2, bMz[ks]);
                dmma(p0, p1, a1, bKz[ks]);
            }
            if (line < L) {
                if (c0 < D) put_partial(tx, ty, tz, c0 * L + line, p0);
                if (c0 + 1 < D) put_partial(tx, ty, tz, (c0 + 1) * L + line, p1);
            }
        }
        __syncwarp();
    }

    // A full tile by one warp: E-gather of the D^3 window, then the x, y, z
    // banded passes with __syncwarp between them (no block barrier), so a
    // block has NW tiles in flight: on the FP64 tensor cores for D <= 8, else
    // per lane, where every loop has a compile-time trip count (KPL entries)
    // and is unrolled, so a lane's loads are all in flight together.
    // ws: 4 * D3a doubles.
    static constexpr int KPL = (D3 + 31) / 32;
    __device__ void full_tile_warp(const double* pred, int tile, double* ws) const {
        const int lane = threadIdx.x & 31;
        const int nta = td.nta, nb = td.nb;
        const int tx = tile % nta, ty = (tile / nta) % nta, tz = tile / (nta * nta);
        double* xs = ws;
        double* u1 = ws + D3a;
        double* u2 = u1 + D3a;
        double* v2 = u2 + D3a;
        double* v1 = xs;  // the window is dead after the x pass
        TileB bf;
        if constexpr (D <= 8) bf = tile_bfrags(tx, ty, tz);
        {
            int gi[KPL];
#pragma unroll
            for (int t = 0; t < KPL; ++t) {
                const int k = lane + 32 * t;
                const int dx = k % D, dy = (k / D) % D, dz = k / (D * D);
                const int gx = tx * T + dx, gy = ty * T + dy, gz = tz * T + dz;
                gi[t] = (k < D3 && gx < nb && gy < nb && gz < nb) ? (gz * nb + gy) * nb + gx : -1;
            }
            int rr[KPL];
#pragma unroll
            for (int t = 0; t < KPL; ++t) rr[t] = gi[t] >= 0 ? __ldg(td.ext.red_of_full + gi[t]) : -1;
            double xv[KPL];
#pragma unroll
            for (int t = 0; t < KPL; ++t) {
                if (rr[t] >= 0)
                    xv[t] = __ldcg(pred + rr[t]);
                else if (gi[t] >= 0) {
                    const int sl = __ldg(td.ext.small_slot + gi[t]);
                    xv[t] = sl >= 0 ? __ldcg(td.ext.psmall + sl) : 0.0;
                } else
                    xv[t] = 0.0;
            }
#pragma unroll
            for (int t = 0; t < KPL; ++t)
                if (lane + 32 * t < D3) xs[lane + 32 * t] = xv[t];
        }
        __syncwarp();
        if constexpr (D <= 8) {
            full_tile_passes_mma(bf, tile, ws);
            return;
        }
        const double* Mx = td.TM + (size_t)tx * D * D;
        const double* Ax = td.TA + (size_t)tx * D * D;
        const double* My = td.TM + (size_t)ty * D * D;
        const double* Ky = td.TK + ((size_t)1 * nta + ty) * D * D;
        const double* Mz = td.TM + (size_t)tz * D * D;
        const double* Kz = td.TK + ((size_t)2 * nta + tz) * D * D;
        constexpr int p = P1 - 1;
#pragma unroll
        for (int t = 0; t < KPL; ++t) {
            const int k = lane + 32 * t;
            if (k < D3) {
                const int i = k % D, row = k - i;
                double s1 = 0.0, s2 = 0.0;
#pragma unroll
                for (int o = -p; o <= p; ++o) {
                    const int j = i + o;
                    if (j >= 0 && j < D) {
                        const double xv = xs[row + j];
                        s1 += __ldg(Mx + i * D + j) * xv;
                        s2 += __ldg(Ax + i * D + j) * xv;
                    }
                }
                u1[k] = s1;
                u2[k] = s2;
            }
        }
        __syncwarp();
#pragma unroll
        for (int t = 0; t < KPL; ++t) {
            const int k = lane + 32 * t;
            if (k < D3) {
                const int x = k % D, i = (k / D) % D, z = k / (D * D);
                double s1 = 0.0, s2 = 0.0;
#pragma unroll
                for (int o = -p; o <= p; ++o) {
                    const int j = i + o;
                    if (j >= 0 && j < D) {
                        const int q = (z * D + j) * D + x;
                        const double m = __ldg(My + i * D + j);
                        s1 += m * u1[q];
                        s2 += m * u2[q] + __ldg(Ky + i * D + j) * u1[q];
                    }
                }
                v1[k] = s1;
                v2[k] = s2;
            }
        }
        __syncwarp();
#pragma unroll
        for (int t = 0; t < KPL; ++t) {
            const int k = lane + 32 * t;
            if (k < D3) {
                const int xy = k % (D * D), i = k / (D * D);
                double s = 0.0;
#pragma unroll
                for (int o = -p; o <= p; ++o) {
                    const int j = i + o;
                    if (j >= 0 && j < D) {
                        const int q = j * D * D + xy;
                        s += __ldg(Mz + i * D + j) * v2[q] + __ldg(Kz + i * D + j) * v1[q];
                    }
                }
                put_partial(tx, ty, tz, k, s);
            }
        }
        __syncwarp();
    }

    // Uncut elements of a mixed tile for p = 3, one element per warp on the
    // FP64 tensor cores (the element's 4-point lines fill k = 4 exactly), so
    // a block has NW elements in flight.  Each pass is one or two m8n8k4
    // products per 8 lines, the two factors a pass needs side by side in the
    // n dimension:
    //   x: [u1 | u2] = X [Mx^T | Ax^T]                 (line = (z, y))
    //   y: [e3 | e0] = U1 [My^T | Ky^T] + U2 [0 | My^T] (line = (z, x))
    //   z: s = E0 Mz^T + E3 Kz^T                        (line = (y, x))
    // Each warp accumulates into its own window, summed in a fixed order.
    // The tile's 1D element factors into shared memory and the per-warp
    // windows zeroed; independent of the window gather, so phase 1 issues it
    // before the barrier that completes the gather.
    __device__ void mixed_prep_mma(int tx, int ty, int tz, double* xs) const {
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        double* acc = xs + D3a + (size_t)warp * D3a;
        double* fac = xs + D3a + (size_t)NW * D3a + (size_t)NW * 4 * Pa;  // [axis][4 pos][M, K~][PP]
        const int n = td.n;
        for (int k = threadIdx.x; k < 3 * 4 * 2 * PP; k += blockDim.x) {
            const int e = k % PP, w = (k / PP) % 2, pos = (k / (2 * PP)) % 4, ax = k / (8 * PP);
            const int t = ax == 0 ? tx : (ax == 1 ? ty : tz);
            const int el = min(t * T + pos, n - 1);
            double v = w == 0 ? __ldg(td.M1 + (size_t)el * PP + e) : __ldg(td.Kt1 + ((size_t)ax * n + el) * PP + e);
            if (ax == 0 && w == 1) v += td.a_mass * __ldg(td.M1 + (size_t)el * PP + e);  // a M + K~ on x
            fac[k] = v;
        }
        for (int k = lane; k < D3; k += 32) acc[k] = 0.0;
    }

    // (after mixed_prep_mma and a block barrier)
    __device__ void mixed_tile_mma(int tile, int tx, int ty, int tz, double* xs) const {
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int g = lane >> 2, t4 = lane & 3;
        double* acc = xs + D3a + (size_t)warp * D3a;
        double* u1 = xs + D3a + (size_t)NW * D3a + (size_t)warp * 4 * Pa;  // [line (z, y)][x]
        double* u2 = u1 + Pa;
        double* e3 = u2 + Pa;  // [z][i = y][x]
        double* e0 = e3 + Pa;
        const double* fac = xs + D3a + (size_t)NW * D3a + (size_t)NW * 4 * Pa;
        const int hi = g >> 2, gi = g & 3;  // B column g: factor hi, row gi
        const int eb = __ldg(td.tile_eptr + tile), ee = __ldg(td.tile_eptr + tile + 1);
        for (int it = eb + warp; it < ee; it += NW) {
            const int le = __ldg(td.tile_elem + it);
            const int lx = le % T, ly = (le / T) % T, lz = le / (T * T);
            const double* fx = fac + (0 * 4 + lx) * 2 * PP;  // M, then a M + K~
            const double* fy = fac + (1 * 4 + ly) * 2 * PP;
            const double* fz = fac + (2 * 4 + lz) * 2 * PP;
            // B(k = t4, n = g) fragments
            const double bx = fx[hi * PP + gi * P1 + t4];
            const double by1 = fy[hi * PP + gi * P1 + t4];
            const double by2 = hi ? fy[gi * P1 + t4] : 0.0;
            const double bz1 = hi ? 0.0 : fz[gi * P1 + t4];
            const double bz2 = hi ? 0.0 : fz[PP + gi * P1 + t4];
            const int c0 = 2 * t4;
            __syncwarp();  // the previous element's buffers are free
#pragma unroll
            for (int mb = 0; mb < 2; ++mb) {  // x pass, line = (z, y) = 8 mb + g
                const int line = 8 * mb + g, z = line >> 2, y = line & 3;
                const double a = xs[((lz + z) * D + (ly + y)) * D + (lx + t4)];
                double d0 = 0.0, d1 = 0.0;
                dmma(d0, d1, a, bx);
                double* dst = (c0 < P1 ? u1 : u2) + line * P1 + (c0 & 3);
                dst[0] = d0;
                dst[1] = d1;
            }
            __syncwarp();
#pragma unroll
            for (int mb = 0; mb < 2; ++mb) {  // y pass, line = (z, x)
                const int line = 8 * mb + g, z = line >> 2, x = line & 3;
                const double a1 = u1[(z * P1 + t4) * P1 + x];
                const double a2 = u2[(z * P1 + t4) * P1 + x];
                double d0 = 0.0, d1 = 0.0;
                dmma(d0, d1, a1, by1);
                dmma(d0, d1, a2, by2);
                double* dst = (c0 < P1 ? e3 : e0) + (z * P1 + (c0 & 3)) * P1 + x;
                dst[0] = d0;
                dst[P1] = d1;
            }
            __syncwarp();
#pragma unroll
            for (int mb = 0; mb < 2; ++mb) {  // z pass, line = (y, x)
                const int line = 8 * mb + g;
                const double a1 = e0[t4 * PP + line];
                const double a2 = e3[t4 * PP + line];
                double d0 = 0.0, d1 = 0.0;
                dmma(d0, d1, a1, bz1);
                dmma(d0, d1, a2, bz2);
                if (c0 < P1) {  // columns 0..3 carry the element's output rows i = c0, c0 + 1
                    const int y = line >> 2, x = line & 3;
                    double* dst = acc + ((lz + c0) * D + (ly + y)) * D + (lx + x);
                    dst[0] += d0;
                    dst[D * D] += d1;
                }
            }
        }
        __syncthreads();
        double* acc0 = xs + D3a;
        for (int k = threadIdx.x; k < D3; k += blockDim.x) {
            double s = 0.0;
#pragma unroll
            for (int w = 0; w < NW; ++w) s += acc0[(size_t)w * D3a + k];
            put_partial(tx, ty, tz, k, s);
        }
    }

    // Uncut elements of a mixed tile, one per half-warp (16 lanes), so a block
    // has 2 NW elements in flight; each half-warp accumulates into its own
    // window, summed in a fixed order at the end.  p = 3 runs mixed_tile_mma.
    static constexpr int NH = 2 * NW;  // half-warps per block
    __device__ void mixed_tile(int tile, int tx, int ty, int tz, double* xs) const {
        if constexpr (P1 == 4) {
            mixed_tile_mma(tile, tx, ty, tz, xs);
            return;
        }
        const int half = threadIdx.x >> 4, hl = threadIdx.x & 15;
        const unsigned hmask = 0xffffu << (16 * ((threadIdx.x >> 4) & 1));
        double* acc = xs + D3a + (size_t)half * D3a;
        double* e0 = xs + D3a + (size_t)NH * D3a + (size_t)half * 4 * Pa;
        double* e1 = e0 + Pa;
        double* e2 = e1 + Pa;
        double* e3 = e2 + Pa;
        double* fac = xs + D3a + (size_t)NH * D3a + (size_t)NH * 4 * Pa;  // [axis][4 pos][M, K~][PP]
        const int n = td.n;
        for (int k = threadIdx.x; k < 3 * 4 * 2 * PP; k += blockDim.x) {
            const int e = k % PP, w = (k / PP) % 2, pos = (k / (2 * PP)) % 4, ax = k / (8 * PP);
            const int t = ax == 0 ? tx : (ax == 1 ? ty : tz);
            const int el = min(t * T + pos, n - 1);
            double v = w == 0 ? __ldg(td.M1 + (size_t)el * PP + e) : __ldg(td.Kt1 + ((size_t)ax * n + el) * PP + e);
            if (ax == 0 && w == 1) v += td.a_mass * __ldg(td.M1 + (size_t)el * PP + e);  // a M + K~ on x
            fac[k] = v;
        }
        for (int k = hl; k < D3; k += 16) acc[k] = 0.0;
        __syncthreads();
        const int eb = __ldg(td.tile_eptr + tile), ee = __ldg(td.tile_eptr + tile + 1);
        for (int it = eb + half; it < ee; it += NH) {
            const int le = __ldg(td.tile_elem + it);
            const int lx = le % T, ly = (le / T) % T, lz = le / (T * T);
            const double* Mx = fac + ((0 * 4 + lx) * 2 + 0) * PP;
            const double* Ax = fac + ((0 * 4 + lx) * 2 + 1) * PP;
            const double* My = fac + ((1 * 4 + ly) * 2 + 0) * PP;
            const double* Ky = fac + ((1 * 4 + ly) * 2 + 1) * PP;
            const double* Mz = fac + ((2 * 4 + lz) * 2 + 0) * PP;
            const double* Kz = fac + ((2 * 4 + lz) * 2 + 1) * PP;
            __syncwarp(hmask);
            for (int k = hl; k < P; k += 16) {
                const int a = k % P1, b = (k / P1) % P1, c = k / PP;
                e0[k] = xs[((lz + c) * D + (ly + b)) * D + (lx + a)];
            }
            __syncwarp(hmask);
            for (int k = hl; k < P; k += 16) {
                const int i = k % P1, row = k - i;
                double s1 = 0.0, s2 = 0.0;
#pragma unroll
                for (int j = 0; j < P1; ++j) {
                    s1 += Mx[i * P1 + j] * e0[row + j];
                    s2 += Ax[i * P1 + j] * e0[row + j];
                }
                e1[k] = s1;
                e2[k] = s2;
            }
            __syncwarp(hmask);
            for (int k = hl; k < P; k += 16) {
                const int x = k % P1, i = (k / P1) % P1, z = k / PP;
                double s1 = 0.0, s2 = 0.0;
#pragma unroll
                for (int j = 0; j < P1; ++j) {
                    const int q = (z * P1 + j) * P1 + x;
                    s1 += My[i * P1 + j] * e1[q];
                    s2 += My[i * P1 + j] * e2[q] + Ky[i * P1 + j] * e1[q];
                }
                e3[k] = s1;
                e0[k] = s2;
            }
            __syncwarp(hmask);
            for (int k = hl; k < P; k += 16) {
                const int xy = k % PP, i = k / PP;
                double s = 0.0;
#pragma unroll
                for (int j = 0; j < P1; ++j) {
                    const int q = j * PP + xy;
                    s += Mz[i * P1 + j] * e0[q] + Kz[i * P1 + j] * e3[q];
                }
                acc[((lz + i) * D + (ly + xy / P1)) * D + (lx + xy % P1)] += s;
            }
        }
        __syncthreads();
        double* acc0 = xs + D3a;
        for (int k = threadIdx.x; k < D3; k += blockDim.x) {
            double s = 0.0;
#pragma unroll
            for (int w = 0; w < NH; ++w) s += acc0[(size_t)w * D3a + k];
            put_partial(tx, ty, tz, k, s);
        }
    }

    // one cut element per warp: x_e gathered through E into the warp's
    // shared slice, y_e = A_e x_e with lane-owned rows (A_e symmetric, so
    // column c of the row-major block is row c: for fixed c the 32 lanes read
    // 32 consecutive entries), ceil(P/32) independent accumulators per lane.
    static constexpr int RPL = (P + 31) / 32;
    // Dense cut-element block product by one warp.  When a column of the block
    // is a whole number of 16-byte pieces (p = 3 in every storage type), the
    // block is streamed through two shared-memory chunk buffers with 16-byte
    // cp.async copies: the next chunk is in flight while the current one is
    // multiplied, so each warp keeps about 10 KB of loads outstanding (the
    // completion wait is cp.async.wait_group, a hardware wait).
    __device__ void cut_element_warp(const double* pred, int c, double* xe) const {
        typedef typename Conv<CT>::acc acc_t;
        const int lane = threadIdx.x & 31;
        const int nb = td.nb;
        const int base = __ldg(td.cut_base + c);
        auto gather = [&]() {
#pragma unroll
            for (int t = 0; t < RPL; ++t) {
                const int k = lane + 32 * t;
                if (k < P) {
                    const int a = k % P1, b = (k / P1) % P1, cc = k / PP;
                    xe[k] = td.ext.gather_fast(pred, base + (cc * nb + b) * nb + a);
                }
            }
        };
        const CT* A = cut_mats + (size_t)c * CUT_ENTRIES;
        acc_t acc[RPL];
#pragma unroll
        for (int q = 0; q < RPL; ++q) acc[q] = 0;
        constexpr int COLB = P * (int)sizeof(CT);  // bytes per column
        if constexpr (kSym) {
            // four chunks (A00, A01 left, A01 right, A11) through two buffers;
            // lane l owns rows l (acc[0]) and 32 + l (acc[1]) and adds every
            // row's terms in ascending column order, as the dense product does
            constexpr int SLOT = 528 * (int)sizeof(CT);  // bytes per buffer (largest chunk)
            static_assert(Pa + 2 * 528 * (int)sizeof(CT) / 8 <= WS, "chunk buffers exceed the warp slice");
            char* bufs = reinterpret_cast<char*>(xe + Pa);
            const char* src = reinterpret_cast<const char*>(A);
            auto issue = [&](int ch) {
                const int e0 = ch == 0 ? 0 : (ch == 1 ? 528 : (ch == 2 ? 1040 : 1552));
                const int bytes = (ch == 0 || ch == 3 ? 528 : 512) * (int)sizeof(CT);
                char* dst = bufs + (ch & 1) * SLOT;
                const char* s = src + (size_t)e0 * sizeof(CT);
                for (int off = lane * 16; off < bytes; off += 32 * 16) {
                    const unsigned d = (unsigned)__cvta_generic_to_shared(dst + off);
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(s + off) : "memory");
                }
                asm volatile("cp.async.commit_group;\n" ::: "memory");
            };
            const int tl = lane * (lane + 1) / 2;
            issue(0);  // the first two chunks stream in while x_e is gathered
            issue(1);
            gather();
            __syncwarp();  // xe complete
#pragma unroll 1
            for (int ch = 0; ch < 4; ++ch) {
                if (ch < 3)
                    asm volatile("cp.async.wait_group 1;\n" ::: "memory");
                else
                    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
                __syncwarp();  // every lane's pieces of chunk ch have landed
                const CT* S = reinterpret_cast<const CT*>(bufs + (ch & 1) * SLOT);
                if (ch == 0 || ch == 3) {  // diagonal block: the whole row of lane l
                    const int q = ch == 0 ? 0 : 1;
                    const double* xs = xe + 32 * q;
                    int tc = 0;
#pragma unroll 8
                    for (int cc = 0; cc < 32; ++cc) {
                        const int a = cc >= lane ? tc + lane : tl + cc;
                        acc[q] += Conv<CT>::sld(S + a) * (acc_t)xs[cc];
                        tc += cc + 1;
                    }
                } else {
                    const int cb = (ch - 1) * 16;  // first A01 column of this chunk
                    // row walk: row l of A01, columns cb .. cb + 15 (global 32 + c)
#pragma unroll 8
                    for (int cc = 0; cc < 16; ++cc) {
                        const int cg = cb + cc;
                        acc[0] += Conv<CT>::sld(S + cc * 32 + ((lane + cg) & 31)) * (acc_t)xe[32 + cg];
                    }
                    // column walk: lanes whose A01 column lies in this chunk form
                    // (A01^T x_0)_l, which precedes A11 in row 32 + l
                    if ((lane >> 4) == ch - 1) {
                        const int cl = lane & 15;
#pragma unroll 8
                        for (int r = 0; r < 32; ++r)
                            acc[1] += Conv<CT>::sld(S + cl * 32 + ((r + lane) & 31)) * (acc_t)xe[r];
                    }
                }
                __syncwarp();  // buffer (ch & 1) is free again
                if (ch + 2 < 4) issue(ch + 2);
            }
        } else if constexpr (COLB % 16 == 0) {
            gather();
            constexpr int BUFB = ((WS - Pa) * 8 / 2) / COLB * COLB;  // bytes per chunk buffer
            constexpr int CPC = BUFB / COLB;                         // columns per chunk
            constexpr int NCH = (P + CPC - 1) / CPC;
            static_assert(CPC >= 1, "chunk buffer holds no column");
            char* bufs = reinterpret_cast<char*>(xe + Pa);
            const char* src = reinterpret_cast<const char*>(A);
            auto issue = [&](int ch) {
                const int c0 = ch * CPC;
                const int bytes = min(CPC, P - c0) * COLB;
                char* dst = bufs + (ch & 1) * BUFB;
                const char* s = src + (size_t)c0 * COLB;
                for (int off = lane * 16; off < bytes; off += 32 * 16) {
                    const unsigned d = (unsigned)__cvta_generic_to_shared(dst + off);
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(s + off) : "memory");
                }
                asm volatile("cp.async.commit_group;\n" ::: "memory");
            };
            issue(0);
            __syncwarp();  // xe complete
            for (int ch = 0; ch < NCH; ++ch) {
                if (ch + 1 < NCH) {
                    issue(ch + 1);
                    asm volatile("cp.async.wait_group 1;\n" ::: "memory");
                } else {
                    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
                }
                __syncwarp();  // every lane's pieces of chunk ch have landed
                const CT* As = reinterpret_cast<const CT*>(bufs + (ch & 1) * BUFB);
                const int c0 = ch * CPC;
#pragma unroll 2
                for (int cl = 0; cl < CPC; ++cl) {
                    if (c0 + cl < P) {
                        const acc_t xv = (acc_t)xe[c0 + cl];
#pragma unroll
                        for (int q = 0; q < RPL; ++q)
                            if (lane + 32 * q < P) acc[q] += Conv<CT>::sld(As + cl * P + lane + 32 * q) * xv;
                    }
                }
                __syncwarp();  // chunk buffer (ch & 1) is refilled by issue(ch + 2)
            }
        } else {
            gather();
            __syncwarp();
#pragma unroll 8
            for (int col = 0; col < P; ++col) {
                const acc_t xv = (acc_t)xe[col];
                const CT* Ac = A + (size_t)col * P + lane;
#pragma unroll
                for (int q = 0; q < RPL; ++q)
                    if (lane + 32 * q < P) acc[q] += Conv<CT>::ld(Ac + 32 * q) * xv;
            }
        }
#pragma unroll
        for (int q = 0; q < RPL; ++q)
            if (lane + 32 * q < P) td.ycut[__ldg(td.cut_pos + (size_t)c * P + lane + 32 * q)] = (double)acc[q];
        __syncwarp();
    }

    __device__ void phase1(const double* pred, double* smem) const {
        int& s_item = *reinterpret_cast<int*>(smem);
        double* sm = smem + CTRL;
#ifdef CUTCELL_DEBUG_CHECKS
        unsigned* dbgw = (td.work + 64);
        if (threadIdx.x == 0) {
            CUTCELL_OK_IF(CUTCELL_ALIGNED(sm, 16), 1, 0, dbgw);
            CUTCELL_OK_IF(CUTCELL_ALIGNED(cut_mats, sizeof(CT)), 2, 0, dbgw);
            CUTCELL_OK_IF(CUTCELL_ALIGNED(td.ypart, 8) && CUTCELL_ALIGNED(td.ycut, 8), 3, 0, dbgw);
            CUTCELL_OK_IF(CUTCELL_ALIGNED(td.M1, 8) && CUTCELL_ALIGNED(td.Kt1, 8) && CUTCELL_ALIGNED(td.TM, 8) &&
                              CUTCELL_ALIGNED(td.TA, 8) && CUTCELL_ALIGNED(td.TK, 8),
                          4, 0, dbgw);
            CUTCELL_OK_IF(CUTCELL_ALIGNED(pred, 8), 5, 0, dbgw);
            CUTCELL_OK_IF(CUTCELL_ALIGNED(td.ext.small_val, 8) && CUTCELL_ALIGNED(td.ext.smallT_val, 8), 6, 0, dbgw);
            CUTCELL_OK_IF(CUTCELL_ALIGNED(&s_item, 4), 7, 0, dbgw);
        }
#else
        unsigned* dbgw = nullptr;
#endif
        (void)dbgw;
        // block-level items: mixed tiles, and the full tiles unless they are warp-level
        const int n_block_items = td.full_warp ? td.n_mixed : td.n_items;
        while (true) {
            if (threadIdx.x == 0) s_item = (int)atomicAdd(td.work, 1u);
            __syncthreads();
            const int item = s_item;
            __syncthreads();
            if (item >= n_block_items) break;
            if (!CUTCELL_OK_IF(item >= 0, 8, item, (td.work + 64))) break;
            const int tile = __ldg(td.item_list + item);
            const int nta = td.nta;
            if (!CUTCELL_OK_IF(tile < nta * nta * nta, 9, tile, (td.work + 64))) continue;
            const int tx = tile % nta, ty = (tile / nta) % nta, tz = tile / (nta * nta);
            double* xs = sm;
            gather_window(pred, tx, ty, tz, xs);
            if constexpr (P1 == 4) {
                if (item < td.n_mixed) mixed_prep_mma(tx, ty, tz, xs);
            }
            __syncthreads();
            if (item >= td.n_mixed)
                full_tile(tx, ty, tz, xs);
            else
                mixed_tile(tile, tx, ty, tz, xs);
            __syncthreads();
        }
        // warp-level items: cut elements, then (if warp-level) full tiles
        const int lane = threadIdx.x & 31;
        double* ws = sm + (size_t)(threadIdx.x >> 5) * WS;
        const int n_warp_items = td.n_cut + (td.full_warp ? td.n_items - td.n_mixed : 0);
        while (true) {
            int w = 0;
            if (lane == 0) w = (int)atomicAdd(td.work2, 1u);
            w = __shfl_sync(0xffffffffu, w, 0);
            if (w >= n_warp_items) break;
            if (w < td.n_cut)
                cut_element_warp(pred, w, ws);
            else
                full_tile_warp(pred, __ldg(td.item_list + td.n_mixed + (w - td.n_cut)), ws);
        }
        __syncthreads();
    }

    // full-space value of DOF rec.x: its NS tile-partial slots (one per plane)
    // and its cut partials [rec.z, rec.w) of ycut (contiguous), summed by G = 1 thread
    // or by the q-th of a group of G = 4 lanes (partials interleaved over the
    // lanes, then a fixed xor tree, so every lane of the group returns the
    // same bits).
    template <int G>
    __device__ __forceinline__ double yfull_rec(const int4 rec, int q) const {
        const double* yp = td.ypart + rec.x;
        const size_t plane = td.ext.n_full;
        double s = 0.0;
#pragma unroll
        for (int m = q; m < NS; m += G) s += __ldcg(yp + m * plane);
        int k = rec.z + q;
        if constexpr (G == 1) {
            for (; k + 4 <= rec.w; k += 4) {  // four loads in flight
                double v[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) v[u] = __ldcg(td.ycut + k + u);
#pragma unroll
                for (int u = 0; u < 4; ++u) s += v[u];
            }
        }
        for (; k < rec.w; k += G) s += __ldcg(td.ycut + k);
        if constexpr (G == 4) {
            s += __shfl_xor_sync(0xffffffffu, s, 1);
            s += __shfl_xor_sync(0xffffffffu, s, 2);
        }
        return s;
    }

    // (E^T yf) of row rec.x: the value of its own DOF rec.y and its E^T
    // entries [rec.z, rec.w), by G = 1 thread or a group of G = 4 lanes.
    template <int G>
    __device__ __forceinline__ double scatter_rec(const int4 rec, int q) const {
        double y = (q == 0) ? __ldcg(td.yfv + rec.y) : 0.0;
        int k = rec.z + q;
        if constexpr (G == 1) {
            for (; k + 4 <= rec.w; k += 4) {  // four entries' loads in flight
                int rw[4];
                double vv[4], yv[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    rw[u] = __ldg(td.ext.smallT_row + k + u);
                    vv[u] = __ldg(td.ext.smallT_val + k + u);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) yv[u] = __ldcg(td.yfv + rw[u]);
#pragma unroll
                for (int u = 0; u < 4; ++u) y += vv[u] * yv[u];
            }
        }
        for (; k < rec.w; k += G) y += __ldg(td.ext.smallT_val + k) * __ldcg(td.yfv + __ldg(td.ext.smallT_row + k));
        if constexpr (G == 4) {
            y += __shfl_xor_sync(0xffffffffu, y, 1);
            y += __shfl_xor_sync(0xffffffffu, y, 2);
        }
        return y;
    }

    // phase 0: small-row values of E p; phase 1: tiles and cut elements;
    // phase 2a: full-space values of the DOFs the scatter reads; phase 2b:
    // y = E^T yf and the partial of p.y.  Phase 2 walks the host-built
    // records (longest lists first): each DOF / row is owned by a group of 4
    // lanes (small problems, and the long lists of large ones) or by one thread.
    __device__ __forceinline__ double apply(const double* p, double* y, const GridSync& gs, double* sm) const {
        td.ext.small_rows(p);
        if (!grid_sync(gs)) return 0.0;
        return apply_tail(p, y, gs, sm);
    }

    // Phase 0 also forms p_new = D^-1 r + beta p_old for every reduced DOF
    // (written to pnew), its small rows computed from the same formula.
    __device__ __forceinline__ double apply_next(const double* pold, double* pnew, const double* r, const double* dinv,
                                                 double beta, double* y, const GridSync& gs, double* sm) const {
        const int n = td.ext.n_red;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            pnew[i] = p_next(__ldg(dinv + i), __ldcg(r + i), beta, __ldcg(pold + i));
        td.ext.small_rows_next(pold, r, dinv, beta);
        if (!grid_sync(gs)) return 0.0;
        return apply_tail(pnew, y, gs, sm);
    }

    // Phase 0 forms p_new = z + beta p_old (p_next_sum, z a sum of vectors) for
    // every reduced DOF and its small rows from the same formula, then the apply.
    __device__ __forceinline__ double apply_next_sum(const double* pold, double* pnew, const ZSum& z, double beta,
                                                     double* y, const GridSync& gs, double* sm) const {
        const int n = td.ext.n_red;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            pnew[i] = p_next_sum(z, i, beta, __ldcg(pold + i));
        td.ext.small_rows_next_sum(pold, z, beta);
        if (!grid_sync(gs)) return 0.0;
        return apply_tail(pnew, y, gs, sm);
    }

    // phases 1-2b of the apply (phase 0 has completed grid-wide)
    __device__ __forceinline__ double apply_tail(const double* p, double* y, const GridSync& gs, double* sm) const {
        phase1(p, sm);
        if (!grid_sync(gs)) return 0.0;
        if (blockIdx.x == 0 && threadIdx.x == 0) {  // every block has left phase 1
            *td.work = 0u;
            *td.work2 = 0u;
        }
        // Records [0, n4) by groups of 4 lanes (every listed record when there
        // are few per thread, else only the long lists), then the other listed
        // records one per thread; both dealt round-robin over the blocks
        // (record base + s owned by slot s = local * gridDim.x + block), so
        // every block gets an equal share of the long lists at the front.  The
        // unlisted records follow one per thread in index order (contiguous
        // lanes read contiguous partials).
        const int q = threadIdx.x & 3;
        const int gstride = gridDim.x * blockDim.x, ng = gstride >> 2;
        const int slot4 = (threadIdx.x >> 2) * gridDim.x + blockIdx.x;
        const int slot1 = threadIdx.x * gridDim.x + blockIdx.x;
        const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
        const int4 none = make_int4(0, -1, 0, 0);
        // a DOF whose row has no E^T entries completes that row here: y_j and
        // its p.y term; the others go to yfv for the scatter
        double part = 0.0;
        auto finish = [&](const int4& rec, double v) {
            if (rec.y >= 0) {
                y[rec.y] = v;
                part += __ldcg(p + rec.y) * v;
            } else {
                td.yfv[rec.x] = v;
            }
        };
        {
            const int n4 = td.lane1 ? td.n_need_heavy : td.n_need_list;
            for (int base = 0; base < n4; base += ng) {  // warp-uniform trip count
                const int k = base + slot4;
                const bool ok = k < n4;
                const int4 rec = ok ? __ldg(td.need_rec + k) : none;
                const double v = yfull_rec<4>(rec, q);
                if (ok && q == 0) finish(rec, v);
            }
            for (int k = n4 + slot1; k < td.n_need_list; k += gstride) {
                const int4 rec = __ldg(td.need_rec + k);
                finish(rec, yfull_rec<1>(rec, 0));
            }
            for (int k = td.n_need_list + gtid; k < td.n_need; k += gstride) {
                const int4 rec = __ldg(td.need_rec + k);
                finish(rec, yfull_rec<1>(rec, 0));
            }
        }
        if (!grid_sync(gs)) return 0.0;
        const int n4 = td.lane1 ? td.n_row_heavy : td.n_row_list;
        for (int base = 0; base < n4; base += ng) {
            const int k = base + slot4;
            const bool ok = k < n4;
            const int4 rec = ok ? __ldg(td.row_rec + k) : make_int4(0, 0, 0, 0);  // idle groups read DOF 0
            const double yj = scatter_rec<4>(rec, q);
            if (ok && q == 0) {
                y[rec.x] = yj;
                part += __ldcg(p + rec.x) * yj;
            }
        }
        for (int k = n4 + slot1; k < td.n_row_list; k += gstride) {
            const int4 rec = __ldg(td.row_rec + k);
            const double yj = scatter_rec<1>(rec, 0);
            y[rec.x] = yj;
            part += __ldcg(p + rec.x) * yj;
        }
        // rows [n_row_list, n_red) have no E^T entries and were completed above
        return part;
    }
};
