// Two-level patch preconditioner inside the persistent flexible PCG:
//
//   z = zc + B (r - A zc),   zc = P Ac^-1 P^T r,   Ac = P^T A P,
//
// B the exact 4x4x4 patch solves (Jacobi on patches without a stored block),
// P the uniform B-spline refinement (knot insertion) from n / c to n elements
// per axis, restricted to the rows of the reduced (kept) DOFs, and Ac its
// Galerkin coarse operator, inverted densely on the host (a few thousand
// coarse DOFs, read from L2 every iteration).  Coarse correction first, patch
// solves on the corrected residual: the two-grid cycle without pre-smoothing.
// Optionally B = omega (B_0 + B_1 + ...) with up to three more patch tilings,
// offset from the first by whole DOFs per axis; all tilings run in the same
// phase and keep their shares in separate vectors, summed by the next
// iteration's p update.
//
// The tensor structure of P is used in both directions:
//   restriction  P^T r : the x-contraction is fused into the x / r update
//                        (one warp per x-line of the background grid), the
//                        y-z contraction is one warp per coarse DOF;
//   prolongation P y   : each reduced DOF sums its (p + 1)^3 coarse terms
//                        from the coarse vector staged in shared memory, in
//                        its own phase before the apply A zc.  (Fusing it into
//                        the apply's phase 0 saves a grid barrier but makes the
//                        small rows of E zc re-evaluate the prolongation per
//                        entry; measured 1.5 us per iteration slower at n = 32.)
// Every sum has a fixed order; results are bit-reproducible.
#pragma once

#include "learned.cuh"

struct CoarseDev {
    int nb, nbc, ncg;           // fine / coarse DOFs per axis, nbc^3
    int pw, rw;                 // band widths of the prolongation rows / restriction rows
    const int* plo;             // [nb] first coarse index of fine row x (plo + pw <= nbc)
    const double* pval;         // [nb][pw], pw = p + 1
    const int* rlo;             // [nbc] first fine index of coarse column a (rlo + rw <= nb)
    const double* rval;         // [nbc][rw]
    const double* minv;         // [ncg][ncg] Ac^-1, zero rows / columns for coarse DOFs without fluid
    double* t1;                 // [nb * nb][nbc] x-contracted residual, line (z, y) major
    double* rc;                 // [ncg] P^T r
    double* yc;                 // [ncg] Ac^-1 P^T r
    double* zc;                 // [n] P yc
    double* azc;                // [n] A zc
    // optional extra patch tilings (offset from the first):
    //   z = zc + omega (B_0 + B_1 + ...) (r - A zc),
    // tiling i's share kept in zx[i] (n_extra = 0: z = zc + B_0 (r - A zc))
    int n_extra;
    int n_patch_x[ZSUM_MAX];
    const int* red_x[ZSUM_MAX];     // [n_patch_x][64] reduced index or -1
    const __nv_bfloat16* binv_x[ZSUM_MAX];  // [n_patch_x][64][64] symmetric patch inverses (BF16 storage)
    double* zx[ZSUM_MAX];           // [n] each
    double omega;
    // BF16 copy of the first tiling's inverses (by block slot); null: its FP64 blocks
    const __nv_bfloat16* binv0h;
};

// zc_j = (P yc)_j from the coarse vector in shared memory.  PW = p + 1 is the
// width of every prolongation row band (a fine B-spline lies in the support
// of at most p + 1 coarse ones per axis); the host pads the bands to exactly
// PW, so the loops unroll with the weights in registers.  Indices are clamped
// into the coarse grid, so a corrupt table cannot read outside ys.
template <int PW>
struct ProlongFn {
    CoarseDev cd;
    const int* full_of_red;
    const double* ys;
    __device__ __forceinline__ double operator()(int j) const {
        const int f = __ldg(full_of_red + j), nb = cd.nb, nbc = cd.nbc;
        const int z = f / (nb * nb), rem = f - z * nb * nb;
        const int y = rem / nb, x = rem - y * nb;
        const int xl = min(max(__ldg(cd.plo + x), 0), nbc - PW);
        const int yl = min(max(__ldg(cd.plo + y), 0), nbc - PW);
        const int zl = min(max(__ldg(cd.plo + z), 0), nbc - PW);
        double wx[PW], wy[PW], wz[PW];
#pragma unroll
        for (int t = 0; t < PW; ++t) {
            wx[t] = __ldg(cd.pval + x * PW + t);
            wy[t] = __ldg(cd.pval + y * PW + t);
            wz[t] = __ldg(cd.pval + z * PW + t);
        }
        double s = 0.0;
#pragma unroll
        for (int tz = 0; tz < PW; ++tz) {
            double sy = 0.0;
#pragma unroll
            for (int ty = 0; ty < PW; ++ty) {
                const double* row = ys + ((size_t)(zl + tz) * nbc + (yl + ty)) * nbc + xl;
                double sx = 0.0;
#pragma unroll
                for (int tx = 0; tx < PW; ++tx) sx += wx[tx] * row[tx];
                sy += wy[ty] * sx;
            }
            s += wz[tz] * sy;
        }
        return s;
    }
};

// x-lines of the background grid, one warp each: x += alpha p, r_old = r,
// r -= alpha A p on the line's reduced DOFs (alpha = 0: r_old = r only), this
// lane's share of r.r, and t1[line][a] = sum_x R[a][x] r(x) (zero off the
// reduced DOFs).  lbuf: nb doubles of this warp's shared memory.
__device__ __forceinline__ void tl_update_lines(const CoarseDev& cd, const ExtDev& ext, const PcgBufs& B, double* rold,
                                                double alpha, const double* pk, double* x, double* lbuf, double& rr) {
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    const int nb = cd.nb, nbc = cd.nbc, rw = cd.rw;
    for (int line = gw; line < nb * nb; line += nw) {
        const size_t base = (size_t)line * nb;
        for (int xi = lane; xi < nb; xi += 32) {
            const int j = __ldg(ext.red_of_full + base + xi);
            double rv = 0.0;
            if (j >= 0) {
                const double ro = __ldcg(B.r + j);
                rv = ro;
                if (alpha != 0.0) {
                    x[j] += alpha * __ldcg(pk + j);
                    rv = ro - alpha * __ldcg(B.Ap + j);
                    B.r[j] = rv;
                }
                rold[j] = ro;
                rr += rv * rv;
            }
            lbuf[xi] = rv;
        }
        __syncwarp();
        for (int a = lane; a < nbc; a += 32) {
            const int lo = __ldg(cd.rlo + a);
            double s = 0.0;
            for (int t = 0; t < rw; ++t) {
                const int xi = lo + t;
                if (xi >= 0 && xi < nb) s += __ldg(cd.rval + a * rw + t) * lbuf[xi];
            }
            cd.t1[(size_t)line * nbc + a] = s;
        }
        __syncwarp();
    }
}

// rc[(c nbc + b) nbc + a] = sum_{z, y} R[c][z] R[b][y] t1[z nb + y][a], one warp per coarse DOF
__device__ __forceinline__ void tl_restrict(const CoarseDev& cd) {
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    const int nb = cd.nb, nbc = cd.nbc, rw = cd.rw;
    for (int q = gw; q < cd.ncg; q += nw) {
        const int a = q % nbc, b = (q / nbc) % nbc, c = q / (nbc * nbc);
        const int ylo = __ldg(cd.rlo + b), zlo = __ldg(cd.rlo + c);
        double s = 0.0;
        for (int t = lane; t < rw * rw; t += 32) {
            const int tz = t / rw, ty = t - tz * rw;
            const int z = zlo + tz, y = ylo + ty;
            if (z >= 0 && z < nb && y >= 0 && y < nb)
                s += __ldg(cd.rval + c * rw + tz) * __ldg(cd.rval + b * rw + ty) *
                     __ldcg(cd.t1 + ((size_t)z * nb + y) * nbc + a);
        }
        s = warp_sum(s);
        if (lane == 0) cd.rc[q] = s;
    }
}

// yc = Ac^-1 rc: rc staged in shared memory, one warp per row
__device__ __forceinline__ void tl_coarse_solve(const CoarseDev& cd, double* srb) {
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    const int ncg = cd.ncg;
    for (int i = threadIdx.x; i < ncg; i += blockDim.x) srb[i] = __ldcg(cd.rc + i);
    __syncthreads();
    for (int row = gw; row < ncg; row += nw) {
        const double* m = cd.minv + (size_t)row * ncg;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;  // four chains: more row loads in flight
        int col = lane;
        for (; col + 96 < ncg; col += 128) {
            s0 += __ldg(m + col) * srb[col];
            s1 += __ldg(m + col + 32) * srb[col + 32];
            s2 += __ldg(m + col + 64) * srb[col + 64];
            s3 += __ldg(m + col + 96) * srb[col + 96];
        }
        for (; col < ncg; col += 32) s0 += __ldg(m + col) * srb[col];
        double s = warp_sum((s0 + s1) + (s2 + s3));
        if (lane == 0) cd.yc[row] = s;
    }
    __syncthreads();
}

// Half h of patch k of one tiling, by one warp (two warps per patch, lane l
// owns patch row 32 h + l): r' = r - A zc on the patch (both halves, for the
// block product), zout = zbase + wgt B_P r' on this half (exact block, or
// Jacobi where the tiling has no block for the patch; zbase may be null), and
// this lane's shares of r.zout and r_old.zout.  slot null with binv set means
// block k for patch k.  (Four warps per patch, 16 rows each with the columns
// split over two lanes, measured slower: each item repeats the patch's r and
// A zc loads.)
// one stored patch-inverse entry, widened to FP64
__device__ __forceinline__ double inv_entry(const double* p) { return __ldg(p); }
__device__ __forceinline__ double inv_entry(const __nv_bfloat16* p) { return (double)__bfloat162float(__ldg(p)); }

template <typename BT>
__device__ __forceinline__ void tl_patch_half(const int* red, const int* slot_map, const BT* binv,
                                              const double* zbase, double* zout, double wgt, const CoarseDev& cd,
                                              const PcgBufs& B, const double* rold, int k, int h, double& rz,
                                              double& roz) {
    const int l = threadIdx.x & 31;
    const int j0 = __ldg(red + (size_t)k * 64 + l), j1 = __ldg(red + (size_t)k * 64 + l + 32);
    const double q0 = j0 >= 0 ? __ldcg(B.r + j0) - __ldcg(cd.azc + j0) : 0.0;
    const double q1 = j1 >= 0 ? __ldcg(B.r + j1) - __ldcg(cd.azc + j1) : 0.0;
    const int j = h ? j1 : j0;
    const int row = 32 * h + l;
    const int slot = binv ? (slot_map ? __ldg(slot_map + k) : k) : -1;
    double w;
    if (slot >= 0) {  // exact block solve: column q of the symmetric inverse is row q
        const BT* Bk = binv + (size_t)slot * 4096 + row;
        double w0 = 0.0, w1 = 0.0;  // FP64 accumulation whatever the storage
#pragma unroll 16
        for (int q = 0; q < 32; ++q) {
            w0 += inv_entry(Bk + q * 64) * __shfl_sync(0xffffffffu, q0, q);
            w1 += inv_entry(Bk + (q + 32) * 64) * __shfl_sync(0xffffffffu, q1, q);
        }
        w = w0 + w1;
    } else {
        w = j >= 0 ? __ldg(B.dinv + j) * (h ? q1 : q0) : 0.0;
    }
    if (j >= 0) {
        const double zj = (zbase ? __ldcg(zbase + j) : 0.0) + wgt * w;
        zout[j] = zj;
        rz += __ldcg(B.r + j) * zj;
        roz += __ldcg(rold + j) * zj;
    }
}

// z = M(r) from t1 (already formed by tl_update_lines): restriction, coarse
// solve, prolongation + A zc, patch step; leaves this block's r.z and r_old.z
// partials in part slots 3 and 5 (the caller syncs the grid before reading
// them).  False if a grid barrier gave up.
template <class Op>
__device__ __forceinline__ bool tl_precond(const Op& op, const CoarseDev& cd, const LearnedArgs& L, const PcgBufs& B,
                                           const GridSync& gs, double* sm, double* sh) {
    const int nb = gridDim.x;
    const int warp = threadIdx.x >> 5;
    const int gw = blockIdx.x * (blockDim.x >> 5) + warp, nw = gridDim.x * (blockDim.x >> 5);
    tl_restrict(cd);
    if (!grid_sync(gs)) return false;
    tl_coarse_solve(cd, sm);
    if (!grid_sync(gs)) return false;
    for (int i = threadIdx.x; i < cd.ncg; i += blockDim.x) sm[i] = __ldcg(cd.yc + i);
    __syncthreads();
    {
        const ProlongFn<Op::kDegree1> f{cd, op.td.ext.full_of_red, sm};
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < op.td.ext.n_red; i += gridDim.x * blockDim.x)
            cd.zc[i] = f(i);
    }
    if (!grid_sync(gs)) return false;
    (void)op.apply(cd.zc, cd.azc, gs, sm);
    if (grid_error(gs) || !grid_sync(gs)) return false;
    // both tilings in one phase: each reduced DOF lies in one patch of each,
    // and r.z = r.z_0 + r.z_2 is summed from the two tilings' shares
    double rz = 0.0, roz = 0.0;
    const int n0 = 2 * L.pm.n_patch;
    int ntot = n0;
    for (int i = 0; i < cd.n_extra; ++i) ntot += 2 * cd.n_patch_x[i];
    const double w0 = cd.n_extra ? cd.omega : 1.0;
    for (int q = gw; q < ntot; q += nw) {
        if (q >= n0) {
            int t = q - n0, i = 0;
            while (i + 1 < cd.n_extra && t >= 2 * cd.n_patch_x[i]) t -= 2 * cd.n_patch_x[i++];
            tl_patch_half(cd.red_x[i], (const int*)nullptr, cd.binv_x[i], nullptr, cd.zx[i], cd.omega, cd, B, L.rold,
                          t >> 1, t & 1, rz, roz);
        } else if (cd.binv0h)
            tl_patch_half(L.pm.red, L.pm.slot, cd.binv0h, cd.zc, L.z, w0, cd, B, L.rold, q >> 1, q & 1, rz, roz);
        else
            tl_patch_half(L.pm.red, L.pm.slot, L.pm.binv, cd.zc, L.z, w0, cd, B, L.rold, q >> 1, q & 1, rz, roz);
    }
    rz = block_sum(rz, sh);
    roz = block_sum(roz, sh);
    if (threadIdx.x == 0) {
        B.part[3 * nb + blockIdx.x] = rz;
        B.part[5 * nb + blockIdx.x] = roz;
    }
    return true;
}

// Two-level flexible PCG (Polak-Ribiere beta).  Per iteration:
//   apply:  p = z + beta p_old fused into phase 0, A p, p.A p   (operator barriers)
//   barrier, alpha
//   lines:  x += alpha p, r -= alpha A p, r.r, x-contraction of r
//   barrier, convergence test on ||r|| / ||b||
//   z = M(r) (tl_precond), barrier, beta = (r.z - r_old.z) / r.z_old
template <class Op>
__global__ void __launch_bounds__(CUTCELL_BLOCK, 2) tlpcg_kernel(Op op, SolveArgs a, LearnedArgs L, CoarseDev cd) {
    static_assert(Op::kFusedP, "the two-level PCG forms p inside the operator's first phase");
    extern __shared__ __align__(16) double sm[];
    __shared__ double sh[CUTCELL_WARPS + 1];
    const PcgBufs& B = a.B;
    const int n = B.n, nb = gridDim.x;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gstride = gridDim.x * blockDim.x;
    double* lbuf = sm + (size_t)(threadIdx.x >> 5) * cd.nb;
    ZSum zs;  // z = z_0 + the extra tilings' shares
    zs.z0 = L.z;
    zs.nx = cd.n_extra;
    for (int i = 0; i < ZSUM_MAX; ++i) zs.zx[i] = cd.zx[i];
    double* part = B.part;
    const GridSync& gs = a.gs;
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
    double rr = 0.0;
    double rz = 0.0;
    if (status != CUTCELL_E_BARRIER) {
        tl_update_lines(cd, op.td.ext, B, L.rold, 0.0, B.p, a.x, lbuf, rr);
        if (!grid_sync(gs) || !tl_precond(op, cd, L, B, gs, sm, sh) || !grid_sync(gs)) status = CUTCELL_E_BARRIER;
    }
    if (status != CUTCELL_E_BARRIER) {
        rz = grid_reduce(part + 3 * nb, nb, sh);
        for (int i = gtid; i < n; i += gstride) B.p[i] = zs.at(i);
        if (!grid_sync(gs)) status = CUTCELL_E_BARRIER;
    }
    double* P[2] = {B.p, B.p2};
    double beta = 0.0;
    for (k = 1; k <= a.maxiter && status != CUTCELL_E_BARRIER; ++k) {
        double* pk = P[(k - 1) & 1];
        double pap = (k == 1)      ? op.apply(pk, B.Ap, gs, sm)
                     : cd.n_extra ? op.apply_next_sum(P[k & 1], pk, zs, beta, B.Ap, gs, sm)
                                  : op.apply_next(P[k & 1], pk, L.z, L.ones, beta, B.Ap, gs, sm);
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
        rr = 0.0;
        tl_update_lines(cd, op.td.ext, B, L.rold, alpha, pk, a.x, lbuf, rr);
        rr = block_sum(rr, sh);
        if (threadIdx.x == 0) part[4 * nb + blockIdx.x] = rr;
        if (!grid_sync(gs)) {
            status = CUTCELL_E_BARRIER;
            break;
        }
        rel = sqrt(grid_reduce(part + 4 * nb, nb, sh)) / bnorm;
        if (!isfinite(rel)) {
            status = CUTCELL_E_NAN;
            break;
        }
        if (rel <= a.tol) {
            status = CUTCELL_OK;
            break;
        }
        if (!tl_precond(op, cd, L, B, gs, sm, sh) || !grid_sync(gs)) {
            status = CUTCELL_E_BARRIER;
            break;
        }
        const double rzn = grid_reduce(part + 3 * nb, nb, sh);
        const double roz_n = grid_reduce(part + 5 * nb, nb, sh);
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
