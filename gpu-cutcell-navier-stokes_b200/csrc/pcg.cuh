// Persistent Jacobi-PCG and its reduced-precision form with FP64 residual
// replacement, one cooperative launch per solve.  The iteration is the one of solve_gpu_cg
// (code/fast_solver_backends.py:236-274):
//
//   x = 0, r = b, z = D^{-1} r (z = r where the diagonal is zero), p = z
//   loop k = 1..maxiter:
//     Ap = A p; pAp = p.Ap; stop "breakdown" if pAp <= 0 or non-finite
//     alpha = rz/pAp; x += alpha p; r -= alpha Ap
//     stop "converged" if ||r||/||b|| <= tol (iterations = k)
//     z = D^{-1} r; beta = rz_new/rz; p = z + beta p
//
// Every dot product is a deterministic two-level reduction (block tree, then
// a fixed-order sum of the per-block partials that every block repeats), so
// all blocks take identical branch decisions and reruns are bit-identical.
#pragma once

#include "ops.cuh"

struct DevResult {
    int status;
    int iterations;
    int outer;
    int pad;
    double rel;
    double true_rel;
};

struct PcgBufs {
    int n;
    const double* dinv;  // Jacobi inverse (1 where the diagonal is zero)
    double* r;
    double* p;
    double* Ap;
    double* part;        // [8][nblocks]
    double* p2;          // second search-direction buffer (operators that fuse the p update)
};

// Inner PCG on A d = rhs from d = 0.  Returns the status; *iters receives the
// iteration count and *rel the final recursive relative residual.
template <class Op>
__device__ int pcg_core(const Op& op, const PcgBufs& B, const double* rhs, double* d, double tol, int maxiter,
                        const GridSync& gs, double* sm, double* sh, double diverge, int* iters,
                        double* rel_out) {
    const int n = B.n;
    const int nb = gridDim.x;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gstride = gridDim.x * blockDim.x;
    double* part = B.part;
    double rz_p = 0.0, bb_p = 0.0;
    for (int i = gtid; i < n; i += gstride) {
        const double bi = rhs[i];
        d[i] = 0.0;
        B.r[i] = bi;
        const double zi = B.dinv[i] * bi;
        B.p[i] = zi;
        rz_p += bi * zi;
        bb_p += bi * bi;
    }
    rz_p = block_sum(rz_p, sh);
    bb_p = block_sum(bb_p, sh);
    if (threadIdx.x == 0) {
        part[0 * nb + blockIdx.x] = rz_p;
        part[1 * nb + blockIdx.x] = bb_p;
    }
    if (!grid_sync(gs)) return CUTCELL_E_BARRIER;
    double rz = grid_reduce(part + 0 * nb, nb, sh);
    double bnorm = sqrt(grid_reduce(part + 1 * nb, nb, sh));
    if (bnorm == 0.0) bnorm = 1.0;
    int status = CUTCELL_E_NOCONV;
    int k = 0;
    double rel = 1.0;
    // Operators with kFusedP form p_k = D^-1 r + beta p_{k-1} inside the first
    // phase of their apply (double-buffered p), which saves the grid barrier
    // that a separate p update needs; the others update p here.
    double* P[2] = {B.p, Op::kFusedP ? B.p2 : B.p};
    double beta = 0.0;
    for (k = 1; k <= maxiter; ++k) {
        double* pk = P[(k - 1) & 1];
        double pap;
        if constexpr (Op::kFusedP) {
            pap = (k > 1) ? op.apply_next(P[k & 1], pk, B.r, B.dinv, beta, B.Ap, gs, sm) : op.apply(pk, B.Ap, gs, sm);
        } else {
            pap = op.apply(pk, B.Ap, gs, sm);
        }
        if (grid_error(gs)) return CUTCELL_E_BARRIER;
        pap = block_sum(pap, sh);
        if (threadIdx.x == 0) part[2 * nb + blockIdx.x] = pap;
        if (!grid_sync(gs)) return CUTCELL_E_BARRIER;
        pap = grid_reduce(part + 2 * nb, nb, sh);
        if (!(pap > 0.0) || !isfinite(pap)) {
            status = CUTCELL_E_BREAKDOWN;
            break;
        }
        const double alpha = rz / pap;
        double rr_p = 0.0, rzn_p = 0.0;
        for (int i = gtid; i < n; i += gstride) {
            const double pi = __ldcg(pk + i);
            d[i] += alpha * pi;
            const double ri = B.r[i] - alpha * __ldcg(B.Ap + i);
            B.r[i] = ri;
            rr_p += ri * ri;
            rzn_p += ri * (B.dinv[i] * ri);
        }
        rr_p = block_sum(rr_p, sh);
        rzn_p = block_sum(rzn_p, sh);
        if (threadIdx.x == 0) {
            part[3 * nb + blockIdx.x] = rr_p;
            part[4 * nb + blockIdx.x] = rzn_p;
        }
        if (!grid_sync(gs)) return CUTCELL_E_BARRIER;
        const double rr = grid_reduce(part + 3 * nb, nb, sh);
        const double rzn = grid_reduce(part + 4 * nb, nb, sh);
        rel = sqrt(rr) / bnorm;
        if (!isfinite(rel)) {
            status = CUTCELL_E_NAN;
            break;
        }
        if (rel <= tol) {
            status = CUTCELL_OK;
            break;
        }
        if (diverge > 0.0 && rel > diverge) {  // inner solve of a refinement sweep ran away
            status = CUTCELL_E_NAN;
            break;
        }
        beta = rzn / rz;
        rz = rzn;
        if constexpr (!Op::kFusedP) {
            for (int i = gtid; i < n; i += gstride) B.p[i] = p_next(B.dinv[i], B.r[i], beta, B.p[i]);
            if (!grid_sync(gs)) return CUTCELL_E_BARRIER;
        }
    }
    *iters = (k > maxiter) ? maxiter : k;
    *rel_out = rel;
    return status;
}

// ||b - A x|| / ||b|| with the FP64 operator (overwrites Ap).
template <class Op>
__device__ double true_residual(const Op& op, const PcgBufs& B, const double* b, const double* x, double bnorm,
                                const GridSync& gs, double* sm, double* sh, double* resid_out) {
    const int nb = gridDim.x;
    op.apply(x, B.Ap, gs, sm);
    if (!grid_sync(gs)) return -1.0;
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < B.n; i += gridDim.x * blockDim.x) {
        const double ri = b[i] - __ldcg(B.Ap + i);
        if (resid_out) resid_out[i] = ri;
        s += ri * ri;
    }
    s = block_sum(s, sh);
    if (threadIdx.x == 0) B.part[5 * nb + blockIdx.x] = s;
    if (!grid_sync(gs)) return -1.0;
    return sqrt(grid_reduce(B.part + 5 * nb, nb, sh)) / bnorm;
}

__device__ __forceinline__ double norm_of(const double* v, int n, double* part, const GridSync& gs, double* sh,
                                          int slot) {
    const int nb = gridDim.x;
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += v[i] * v[i];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) part[slot * nb + blockIdx.x] = s;
    if (!grid_sync(gs)) return -1.0;
    return sqrt(grid_reduce(part + slot * nb, nb, sh));
}

struct SolveArgs {
    const double* b;
    double* x;
    double tol;
    int maxiter;
    // reduced-precision forms
    double inner_tol;   // residual-replacement factor (ru_kernel)
    int inner_maxiter;  // unused
    int max_outer;      // replacement cap (ru_kernel)
    double* d;          // scratch vector
    double* rhat;       // scratch vector
    GridSync gs;
    PcgBufs B;
    DevResult* res;
};

// Plain FP64 PCG (the default form).
template <class Op>
__global__ void __launch_bounds__(CUTCELL_BLOCK, 2) pcg_kernel(Op op, SolveArgs a) {
    extern __shared__ double sm[];
    __shared__ double sh[CUTCELL_WARPS + 1];
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

// Reduced-precision PCG with FP64 residual replacement ("reliable updates",
// the refinement form of the FP32 / BF16 operators).  It is the Jacobi-PCG of
// pcg_core with A p evaluated by the reduced-precision operator `lo`; the
// iterate, the residual, the search direction and every dot product stay in
// FP64.  The recursive residual drifts from the true one by the operator's
// rounding, so it is replaced by the FP64 true residual b - A x (operator `hi`)
// whenever its norm has fallen by `replace` below the largest norm since the
// last replacement, and whenever the recursive test says converged.  The
// search direction is kept across a replacement, so the Krylov space is not
// restarted (a restarted refinement re-grows it every sweep).  Success needs
// the TRUE residual <= tol, or, once the recursive test has passed and the
// true residual has stopped halving (the FP64 attainable-accuracy floor), the
// reference's success bound true <= max(10 tol, 1e-14).  A run of
// replacements whose true residuals do not halve otherwise means the reduced
// operator cannot resolve the remaining error: the solve stops with
// CUTCELL_E_NOCONV instead of spinning to maxiter.
//   iterations: total PCG iterations (each one reduced-precision apply);
//   outer: replacements made + 1.
template <class OpHi, class OpLo>
__global__ void __launch_bounds__(CUTCELL_BLOCK, 2) ru_kernel(OpHi hi, OpLo lo, SolveArgs a) {
    extern __shared__ double sm[];
    __shared__ double sh[CUTCELL_WARPS + 1];
    const PcgBufs& B = a.B;
    const int n = B.n;
    const int nb = gridDim.x;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gstride = gridDim.x * blockDim.x;
    double* part = B.part;
    double* x = a.x;
    double rz_p = 0.0, bb_p = 0.0;
    for (int i = gtid; i < n; i += gstride) {
        const double bi = a.b[i];
        x[i] = 0.0;
        B.r[i] = bi;
        const double zi = B.dinv[i] * bi;
        B.p[i] = zi;
        rz_p += bi * zi;
        bb_p += bi * bi;
    }
    rz_p = block_sum(rz_p, sh);
    bb_p = block_sum(bb_p, sh);
    if (threadIdx.x == 0) {
        part[0 * nb + blockIdx.x] = rz_p;
        part[1 * nb + blockIdx.x] = bb_p;
    }
    int status = CUTCELL_E_NOCONV;
    int k = 0, nrep = 0, stall = 0;
    double rel = 1.0, true_rel = 1.0, last_true = 1.0;
    if (grid_sync(a.gs)) {
        double rz = grid_reduce(part + 0 * nb, nb, sh);
        double bnorm = sqrt(grid_reduce(part + 1 * nb, nb, sh));
        if (bnorm == 0.0) bnorm = 1.0;
        double rmax = bnorm * rel;
        double* P[2] = {B.p, OpLo::kFusedP ? B.p2 : B.p};
        double beta = 0.0;
        for (k = 1; k <= a.maxiter; ++k) {
            double* pk = P[(k - 1) & 1];
            double pap;
            if constexpr (OpLo::kFusedP) {
                pap = (k > 1) ? lo.apply_next(P[k & 1], pk, B.r, B.dinv, beta, B.Ap, a.gs, sm) : lo.apply(pk, B.Ap, a.gs, sm);
            } else {
                pap = lo.apply(pk, B.Ap, a.gs, sm);
            }
            if (grid_error(a.gs)) break;
            pap = block_sum(pap, sh);
            if (threadIdx.x == 0) part[2 * nb + blockIdx.x] = pap;
            if (!grid_sync(a.gs)) break;
            pap = grid_reduce(part + 2 * nb, nb, sh);
            if (!(pap > 0.0) || !isfinite(pap)) {
                status = CUTCELL_E_BREAKDOWN;
                break;
            }
            const double alpha = rz / pap;
            double rr_p = 0.0, rzn_p = 0.0;
            for (int i = gtid; i < n; i += gstride) {
                const double pi = __ldcg(pk + i);
                x[i] += alpha * pi;
                const double ri = B.r[i] - alpha * __ldcg(B.Ap + i);
                B.r[i] = ri;
                rr_p += ri * ri;
                rzn_p += ri * (B.dinv[i] * ri);
            }
            rr_p = block_sum(rr_p, sh);
            rzn_p = block_sum(rzn_p, sh);
            if (threadIdx.x == 0) {
                part[3 * nb + blockIdx.x] = rr_p;
                part[4 * nb + blockIdx.x] = rzn_p;
            }
            if (!grid_sync(a.gs)) break;
            double rn = sqrt(grid_reduce(part + 3 * nb, nb, sh));
            double rzn = grid_reduce(part + 4 * nb, nb, sh);
            rel = rn / bnorm;
            if (!isfinite(rel)) {
                status = CUTCELL_E_NAN;
                break;
            }
            rmax = rn > rmax ? rn : rmax;
            const bool by_test = rel <= a.tol;
            if (by_test || rn < a.inner_tol * rmax) {
                // replacement: r = b - A_64 x in FP64, and its dots
                hi.apply(x, B.Ap, a.gs, sm);
                if (!grid_sync(a.gs)) break;
                double t_p = 0.0, tz_p = 0.0;
                for (int i = gtid; i < n; i += gstride) {
                    const double ri = a.b[i] - __ldcg(B.Ap + i);
                    B.r[i] = ri;
                    t_p += ri * ri;
                    tz_p += ri * (B.dinv[i] * ri);
                }
                t_p = block_sum(t_p, sh);
                tz_p = block_sum(tz_p, sh);
                if (threadIdx.x == 0) {
                    part[5 * nb + blockIdx.x] = t_p;
                    part[6 * nb + blockIdx.x] = tz_p;
                }
                if (!grid_sync(a.gs)) break;
                rn = sqrt(grid_reduce(part + 5 * nb, nb, sh));
                rzn = grid_reduce(part + 6 * nb, nb, sh);
                ++nrep;
                true_rel = rn / bnorm;
                rel = true_rel;
                rmax = rn;
                if (!isfinite(true_rel)) {
                    status = CUTCELL_E_NAN;
                    break;
                }
                if (true_rel <= a.tol) {
                    status = CUTCELL_OK;
                    break;
                }
                // at the FP64 attainable-accuracy floor: the recursive test
                // passed, the true residual meets the reference's success
                // bound max(10 tol, 1e-14) (code/fast_solver_backends.py:283)
                // and no longer halves between replacements
                const double floor_ok = fmax(10.0 * a.tol, 1e-14);
                if (by_test && true_rel <= floor_ok && true_rel > 0.5 * last_true) {
                    status = CUTCELL_OK;
                    break;
                }
                // the reduced operator no longer resolves the error
                stall = (true_rel > 0.5 * last_true) ? stall + 1 : 0;
                last_true = true_rel;
                if (stall >= 3 || nrep >= a.max_outer) {
                    status = CUTCELL_E_NOCONV;
                    break;
                }
            }
            beta = rzn / rz;
            rz = rzn;
            if constexpr (!OpLo::kFusedP) {
                for (int i = gtid; i < n; i += gstride) B.p[i] = p_next(B.dinv[i], B.r[i], beta, B.p[i]);
                if (!grid_sync(a.gs)) break;
            }
        }
    }
    if (grid_error(a.gs)) status = CUTCELL_E_BARRIER;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.res->status = status;
        a.res->iterations = k > a.maxiter ? a.maxiter : k;
        a.res->outer = nrep + 1;
        a.res->rel = rel;
        a.res->true_rel = nrep > 0 ? true_rel : -1.0;
    }
}

// Single apply (operator benchmarks and tests): y = A x.
template <class Op>
__global__ void __launch_bounds__(CUTCELL_BLOCK, 2) apply_kernel(Op op, const double* x, double* y, GridSync gs) {
    extern __shared__ double sm[];
    op.apply(x, y, gs, sm);
}
