// Matrix-free Kronecker forms of a tensor-product cut box (the operators of
// assemble_cut_3d and solve_poisson_3d, code/cut_3d_sbp.py:89-146,386-503).
//
// With E = Ez (x) Ey (x) Ex every pulled-back form is a sum of Kronecker
// products of reduced 1D factors (n_a x n_a, E_a^T C_a E_a), applied here by
// three sum-factorised passes over the reduced vector (x fastest):
//
//   x pass:  U1 = (I (x) I (x) X0) p,   U2 = (I (x) I (x) X1) p
//   y pass:  V1 = (I (x) Y0 (x) I) U1,  V2 = (I (x) Y1 (x) I) U2 + (I (x) Y2 (x) I) U1
//   z pass:  y  = (Z0 (x) I (x) I) V2 + (Z1 (x) I (x) I) V1
//
// A single product Cz (x) Cy (x) Cx is X0 = Cx, Y0 = Cy, Z1 = Cz; a sum
// Hz (x) Hy (x) Cx + Hz (x) Cy (x) Hx + Cz (x) Hy (x) Hx (stiffness, the
// weak-penalty Poisson form) is X0 = Hx, X1 = Cx, Y0 = Y1 = Hy, Y2 = Cy,
// Z0 = Hz, Z1 = Cz.  Each factor is stored as a band: row i's nonzeros lie in
// columns [lo[i], lo[i] + W) (the reduced factors are banded apart from the
// few rows the extension couples, so W stays near 2p + 1 + the stencil of the
// small functions).  One thread per output entry: in the x pass consecutive
// threads read consecutive entries of one line, in the y and z passes they
// read the same band rows at consecutive x, so every pass coalesces.  Passes
// are separated by grid barriers; the z pass also returns the thread's share
// of p.y, so the operator plugs into the persistent PCG like CsrOp.
#pragma once

#include "common.cuh"

struct KronBand {
    int W;                     // band width (0: factor absent)
    const int* lo;             // [n] first column of each row's band
    const double* band;        // [n][W]
};

struct KronOp {
    static constexpr bool kFusedP = false;
    int nx, ny, nz;
    KronBand X0, X1, Y0, Y1, Y2, Z0, Z1;
    double* U1;
    double* U2;
    double* V1;
    double* V2;

    __device__ __forceinline__ static double row_dot(const KronBand& F, int i, const double* v, size_t stride) {
        const int lo = __ldg(F.lo + i);
        const double* b = F.band + (size_t)i * F.W;
        const double* vv = v + (size_t)lo * stride;
        // two accumulator chains, four band entries per step: more loads in flight
        double s0 = 0.0, s1 = 0.0;
        int w = 0;
        for (; w + 4 <= F.W; w += 4) {
            const double a0 = __ldg(b + w), a1 = __ldg(b + w + 1), a2 = __ldg(b + w + 2), a3 = __ldg(b + w + 3);
            const double v0 = __ldcg(vv + (size_t)w * stride), v1 = __ldcg(vv + (size_t)(w + 1) * stride);
            const double v2 = __ldcg(vv + (size_t)(w + 2) * stride), v3 = __ldcg(vv + (size_t)(w + 3) * stride);
            s0 += a0 * v0;
            s1 += a1 * v1;
            s0 += a2 * v2;
            s1 += a3 * v3;
        }
        for (; w < F.W; ++w) s0 += __ldg(b + w) * __ldcg(vv + (size_t)w * stride);
        return s0 + s1;
    }

    __device__ __forceinline__ double apply(const double* p, double* y, const GridSync& gs, double*) const {
        const size_t nxy = (size_t)nx * ny, N = nxy * nz;
        const size_t gtid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
        const size_t gstride = (size_t)gridDim.x * blockDim.x;
        for (size_t idx = gtid; idx < N; idx += gstride) {
            const size_t line = idx / nx;
            const int i = (int)(idx - line * nx);
            const double* row = p + line * nx;
            U1[idx] = row_dot(X0, i, row, 1);
            if (X1.W) U2[idx] = row_dot(X1, i, row, 1);
        }
        if (!grid_sync(gs)) return 0.0;
        for (size_t idx = gtid; idx < N; idx += gstride) {
            const size_t z = idx / nxy;
            const size_t rem = idx - z * nxy;
            const int i = (int)(rem / nx);
            const size_t x = rem - (size_t)i * nx;
            const size_t base = z * nxy + x;
            if (Y0.W) V1[idx] = row_dot(Y0, i, U1 + base, nx);
            if (Y1.W || Y2.W) {
                double s = 0.0;
                if (Y1.W) s += row_dot(Y1, i, U2 + base, nx);
                if (Y2.W) s += row_dot(Y2, i, U1 + base, nx);
                V2[idx] = s;
            }
        }
        if (!grid_sync(gs)) return 0.0;
        double part = 0.0;
        for (size_t idx = gtid; idx < N; idx += gstride) {
            const int i = (int)(idx / nxy);
            const size_t xy = idx - (size_t)i * nxy;
            double s = 0.0;
            if (Z0.W) s += row_dot(Z0, i, V2 + xy, nxy);
            if (Z1.W) s += row_dot(Z1, i, V1 + xy, nxy);
            y[idx] = s;
            part += __ldcg(p + idx) * s;
        }
        return part;
    }
};
