/*
 * cutcell_b200.h -- C ABI of libcutcell_b200.so, the B200 (sm_100a) solve path
 * for aggregated cut-cell systems.
 *
 * Conventions for every entry point:
 *   - all array pointers are DEVICE pointers (e.g. torch.Tensor.data_ptr());
 *   - the caller keeps its arrays alive for the lifetime of a context that
 *     references them; contexts own only their device scratch and free it in
 *     cutcell_destroy;
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream);
 *   - every call returns a status code (CUTCELL_OK = 0); solver outcomes that
 *     the reference reports as success=False ("maximum iterations reached",
 *     "CG breakdown: non-positive curvature") come back as a status code and a
 *     filled report, never as a crash, and there is no CPU fallback.
 *
 * Index layout: DOFs are flattened x-fastest, (iz*ny + iy)*nx + ix
 * (code/cut_3d_sbp.py:20-22, code/bell_3d_core.py:313-317).
 */
#ifndef CUTCELL_B200_H
#define CUTCELL_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    CUTCELL_OK = 0,
    CUTCELL_E_NOCONV = 1,     /* maxiter reached: "maximum iterations reached" */
    CUTCELL_E_BREAKDOWN = 2,  /* p.Ap <= 0 or non-finite: "CG breakdown: non-positive curvature" */
    CUTCELL_E_NAN = 3,        /* non-finite residual */
    CUTCELL_E_SHAPE = 4,      /* inconsistent sizes / layout */
    CUTCELL_E_CUDA = 5,       /* a CUDA runtime call failed */
    CUTCELL_E_BARRIER = 6,    /* a bounded device-wide wait ran out */
    CUTCELL_E_ARG = 7         /* invalid argument */
};

enum { CUTCELL_FP64 = 0, CUTCELL_FP32_IR = 1, CUTCELL_BF16_IR = 2 };
enum {
    CUTCELL_PRECOND_NONE = 0,
    CUTCELL_PRECOND_JACOBI = 1,
    CUTCELL_PRECOND_JACOBI_LEARNED = 2, /* patch blocks where set, the network on the other patches */
    CUTCELL_PRECOND_BLOCK = 3,          /* patch blocks where set, Jacobi on the other patches */
    CUTCELL_PRECOND_TWOLEVEL = 4        /* Galerkin coarse-grid correction, then the patch solves */
};

typedef struct cutcell_ctx cutcell_ctx;

/* Mirrors SolverReport (code/fast_solver_backends.py:30-45) for the device
 * part: iterations counts the iteration in which the stopping test passed
 * (code/fast_solver_backends.py:249-266); relative_residual is the recursive
 * ||r||/||b||; true_relative_residual is ||b - A x||/||b|| recomputed in FP64
 * on the device (b = 0 -> denominator 1, code/fast_solver_backends.py:63-71). */
typedef struct {
    int32_t status;
    int32_t iterations;        /* total inner PCG iterations */
    int32_t outer_iterations;  /* refinement sweeps (1 for plain FP64) */
    int32_t blocks;            /* persistent grid size used */
    double relative_residual;
    double true_relative_residual;
    double elapsed_ms;         /* device time of the solve (CUDA events) */
} CutcellReport;

/* Matrix-free operator description (host struct holding device pointers).
 * Element blocks: full elements use per-axis 1D factors
 *   Mz (x) My (x) (a_mass Mx + Kx) + Mz (x) Ky (x) Mx + Kz (x) My (x) Mx,
 * cut elements a dense (p+1)^3 x (p+1)^3 block.  Tiles group tile^3 elements. */
typedef struct {
    int32_t n_elements;    /* per axis */
    int32_t degree;
    int32_t tile;          /* elements per tile edge (4) */
    int32_t n_tiles_axis;
    int32_t n_items;       /* work items: nonempty tiles and cut-element chunks */
    int32_t cut_chunk;     /* cut elements per work item */
    int32_t n_cut;
    int32_t n_full;        /* (n_elements+degree)^3 */
    int32_t n_red;
    int32_t n_small;
    int32_t n_need;        /* full DOFs read by the E^T scatter (identity + small rows) */
    double a_mass;
    const int32_t* item_list;  /* [n_items] >= 0: tile id, < 0: cut chunk -(k+1); heaviest first */
    const int32_t* tile_kind;  /* [n_tiles_axis^3] 0 empty, 1 full, 2 mixed */
    const int32_t* tile_eptr;  /* [n_tiles_axis^3 + 1] uncut elements of mixed tiles */
    const int32_t* tile_elem;  /* local element id (ez*tile+ey)*tile+ex */
    const int32_t* tile_ecut;  /* reserved (cut elements are separate work items) */
    const double* M1;          /* [n][(p+1)^2] */
    const double* Kt1;         /* [3][n][(p+1)^2] */
    const double* TM;          /* [n_tiles_axis][D^2], D = tile+degree */
    const double* TA;          /* [n_tiles_axis][D^2] */
    const double* TK;          /* [3][n_tiles_axis][D^2] */
    const double* cut_mats;    /* [n_cut][(p+1)^6] symmetric, row-major; degree 3 copies the
                                  upper triangles (row <= column) into a half-size split
                                  storage at create and reads only that afterwards */
    const int32_t* cut_base;   /* [n_cut] full index of each cut element's first DOF */
    const int32_t* cut_dof_slot; /* [n_full] slot in the DOF -> cut-element list, -1 if none */
    const int32_t* cut_dof_ptr;  /* [n_slots + 1] */
    const int32_t* cut_dof_ent;  /* cut * (p+1)^3 + local row, ascending per slot; every
                                    (cut, local row) appears exactly once */
    const int32_t* need;         /* [n_need] full DOF indices */
    const int32_t* red_of_full;
    const int32_t* small_slot;
    const int32_t* small_ptr;
    const int32_t* small_idx;
    const double* small_val;
    const int32_t* full_of_red;
    const int32_t* smallT_ptr;
    const int32_t* smallT_row;
    const double* smallT_val;
    const double* diag;        /* [n_red] diagonal of E^T A E (Jacobi) */
    int32_t n_mixed;           /* leading mixed tiles in item_list (the rest are full tiles) */
} CutcellTileDesc;

/* Replaces the CuPy CSR upload + Jacobi-CG loop of solve_gpu_cg
 * (code/fast_solver_backends.py:194-289): CSR of the reduced SPD matrix
 * (int32 indptr/indices, fp64 data), already on the device.  The structure is
 * checked on the device at create (indptr[0] = 0, indptr[n] = nnz, indptr
 * non-decreasing, every column in [0, n)); a malformed matrix returns
 * CUTCELL_E_SHAPE and no context. */
int cutcell_pcg_create_csr(int32_t n, int32_t nnz, const int32_t* indptr, const int32_t* indices,
                           const double* data, cutcell_ctx** out);

/* Structured entry for the matrix-free E^T A E (the operator restrict_spd of
 * code/bell_3d_core.py:550-552 forms explicitly). */
int cutcell_pcg_create_tiles(const CutcellTileDesc* desc, cutcell_ctx** out);

/* Refinement controls for the FP32/BF16 forms: inner relative tolerance,
 * inner iteration cap per sweep, maximum sweeps. */
int cutcell_set_refinement(cutcell_ctx* ctx, double inner_tol, int32_t inner_maxiter, int32_t max_outer);

/* Jacobi-PCG from x = 0 to ||r||/||b|| <= tol; the same algorithm as
 * solve_gpu_cg (code/fast_solver_backends.py:236-274), run as one persistent
 * cooperative launch with no host round trip per iteration. precision is
 * CUTCELL_FP64 (plain) or an iterative-refinement form; precond is
 * CUTCELL_PRECOND_NONE, CUTCELL_PRECOND_JACOBI, or
 * CUTCELL_PRECOND_JACOBI_LEARNED (flexible PCG, FP64, needs
 * cutcell_pcg_set_learned).  Blocks until done. */
int cutcell_pcg_solve(cutcell_ctx* ctx, const double* b, double* x, double tol, int32_t maxiter,
                      int32_t precision, int32_t precond, CutcellReport* report, void* stream);

/* y = E^T A E x (reduced vectors), operator data in the given precision. */
int cutcell_apply(cutcell_ctx* ctx, const double* x, double* y, int32_t precision, void* stream);

/* ---- tensor-product cut boxes (assemble_cut_3d / solve_poisson_3d,
 * code/cut_3d_sbp.py:89-146,386-503) ----
 * All their forms are sums of Kronecker products of reduced 1D factors
 * E_a^T C_a E_a (E = Ez (x) Ey (x) Ex), applied matrix-free by three
 * sum-factorised passes; no N x N matrix is formed.  create: the reduced 1D
 * sizes n[a] (x, y, z) and per axis the dense row-major factors (device, n_a x
 * n_a, copied into a banded form at create) of the mass H, stiffness K,
 * advection Q (Q_ij = int phi_i phi_j'), boundary form S, and the weak-penalty
 * Poisson factor A = K + beta (tL tL^T + tR tR^T) - N - N^T
 * (N = tL (-dL)^T + tR dR^T); diag: the diagonal of the 3D Poisson form
 * (Jacobi).  The context solves (cutcell_pcg_solve, FP64, precond NONE or
 * JACOBI) the Poisson system
 *   A3 = Hz (x) Hy (x) Ax + Hz (x) Ay (x) Hx + Az (x) Hy (x) Hx,
 * and applies every form through cutcell_apply_form. */
enum {
    CUTCELL_FORM_A = 0,  /* the context's SPD system (all context kinds) */
    CUTCELL_FORM_H = 1,  /* Hz (x) Hy (x) Hx */
    CUTCELL_FORM_K = 2,  /* Hz Hy Kx + Hz Ky Hx + Kz Hy Hx */
    CUTCELL_FORM_QX = 3, /* Hz (x) Hy (x) Qx */
    CUTCELL_FORM_QY = 4,
    CUTCELL_FORM_QZ = 5,
    CUTCELL_FORM_SX = 6, /* Hz (x) Hy (x) Sx */
    CUTCELL_FORM_SY = 7,
    CUTCELL_FORM_SZ = 8
};
typedef struct {
    int32_t n[3];
    const double* factors[3][5]; /* [axis x, y, z][H, K, Q, S, A] */
    const double* diag;
} CutcellKronDesc;
int cutcell_kron_create(const CutcellKronDesc* desc, cutcell_ctx** out);
/* y = F x for a form F of the context (CUTCELL_FORM_*, FP64); CSR and tile
 * contexts hold only CUTCELL_FORM_A. */
int cutcell_apply_form(cutcell_ctx* ctx, const double* x, double* y, int32_t which, void* stream);

/* Extension gather x_full = E x_red and transpose scatter y_red = E^T y_full
 * (E as produced by polynomial_preserving_extension_3d,
 * code/bell_3d_core.py:471-542); uses the tile descriptor's E arrays. */
int cutcell_ext_gather(cutcell_ctx* ctx, const double* x_red, double* x_full, void* stream);
int cutcell_ext_scatter(cutcell_ctx* ctx, const double* y_full, double* y_red, void* stream);

/* ---- learned preconditioner (no counterpart in the reference: an addition
 * of this build; its solve is flexible PCG with z = D^{-1} r + s * mlp(x) on
 * 4x4x4 DOF patches, u = D^{-1} r, x = [u / s, gamma * u / s] (128 features),
 * s = patch norm, odd part (mlp(x) - mlp(-x)) / 2,
 * MLP 128 -> 64 -> 64 -> 64 (ReLU), BF16 weights, FP32 accumulation) ---- */
typedef struct cutcell_mlp cutcell_mlp;
#define CUTCELL_MLP_NPARAM 16576  /* FP32: W1[128][64] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] */
/* activation of the two hidden layers: 0 = ReLU, 1 = identity (linear network) */
int cutcell_mlp_create(const float* theta_init, int32_t activation, cutcell_mlp** out);
/* copies of the FP32 parameters and of the last gradient (either may be NULL) */
int cutcell_mlp_params(cutcell_mlp* mlp, float* theta_out, float* grad_out);
/* Y[batch][64] = mlp(X[batch][128]) */
int cutcell_mlp_forward(cutcell_mlp* mlp, const float* X, int32_t batch, float* Y, void* stream);
/* loss = mean((mlp(X) - T)^2); gradients of it; an Adam step when lr > 0;
 * loss_out (device float, may be NULL) */
int cutcell_mlp_train_step(cutcell_mlp* mlp, const float* X, const float* T, int32_t batch, float lr, float* loss_out,
                           void* stream);
int cutcell_mlp_destroy(cutcell_mlp* mlp);
/* features X[n_patch][128] and scales S[n_patch] of a reduced residual r
 * (patch_red[n_patch][64]: reduced index or -1; patch_gamma: fluid ratios) */
int cutcell_patch_features(cutcell_ctx* ctx, const int32_t* patch_red, const float* patch_gamma, int32_t n_patch,
                           const double* r, float* X, float* S, void* stream);
/* training targets T[n_patch][64] = (e - D^{-1} r) / S on the patch DOFs */
int cutcell_patch_targets(cutcell_ctx* ctx, const int32_t* patch_red, int32_t n_patch, const double* e,
                          const double* r, const float* S, float* T, void* stream);
/* attach (mlp != NULL) or detach the learned correction used by
 * CUTCELL_PRECOND_JACOBI_LEARNED (FP64, matrix-free contexts) */
int cutcell_pcg_set_learned(cutcell_ctx* ctx, cutcell_mlp* mlp, const int32_t* patch_red, const float* patch_gamma,
                            int32_t n_patch);

/* exact inverses binv[n_patch][64][64] (symmetric) on every patch of the
 * attached layout (block Jacobi on all patches, the ceiling of patch-local
 * corrections); NULL removes them */
int cutcell_pcg_set_block_inverses(cutcell_ctx* ctx, const double* binv);
/* Exact solves on chosen patches: slot[n_patch] is each patch's block in
 * binv[n_blocks][64][64] (symmetric inverses of the patch blocks of E^T A E),
 * or -1.  Used by CUTCELL_PRECOND_BLOCK (Jacobi on the patches without a
 * block) and CUTCELL_PRECOND_JACOBI_LEARNED (the network on them); both run
 * flexible PCG in FP64.  patch_red is the layout of cutcell_pcg_set_learned
 * (the same pointer when a network is attached).  binv NULL removes the
 * blocks.  All device pointers, kept by reference. */
int cutcell_pcg_set_patch_blocks(cutcell_ctx* ctx, const int32_t* patch_red, int32_t n_patch, const int32_t* slot,
                                 const double* binv);

/* Coarse level of CUTCELL_PRECOND_TWOLEVEL (no reference counterpart: a
 * preconditioner of solve_gpu_cg's systems, code/fast_solver_backends.py:194-289).
 * z = zc + B (r - A zc) with zc = P Ac^-1 P^T r: P the tensor product of the
 * 1D uniform B-spline refinement R1 (nbc coarse -> nb = n + p fine functions
 * per axis) restricted to the reduced DOFs, Ac = P^T A P, B the patch solves
 * of cutcell_pcg_set_patch_blocks (Jacobi on patches without a block).  The
 * 1D refinement is given twice, banded: by fine row x (coarse columns
 * plo[x] .. plo[x] + pw - 1, values pval[x][pw], pw = p + 1) and by coarse column a
 * (fine rows rlo[a] .. rlo[a] + rw - 1, values rval[a][rw]); zero entries pad
 * the bands.  minv is Ac^-1 (FP64: the coarse solve is sensitive to its rounding) on the full coarse grid (nbc^3 x nbc^3,
 * row-major, coarse index (c nbc + b) nbc + a for (x, y, z) = (a, b, c)), zero
 * rows and columns for coarse functions without fluid.  All device pointers,
 * kept by reference; NULL desc removes the level.  At most 16384 coarse
 * DOFs (CUTCELL_E_SHAPE). */
typedef struct {
    int32_t nb, nbc, pw, rw;
    const int32_t* plo;
    const double* pval;
    const int32_t* rlo;
    const double* rval;
    const double* minv;
} CutcellCoarseDesc;
int cutcell_pcg_set_coarse(cutcell_ctx* ctx, const CutcellCoarseDesc* desc);
/* Patch inverses of CUTCELL_PRECOND_TWOLEVEL in BF16 storage (uint16_t bit
 * patterns of bfloat16; FP64 accumulation).  binv0: the first tiling's inverses, indexed like the binv of
 * cutcell_pcg_set_patch_blocks (NULL: use those FP64 blocks).  n_extra (0..3)
 * more tilings, 4x4x4 patches offset from the first by whole DOFs per axis:
 * host arrays of device pointers patch_red[i] ([n_patch[i]][64] reduced index
 * or -1) and binv[i] ([n_patch[i]][64][64] symmetric inverses).  With them the
 * step is z = zc + omega (B_0 + B_1 + ...) (r - A zc), 0 < omega <= 1, and
 * every reduced DOF must lie in exactly one patch of each tiling.  The device
 * pointers are kept by reference. */
int cutcell_pcg_set_twolevel_blocks(cutcell_ctx* ctx, const uint16_t* binv0, int32_t n_extra,
                                    const int32_t* const* patch_red, const int32_t* n_patch,
                                    const uint16_t* const* binv, double omega);

/* ---- periodic-hill fast diagonalisation (FastDiagHill, cpp/include/cut/hill_fastdiag.h:20-80) ----
 * create: the reduced 2D forms M2, Qx2, Qy2 (nr x nr, row-major), the z
 * symbols mu, kap (nz), and the per-mode inverses Ainv[nz][nr][nr],
 * Sinv[nz][nr][nr] that FastDiagHill::build (:26-43) forms; all device
 * pointers, kept by reference.  solve: FastDiagHill::solve (:47-79) on FieldH
 * arrays (v[m*nz + iz]); asynchronous on `stream`. */
typedef struct cutcell_fastdiag cutcell_fastdiag;
int cutcell_fastdiag_create(int32_t nr, int32_t nz, const double* M2, const double* Qx2, const double* Qy2,
                            const double* mu, const double* kap, const double* Ainv, const double* Sinv,
                            cutcell_fastdiag** out);
int cutcell_fastdiag_solve(cutcell_fastdiag* fd, const double* ux, const double* uy, const double* uz, double* ox,
                           double* oy, double* oz, void* stream);
int cutcell_fastdiag_destroy(cutcell_fastdiag* fd);
/* Batched FP64 GEMM on the FP64 tensor cores, the dense work of the
 * fast-diagonalisation build through a shared generalised eigenbasis
 * (the per-mode operators of FastDiagHill::build, hill_fastdiag.h:26-43, as
 * A_k^-1 = Phi diag(d_k) Phi^T and S_k = G diag(w_k) G^T, the
 * Lynch-Rice-Thomas form of cpp/include/solvers/fastdiag3.h:29-92):
 *   C_b = A_b diag(s_b) B_b^T (+ beta C_b),  b = 0 .. batch-1,
 * A_b (M x K) and B_b (N x K) row-major with leading dimensions lda, ldb; s
 * (optional, NULL = ones) a K-vector per batch; strides in elements, 0 shares
 * an operand; asynchronous on `stream`. */
int cutcell_dgemm_nt(int32_t M, int32_t N, int32_t K, const double* A, int64_t lda, int64_t strideA, const double* B,
                     int64_t ldb, int64_t strideB, const double* s, int64_t strideS, double beta, double* C, int64_t ldc,
                     int64_t strideC, int32_t batch, void* stream);

/* ---- periodic-hill advection and fast step ----
 * hill_skew_conv (cpp/include/cut/hill3d.h:519-538) for all three velocity
 * components, and hill_fastdiag_step (cpp/include/cut/hill_fastdiag.h:83-95).
 * The descriptor holds device pointers to the Galerkin sample machinery of
 * Hill3D (hill3d.h:86-93: sparse reduced 2D sample rows sp_idx / sp_phi /
 * sp_dpx / sp_dpy, weights w2; z basis Vz, dVz, weights wz) in the blocked
 * form the host prepares (cutcell_b200/hill.py, HillAdvection): segments of
 * consecutive 2D points sharing one row pattern, per-z-element band tables,
 * and the per-mode gather of segment partials; plus the mass inverses M2inv
 * (nr x nr) and Mzinv (nz x nz).  Supported: nz <= 32, z degree 3 (band 4),
 * <= 16 z points per element, <= 32 modes per 2D row pattern. */
typedef struct {
    int32_t nr, nz;        /* reduced 2D modes, z modes */
    int32_t qpe, nzb;      /* z quadrature points per z element, z band width */
    int32_t n_seg, lmax;   /* segments, longest row pattern */
    int32_t n_part, n2q;   /* sum of pattern lengths, 2D quadrature points */
    const int32_t* seg_q0;   /* [n_seg] */
    const int32_t* seg_q1;   /* [n_seg] */
    const int32_t* seg_pat;  /* [n_seg] offset of the pattern in pat_idx */
    const int32_t* seg_len;  /* [n_seg] */
    const int32_t* pat_idx;  /* [n_part] reduced modes */
    const int32_t* sp_ptr;   /* [n2q + 1] */
    const double* phi;       /* sample row values, aligned with the patterns */
    const double* dpx;
    const double* dpy;
    const double* w2;        /* [n2q] */
    const int32_t* zb;       /* [nz][nzb] modes of each z element in periodic order */
    const double* Vl;        /* [nz][qpe][nzb] */
    const double* dVl;       /* [nz][qpe][nzb] */
    const double* wzl;       /* [nz][qpe] */
    const int32_t* g_ptr;    /* [nr + 1] */
    const int32_t* g_ent;    /* [n_part] partial rows of each mode, segment order */
    const double* Mzinv;
    const double* M2inv;
} CutcellHillDesc;
typedef struct cutcell_hill cutcell_hill;
int cutcell_hill_create(const CutcellHillDesc* desc, cutcell_hill** out);
/* (cx, cy, cz) = hill_skew_conv(w = u, u_c) for c = x, y, z; FieldH arrays. */
int cutcell_hill_skew_conv(cutcell_hill* hill, const double* ux, const double* uy, const double* uz, double* cx,
                           double* cy, double* cz, void* stream);
/* One hill_fastdiag_step in place on (ux, uy, uz): SSP-RK3 of -skew_conv,
 * + dt fx on ux, then cutcell_fastdiag_solve. */
int cutcell_hill_step(cutcell_hill* hill, cutcell_fastdiag* fd, double* ux, double* uy, double* uz, double dt,
                      double fx, void* stream);
int cutcell_hill_destroy(cutcell_hill* hill);

/* ---- batched persistent Jacobi-PCG over many uneven systems ----
 * Replaces the one-system-at-a-time loop of the reference's solver sweeps
 * (code/fast_solver_workbench.py:169-176 calling solve_cpu_cg / solve_gpu_cg,
 * code/fast_solver_backends.py:90-132,194-289) with one persistent launch.
 * Per system the iteration, stopping test and report are those of
 * cutcell_pcg_solve (FP64, precond NONE or JACOBI).
 *
 * create: n[i], nnz[i] are HOST arrays (1 <= n[i] <= 16384); indptr, indices,
 * data are DEVICE arrays holding the systems back to back: system i owns
 * n[i] + 1 row offsets (values 0..nnz[i], relative to the system), nnz[i]
 * column indices (0..n[i]-1, relative to the system) and nnz[i] values.  The
 * caller keeps them alive while the context exists.
 * configure: the launch shape and, per system (HOST arrays of n_problems),
 * lanes_per_row (power of two <= 32) and the claim order (a permutation;
 * teams take systems in this order, heaviest first).  A team is a cluster of
 * `cluster` CTAs; up to smem_matrix bytes of shared memory per CTA hold the
 * CTA's CSR slice when it fits (else it is read from global memory).
 * solve: rhs / x are DEVICE arrays packed like the rows (system i at
 * sum_{j<i} n[j]); reports is a HOST array of n_problems.  The solve is a
 * captured CUDA graph (reset of the work counter, the persistent kernel, the
 * copy of the per-system results), re-captured when the arguments or the
 * configuration change; the call waits for it.  elapsed_ms is the device
 * time of the whole batch; blocks is the cluster size.  Returns
 * CUTCELL_E_SHAPE if a system's CSR arrays are malformed (that system's
 * report has status CUTCELL_E_SHAPE), else CUTCELL_OK; per-system outcomes
 * are in the reports. */
typedef struct cutcell_batch cutcell_batch;
typedef struct {
    int32_t cluster;      /* CTAs per team: 1, 2, 4, 8 or 16 (16 is a non-portable cluster size) */
    int32_t threads;      /* threads per CTA: multiple of 32, <= 512 */
    int32_t smem_matrix;  /* bytes per CTA for a staged CSR slice (multiple of 16; 0 = never stage) */
    int32_t teams;        /* concurrent teams (0 = as many as fit, at most n_problems) */
} CutcellBatchConfig;
int cutcell_batch_create(int32_t n_problems, const int32_t* n, const int32_t* nnz, const int32_t* indptr,
                         const int32_t* indices, const double* data, cutcell_batch** out);
int cutcell_batch_configure(cutcell_batch* batch, const CutcellBatchConfig* cfg, const int32_t* lanes_per_row,
                            const int32_t* order);
/* teams launched and dynamic shared memory per CTA of the current configuration */
int cutcell_batch_info(const cutcell_batch* batch, int32_t* teams, int32_t* smem_bytes);
int cutcell_batch_solve(cutcell_batch* batch, const double* rhs, double* x, double tol, int32_t maxiter,
                        int32_t precond, CutcellReport* reports, void* stream);
/* Per-system timeline of the last solve (HOST arrays of n_problems, any may be
 * NULL): start / end in microseconds from the first system's start (device
 * global timer) and the team that solved it. */
int cutcell_batch_timeline(const cutcell_batch* batch, double* start_us, double* end_us, int32_t* team);
int cutcell_batch_destroy(cutcell_batch* batch);

/* Allocation-free Jacobi-PCG on a device CSR matrix.  No counterpart in the
 * reference: it serves callers that cannot allocate device memory when they
 * solve (a framework's caching allocator holding the device, loops that must
 * not take the synchronisation of cudaMalloc/cudaFree, fixed memory budgets).
 * Same algorithm, arguments and report as cutcell_pcg_create_csr +
 * cutcell_pcg_solve (FP64, precond NONE or JACOBI), but every working array
 * lives in one fixed file-scope device array of the library, sized for
 * n <= 65536 unknowns and <= 1024 persistent blocks (about 2.2 MB per GPU,
 * held until the process exits).  Larger n returns CUTCELL_E_SHAPE.  The
 * first call on each device resolves the array's address and the grid size.
 * Every call copies the result to the host and synchronises its stream, so
 * the call is not meant for stream capture.  Calls share the array:
 * calls that overlap on the GPU race and must be serialised by the caller.
 * The CSR structure is checked on the device first (as in
 * cutcell_pcg_create_csr); a malformed matrix returns CUTCELL_E_SHAPE
 * without being read further.  Solver outcomes (maximum iterations reached,
 * breakdown, non-finite residual) are reported in report->status, as with
 * cutcell_pcg_solve, and the call returns CUTCELL_OK for them; pass a report
 * to see them.  The call waits for its stream before it returns.
 * report->elapsed_ms is 0 (no events are created on this path).
 * cutcell_noalloc_last_error: the message of this thread's last failed call
 * (empty after a call that returned CUTCELL_OK). */
int cutcell_pcg_solve_csr_noalloc(int32_t n, int32_t nnz, const int32_t* indptr, const int32_t* indices,
                                  const double* data, const double* b, double* x, double tol, int32_t maxiter,
                                  int32_t precond, CutcellReport* report, void* stream);
const char* cutcell_noalloc_last_error(void);

/* Bounded waits.  Every device-wide wait of the persistent kernels (grid
 * barriers) gives up after a limit of global-timer (wall-clock) time, sets
 * CUTCELL_E_BARRIER and returns, leaving the context usable.  The limit is
 * process-wide: 10 s by default, or CUTCELL_WAIT_LIMIT_S from the environment
 * at the first launch; set_wait_limit takes seconds in [1e-3, 3600].
 * barrier_selftest runs one grid barrier over `blocks` co-resident blocks that
 * waits for `arrivals` arrivals on the current device and stream 0, and
 * stores the device's status: CUTCELL_OK when arrivals <= blocks, and
 * CUTCELL_E_BARRIER after the limit when arrivals > blocks (nothing ever
 * completes that barrier).  No counterpart in the reference (diagnostics). */
int cutcell_set_wait_limit(double seconds);
double cutcell_get_wait_limit(void);
int cutcell_barrier_selftest(int32_t blocks, int32_t arrivals, int32_t* status_out);

int cutcell_destroy(cutcell_ctx* ctx);
const char* cutcell_status_string(int status);
/* Last CUDA error text seen by the library (diagnostics). */
const char* cutcell_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* CUTCELL_B200_H */
