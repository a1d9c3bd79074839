/*
 * cutcell_setup.h -- native host setup of cut-element blocks
 * (libcutcell_setup.so, C++17 + OpenMP, no GPU).
 *
 * Replaces the per-cell Python loops of the reference's cut assembly
 * (assemble_oblique_cut_matrices, code/oblique_cut_sbp.py:271-433, lifted to
 * 3D; assemble_bell_3d, code/bell_3d_core.py:338-390) for implicit geometries:
 * each cut cell's dense (p+1)^3 x (p+1)^3 block
 *   a_mass M + a_stiff K + nitsche (-N - N^T + beta Mb)
 * (weak penalty of code/cut_3d_sbp.py:426-460), the diagonal of its fluid mass,
 * its fluid volume and its load.  All pointers are HOST pointers.
 * Returns 0 on success, 7 on invalid arguments.
 */
#ifndef CUTCELL_SETUP_H
#define CUTCELL_SETUP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int32_t n_elements;       /* per axis, unit box */
    int32_t degree;
    int32_t subdiv;           /* sub-cells per cell edge for the level-set interpolation */
    int32_t box_faces;        /* integrate unit-box faces inside the cell as boundary */
    int32_t n_cells;
    int32_t n_tet, n_tri, n_tet_load, n_tri_load;
    int32_t pad;
    const int32_t* cells;     /* [n_cells][3] element indices (ex, ey, ez) */
    const double* corner_phi; /* [n_cells][(subdiv+1)^3] level set at sub-cell corners, x fastest */
    const double* knots;      /* open-uniform knot vector, n + 2p + 1 entries */
    const double* tet_rule;   /* [n_tet][4] barycentric (a, b, c) and weight (sum 1/6) */
    const double* tri_rule;   /* [n_tri][3] (a, b) and weight (sum 1/2) */
    const double* tet_load;   /* rules for the load integrals */
    const double* tri_load;
    double a_mass, a_stiff, nitsche, beta;
} CutcellSetupDesc;

/* Load-rule point counts per cell (volume, boundary). */
int cutcell_setup_count(const CutcellSetupDesc* d, int64_t* nvol_load, int64_t* nsurf_load);
/* Load-rule points (xyz) at the given per-cell offsets. */
int cutcell_setup_load_points(const CutcellSetupDesc* d, const int64_t* vol_off, const int64_t* surf_off, double* xv,
                              double* xs);
/* Blocks [n_cells][P][P], fluid-mass diagonals [n_cells][P], volumes [n_cells] and
 * loads [n_cells][P] (forcing values fvals at the load volume points, Dirichlet
 * values gvals at the load boundary points; either may be NULL). */
int cutcell_setup_blocks(const CutcellSetupDesc* d, const int64_t* vol_off, const int64_t* surf_off,
                         const double* fvals, const double* gvals, double* blocks, double* mass_diag, double* volume,
                         double* load);
/* Set (n > 0) and return the OpenMP thread count. */
int cutcell_setup_threads(int n);

#ifdef __cplusplus
}
#endif

#endif /* CUTCELL_SETUP_H */
