// Native host setup of cut-element blocks (OpenMP over cut cells).
//
// Same geometry and rules as cutcell_b200/cutgeom.py: every cut cell (split
// into subdiv^3 sub-cells) is divided into the six Kuhn tetrahedra, the level
// set is interpolated linearly on each tetrahedron, the tetrahedron is clipped
// by phi_lin >= 0 (a tetrahedron or a prism, split into <= 3 tetrahedra), the
// zero set becomes one or two triangles, and tetrahedron faces on the unit-box
// boundary are clipped the same way.  This is the 3D lift of the reference's
// 2D clip + Duffy pipeline (code/oblique_cut_sbp.py:121-248, 271-433); the
// element blocks are the reference's local Gram updates
// (code/oblique_cut_sbp.py:323-359) with the weak-penalty terms of
// code/cut_3d_sbp.py:426-460.  The quadrature rules (conical product on the
// tetrahedron, collapsed rule on the triangle) are passed in from Python.
#include "../../include/cutcell_setup.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct V3 {
    double x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double norm(V3 a) { return std::sqrt(dot(a, a)); }
inline double comp(V3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }

// Kuhn tetrahedra of the unit cube (corner id = x + 2y + 4z), one per axis
// permutation, in itertools.permutations order.
const int KUHN[6][4] = {{0, 1, 3, 7}, {0, 1, 5, 7}, {0, 2, 3, 7}, {0, 2, 6, 7}, {0, 4, 5, 7}, {0, 4, 6, 7}};
const int TFACE[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};

struct Piece {
    V3 v[4];
};
struct Tri {
    V3 v[3];
    V3 n;
};

inline V3 edge_pt(V3 a, V3 b, double fa, double fb) {
    const double t = fa / (fa - fb);
    return a + t * (b - a);
}

void prism(const V3 A[3], const V3 B[3], std::vector<Piece>& out) {
    out.push_back({{A[0], A[1], A[2], B[0]}});
    out.push_back({{A[1], A[2], B[0], B[1]}});
    out.push_back({{A[2], B[0], B[1], B[2]}});
}

// clip tetrahedron by f >= 0: fluid tetrahedra and zero-set triangles
void clip_tet(const V3 P[4], const double f[4], std::vector<Piece>& vol, std::vector<Tri>& surf, V3 nrm) {
    int pos[4], neg[4], np_ = 0, nn = 0;
    for (int i = 0; i < 4; ++i) {
        if (f[i] >= 0.0)
            pos[np_++] = i;
        else
            neg[nn++] = i;
    }
    if (nn == 0) {
        vol.push_back({{P[0], P[1], P[2], P[3]}});
        return;
    }
    if (np_ == 0) return;
    if (np_ == 1) {
        const int a = pos[0];
        V3 q[3];
        for (int k = 0; k < 3; ++k) q[k] = edge_pt(P[a], P[neg[k]], f[a], f[neg[k]]);
        vol.push_back({{P[a], q[0], q[1], q[2]}});
        surf.push_back({{q[0], q[1], q[2]}, nrm});
        return;
    }
    if (np_ == 3) {
        const int d = neg[0];
        V3 A[3], B[3];
        for (int k = 0; k < 3; ++k) {
            A[k] = P[pos[k]];
            B[k] = edge_pt(P[pos[k]], P[d], f[pos[k]], f[d]);
        }
        prism(A, B, vol);
        surf.push_back({{B[0], B[1], B[2]}, nrm});
        return;
    }
    const int a = pos[0], b = pos[1], c = neg[0], d = neg[1];
    V3 A[3] = {P[a], edge_pt(P[a], P[c], f[a], f[c]), edge_pt(P[a], P[d], f[a], f[d])};
    V3 B[3] = {P[b], edge_pt(P[b], P[c], f[b], f[c]), edge_pt(P[b], P[d], f[b], f[d])};
    prism(A, B, vol);
    surf.push_back({{A[1], A[2], B[2]}, nrm});
    surf.push_back({{A[1], B[2], B[1]}, nrm});
}

void clip_tri(const V3 P[3], const double f[3], V3 nrm, std::vector<Tri>& out) {
    V3 poly[4];
    int m = 0;
    for (int k = 0; k < 3; ++k) {
        const int i = k, j = (k + 1) % 3;
        if (f[i] >= 0.0) poly[m++] = P[i];
        if ((f[i] >= 0.0) != (f[j] >= 0.0)) poly[m++] = edge_pt(P[i], P[j], f[i], f[j]);
    }
    for (int k = 1; k + 1 < m; ++k) out.push_back({{poly[0], poly[k], poly[k + 1]}, nrm});
}

struct CellGeom {
    std::vector<Piece> vol;
    std::vector<Tri> surf;
    double volume = 0.0;
};

void cell_geometry(const CutcellSetupDesc& d, int c, CellGeom& g) {
    const int s = d.subdiv, s1 = s + 1;
    const double h = 1.0 / d.n_elements, hs = h / s;
    const int* cell = d.cells + 3 * c;
    const double* fc = d.corner_phi + (size_t)c * s1 * s1 * s1;
    const V3 lo = {cell[0] * h, cell[1] * h, cell[2] * h};
    g.vol.clear();
    g.surf.clear();
    g.volume = 0.0;
    for (int sz = 0; sz < s; ++sz)
        for (int sy = 0; sy < s; ++sy)
            for (int sx = 0; sx < s; ++sx) {
                V3 C[8];
                double f[8];
                bool any = false;
                for (int k = 0; k < 8; ++k) {
                    const int ix = sx + (k & 1), iy = sy + ((k >> 1) & 1), iz = sz + ((k >> 2) & 1);
                    C[k] = {lo.x + ix * hs, lo.y + iy * hs, lo.z + iz * hs};
                    f[k] = fc[(iz * s1 + iy) * s1 + ix];
                    any |= f[k] >= 0.0;
                }
                if (!any) continue;
                for (int t = 0; t < 6; ++t) {
                    V3 P[4];
                    double ft[4];
                    for (int k = 0; k < 4; ++k) {
                        P[k] = C[KUHN[t][k]];
                        ft[k] = f[KUHN[t][k]];
                    }
                    // gradient of the linear interpolant: solve J^T g = df (rows = edges)
                    V3 e1 = P[1] - P[0], e2 = P[2] - P[0], e3 = P[3] - P[0];
                    const double det = dot(e1, cross(e2, e3));
                    V3 gr = {0, 0, 0};
                    if (det != 0.0) {
                        const double d1 = ft[1] - ft[0], d2 = ft[2] - ft[0], d3 = ft[3] - ft[0];
                        V3 c23 = cross(e2, e3), c31 = cross(e3, e1), c12 = cross(e1, e2);
                        gr = (1.0 / det) * ((d1 * c23 + d2 * c31) + d3 * c12);
                    }
                    const double gn = norm(gr);
                    V3 nrm = gn > 0.0 ? (-1.0 / gn) * gr : V3{0, 0, 0};
                    const size_t nv0 = g.vol.size();
                    std::vector<Tri> st;
                    clip_tet(P, ft, g.vol, st, nrm);
                    if (gn > 0.0)
                        for (auto& tr : st) g.surf.push_back(tr);
                    for (size_t k = nv0; k < g.vol.size(); ++k) {
                        const Piece& T = g.vol[k];
                        g.volume += std::fabs(dot(T.v[1] - T.v[0], cross(T.v[2] - T.v[0], T.v[3] - T.v[0]))) / 6.0;
                    }
                    if (d.box_faces) {
                        for (int fi = 0; fi < 4; ++fi) {
                            V3 F[3];
                            double ff[3];
                            for (int k = 0; k < 3; ++k) {
                                F[k] = P[TFACE[fi][k]];
                                ff[k] = ft[TFACE[fi][k]];
                            }
                            for (int ax = 0; ax < 3; ++ax)
                                for (int side = 0; side < 2; ++side) {
                                    const double val = side ? 1.0 : 0.0;
                                    bool on = true;
                                    for (int k = 0; k < 3; ++k) on &= std::fabs(comp(F[k], ax) - val) <= 1e-14;
                                    if (!on) continue;
                                    V3 nb = {0, 0, 0};
                                    if (ax == 0) nb.x = side ? 1.0 : -1.0;
                                    if (ax == 1) nb.y = side ? 1.0 : -1.0;
                                    if (ax == 2) nb.z = side ? 1.0 : -1.0;
                                    clip_tri(F, ff, nb, g.surf);
                                }
                        }
                    }
                }
            }
}

// Cox-de Boor values and first derivatives of the p+1 functions on element e.
void local_basis(const double* t, int p, int e, double x, double* N, double* D) {
    const int span = e + p;
    double left[16], right[16], Nl[16], Np[16];
    auto eval = [&](int deg, double* out) {
        out[0] = 1.0;
        for (int j = 1; j <= deg; ++j) {
            left[j] = x - t[span + 1 - j];
            right[j] = t[span + j] - x;
            double saved = 0.0;
            for (int r = 0; r < j; ++r) {
                const double temp = out[r] / (right[r + 1] + left[j - r]);
                out[r] = saved + right[r + 1] * temp;
                saved = left[j - r] * temp;
            }
            out[j] = saved;
        }
    };
    eval(p, Np);
    eval(p - 1, Nl);
    for (int i = 0; i <= p; ++i) {
        N[i] = Np[i];
        const int g = span - p + i;
        double dv = 0.0;
        if (i >= 1) {
            const double den = t[g + p] - t[g];
            if (den > 0) dv += p * Nl[i - 1] / den;
        }
        if (i <= p - 1) {
            const double den = t[g + p + 1] - t[g + 1];
            if (den > 0) dv -= p * Nl[i] / den;
        }
        D[i] = dv;
    }
}

struct Tables {
    int P1, P;
    std::vector<double> phi, gx, gy, gz;
    explicit Tables(int p) : P1(p + 1), P(P1 * P1 * P1), phi(P), gx(P), gy(P), gz(P) {}
    void eval(const CutcellSetupDesc& d, const int* cell, V3 X) {
        double Nx[16], Dx[16], Ny[16], Dy[16], Nz[16], Dz[16];
        local_basis(d.knots, d.degree, cell[0], X.x, Nx, Dx);
        local_basis(d.knots, d.degree, cell[1], X.y, Ny, Dy);
        local_basis(d.knots, d.degree, cell[2], X.z, Nz, Dz);
        int k = 0;
        for (int c = 0; c < P1; ++c)
            for (int b = 0; b < P1; ++b)
                for (int a = 0; a < P1; ++a, ++k) {
                    phi[k] = Nz[c] * Ny[b] * Nx[a];
                    gx[k] = Nz[c] * Ny[b] * Dx[a];
                    gy[k] = Nz[c] * Dy[b] * Nx[a];
                    gz[k] = Dz[c] * Ny[b] * Nx[a];
                }
    }
};

template <class Fn>
void for_volume_points(const CellGeom& g, const double* rule, int nrule, Fn fn) {
    for (const Piece& T : g.vol) {
        V3 e1 = T.v[1] - T.v[0], e2 = T.v[2] - T.v[0], e3 = T.v[3] - T.v[0];
        const double det = std::fabs(dot(e1, cross(e2, e3)));
        if (det <= 0.0) continue;
        for (int q = 0; q < nrule; ++q) {
            const double* r = rule + 4 * q;
            V3 X = T.v[0] + ((r[0] * e1 + r[1] * e2) + r[2] * e3);
            fn(X, det * r[3]);
        }
    }
}

template <class Fn>
void for_surface_points(const CellGeom& g, const double* rule, int nrule, Fn fn) {
    for (const Tri& S : g.surf) {
        V3 e1 = S.v[1] - S.v[0], e2 = S.v[2] - S.v[0];
        const double a2 = norm(cross(e1, e2));
        if (a2 <= 0.0) continue;
        for (int q = 0; q < nrule; ++q) {
            const double* r = rule + 3 * q;
            V3 X = S.v[0] + (r[0] * e1 + r[1] * e2);
            fn(X, a2 * r[2], S.n);
        }
    }
}

}  // namespace

extern "C" {

int cutcell_setup_count(const CutcellSetupDesc* d, int64_t* nvol_load, int64_t* nsurf_load) {
    if (!d || d->degree < 1 || d->degree > 12 || d->subdiv < 1) return 7;
#pragma omp parallel for schedule(dynamic, 4)
    for (int c = 0; c < d->n_cells; ++c) {
        CellGeom g;
        cell_geometry(*d, c, g);
        nvol_load[c] = (int64_t)g.vol.size() * d->n_tet_load;
        nsurf_load[c] = (int64_t)g.surf.size() * d->n_tri_load;
    }
    return 0;
}

int cutcell_setup_load_points(const CutcellSetupDesc* d, const int64_t* vol_off, const int64_t* surf_off, double* xv,
                              double* xs) {
    if (!d) return 7;
#pragma omp parallel for schedule(dynamic, 4)
    for (int c = 0; c < d->n_cells; ++c) {
        CellGeom g;
        cell_geometry(*d, c, g);
        int64_t k = vol_off[c];
        for_volume_points(g, d->tet_load, d->n_tet_load, [&](V3 X, double) {
            xv[3 * k] = X.x;
            xv[3 * k + 1] = X.y;
            xv[3 * k + 2] = X.z;
            ++k;
        });
        k = surf_off[c];
        for_surface_points(g, d->tri_load, d->n_tri_load, [&](V3 X, double, V3) {
            xs[3 * k] = X.x;
            xs[3 * k + 1] = X.y;
            xs[3 * k + 2] = X.z;
            ++k;
        });
    }
    return 0;
}

int cutcell_setup_blocks(const CutcellSetupDesc* d, const int64_t* vol_off, const int64_t* surf_off,
                         const double* fvals, const double* gvals, double* blocks, double* mass_diag, double* volume,
                         double* load) {
    if (!d) return 7;
    const int P1 = d->degree + 1, P = P1 * P1 * P1;
#pragma omp parallel
    {
        std::vector<double> M((size_t)P * P), K((size_t)P * P), Mb((size_t)P * P), Nn((size_t)P * P);
        std::vector<double> dn(P);
        Tables tb(d->degree);
#pragma omp for schedule(dynamic, 2)
        for (int c = 0; c < d->n_cells; ++c) {
            CellGeom g;
            cell_geometry(*d, c, g);
            const int* cell = d->cells + 3 * c;
            std::fill(M.begin(), M.end(), 0.0);
            std::fill(K.begin(), K.end(), 0.0);
            std::fill(Mb.begin(), Mb.end(), 0.0);
            std::fill(Nn.begin(), Nn.end(), 0.0);
            double* ld = load ? load + (size_t)c * P : nullptr;
            if (ld) std::fill(ld, ld + P, 0.0);
            for_volume_points(g, d->tet_rule, d->n_tet, [&](V3 X, double w) {
                tb.eval(*d, cell, X);
                for (int i = 0; i < P; ++i) {
                    const double wi = w * tb.phi[i];
                    const double wx = w * tb.gx[i], wy = w * tb.gy[i], wz = w * tb.gz[i];
                    double* Mi = &M[(size_t)i * P];
                    double* Ki = &K[(size_t)i * P];
                    for (int j = i; j < P; ++j) {
                        Mi[j] += wi * tb.phi[j];
                        Ki[j] += wx * tb.gx[j] + wy * tb.gy[j] + wz * tb.gz[j];
                    }
                }
            });
            const bool surf = d->nitsche != 0.0 && !g.surf.empty();
            if (surf) {
                for_surface_points(g, d->tri_rule, d->n_tri, [&](V3 X, double w, V3 nr) {
                    tb.eval(*d, cell, X);
                    for (int j = 0; j < P; ++j) dn[j] = nr.x * tb.gx[j] + nr.y * tb.gy[j] + nr.z * tb.gz[j];
                    for (int i = 0; i < P; ++i) {
                        const double wi = w * tb.phi[i];
                        double* Mbi = &Mb[(size_t)i * P];
                        double* Ni = &Nn[(size_t)i * P];
                        for (int j = 0; j < P; ++j) {
                            Mbi[j] += wi * tb.phi[j];
                            Ni[j] += wi * dn[j];
                        }
                    }
                });
            }
            double* B = blocks + (size_t)c * P * P;
            for (int i = 0; i < P; ++i)
                for (int j = i; j < P; ++j) {
                    double v = d->a_mass * M[(size_t)i * P + j] + d->a_stiff * K[(size_t)i * P + j];
                    if (surf)
                        v += d->nitsche * (-Nn[(size_t)i * P + j] - Nn[(size_t)j * P + i] + d->beta * Mb[(size_t)i * P + j]);
                    B[(size_t)i * P + j] = v;
                    B[(size_t)j * P + i] = v;
                }
            for (int i = 0; i < P; ++i) mass_diag[(size_t)c * P + i] = M[(size_t)i * P + i];
            volume[c] = g.volume;
            if (ld) {
                int64_t k = vol_off[c];
                if (fvals)
                    for_volume_points(g, d->tet_load, d->n_tet_load, [&](V3 X, double w) {
                        tb.eval(*d, cell, X);
                        const double fw = w * fvals[k++];
                        for (int i = 0; i < P; ++i) ld[i] += fw * tb.phi[i];
                    });
                k = surf_off[c];
                if (gvals && d->nitsche != 0.0)
                    for_surface_points(g, d->tri_load, d->n_tri_load, [&](V3 X, double w, V3 nr) {
                        tb.eval(*d, cell, X);
                        const double gw = w * gvals[k++];
                        for (int i = 0; i < P; ++i) {
                            const double dni = nr.x * tb.gx[i] + nr.y * tb.gy[i] + nr.z * tb.gz[i];
                            ld[i] += gw * (d->beta * tb.phi[i] - dni);
                        }
                    });
            }
        }
    }
    return 0;
}

int cutcell_setup_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

}  // extern "C"
