// Driver that runs the REFERENCE's own periodic-hill fast-diagonalisation
// (Hill3D::build, FastDiagHill::build/solve from cpp/include/cut/hill3d.h and
// hill_fastdiag.h, included from the reference tree at build time) on seeded
// random fields and dumps operators, symbols, inputs and outputs as raw
// doubles.  Test infrastructure: it generates the golden vectors that pin the
// NumPy restatement (oracle/hill.py) and the device solve.
//
//   hill_ref <ne> <nz> <seed> <out.bin> [steps] [physical]
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "hill3d.h"
#include "hill_fastdiag.h"

static void put(FILE* f, const std::vector<double>& v) { fwrite(v.data(), sizeof(double), v.size(), f); }

int main(int argc, char** argv) {
    if (argc < 5) {
        std::fprintf(stderr, "usage: hill_ref ne nz seed out.bin [steps] [physical]\n");
        return 2;
    }
    const int ne = std::atoi(argv[1]), nz = std::atoi(argv[2]), seed = std::atoi(argv[3]);
    const int steps = argc > 5 ? std::atoi(argv[5]) : 0;
    const bool physical = argc > 6 && std::atoi(argv[6]) != 0;
    const int p = 3;
    const double Lz = 4.5, a = 0.01, dt = 0.02, fx = 0.7;
    Hill3D H;
    H.build(ne, p, nz, Lz, physical);
    FastDiagHill fd;
    fd.build(H, a);
    const int nr = fd.nr;
    srand(seed);
    HillNS s;
    s.ux = FieldH(nr, nz);
    s.uy = FieldH(nr, nz);
    s.uz = FieldH(nr, nz);
    for (auto* f : {&s.ux, &s.uy, &s.uz})
        for (auto& v : f->v) v = (double)rand() / RAND_MAX - 0.5;
    auto out = fd.solve(s.ux, s.uy, s.uz);
    FILE* f = std::fopen(argv[4], "wb");
    double hdr[4] = {(double)nr, (double)nz, a, (double)steps};
    fwrite(hdr, sizeof(double), 4, f);
    put(f, H.M2.a);
    put(f, H.Qx2.a);
    put(f, H.Qy2.a);
    put(f, H.KN2.a);
    std::vector<double> zr(3 * nz);
    for (int j = 0; j < nz; ++j) {
        zr[j] = H.Z.M(0, j);
        zr[nz + j] = H.Sz(0, j);
        zr[2 * nz + j] = H.Kz(0, j);
    }
    put(f, zr);
    put(f, fd.mu);
    put(f, fd.sig);
    put(f, fd.kap);
    put(f, s.ux.v);
    put(f, s.uy.v);
    put(f, s.uz.v);
    put(f, out[0].v);
    put(f, out[1].v);
    put(f, out[2].v);
    // the Galerkin sample / load machinery (hill3d.h:86-93) and the mass inverses
    {
        double dims[2] = {(double)H.n2q, (double)H.nzq};
        fwrite(dims, sizeof(double), 2, f);
        std::vector<double> ptr(H.n2q + 1, 0.0), idx, phi, dpx, dpy;
        for (int q = 0; q < H.n2q; ++q) {
            ptr[q + 1] = ptr[q] + (double)H.sp_idx[q].size();
            for (size_t a = 0; a < H.sp_idx[q].size(); ++a) {
                idx.push_back((double)H.sp_idx[q][a]);
                phi.push_back(H.sp_phi[q][a]);
                dpx.push_back(H.sp_dpx[q][a]);
                dpy.push_back(H.sp_dpy[q][a]);
            }
        }
        double nnz = (double)idx.size();
        fwrite(&nnz, sizeof(double), 1, f);
        put(f, ptr);
        put(f, idx);
        put(f, phi);
        put(f, dpx);
        put(f, dpy);
        put(f, H.w2);
        put(f, H.Vz.a);
        put(f, H.dVz.a);
        put(f, H.wz);
        put(f, H.M2inv.a);
        put(f, H.Mzinv.a);
        // one skew-symmetric convection of each component by the sampled field
        QField wx = hill_sample(H, s.ux), wy = hill_sample(H, s.uy), wz = hill_sample(H, s.uz);
        put(f, hill_skew_conv(H, wx, wy, wz, s.ux).v);
        put(f, hill_skew_conv(H, wx, wy, wz, s.uy).v);
        put(f, hill_skew_conv(H, wx, wy, wz, s.uz).v);
    }
    if (steps > 0) {
        HillNS st = s;
        const auto t0 = std::chrono::steady_clock::now();
        for (int k = 0; k < steps; ++k) hill_fastdiag_step(H, fd, st, dt, fx);
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        std::fprintf(stderr, "step_ms=%.3f\n", ms / steps);
        put(f, st.ux.v);
        put(f, st.uy.v);
        put(f, st.uz.v);
    }
    std::fclose(f);
    std::printf("nr=%d nz=%d\n", nr, nz);
    return 0;
}
