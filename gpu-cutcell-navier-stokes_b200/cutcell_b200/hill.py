"""Periodic-hill fast diagonalisation with the interface of ``FastDiagHill``
(cpp/include/cut/hill_fastdiag.h:20-80).

``build`` forms the z symbols and the per-mode dense inverses on the host
(the reference builds them the same way, :26-43, by Gauss-Jordan; here by
LAPACK), uploads them once, and ``solve`` runs the device solve of
libcutcell_b200.so (DFT in z, per-mode inverse streaming, shared-operator
products, inverse DFT).  Fields are FieldH arrays of shape (nr, nz),
``v[m*nz + iz]`` (cpp/include/cut/hill3d.h:182-187).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


def z_symbols(Mz_row, Sz_row, Kz_row):
    """mu_k, sig_k, kap_k by DFT of the circulant first rows (:31-33)."""
    nz = len(Mz_row)
    jk = np.outer(np.arange(nz), np.arange(nz))
    ang = 2 * np.pi * (jk % nz) / nz
    return np.cos(ang) @ np.asarray(Mz_row), np.cos(ang) @ np.asarray(Sz_row), np.sin(ang) @ np.asarray(Kz_row)


def mode_inverses(M2, Qx2, Qy2, KN2, mu, sig, kap, a):
    """Ainv_k = ((mu_k + a sig_k) M2 + a mu_k KN2)^{-1} and the Schur inverses
    Sinv_k = (mu_k^2 (Qx2 Ainv_k Qx2^T + Qy2 Ainv_k Qy2^T) + kap_k^2 M2 Ainv_k M2)^{-1}."""
    nz = len(mu)
    nr = M2.shape[0]
    Ainv = np.empty((nz, nr, nr))
    Sinv = np.empty((nz, nr, nr))
    for k in range(nz):
        Ak = (mu[k] + a * sig[k]) * M2 + a * mu[k] * KN2
        Ai = np.linalg.inv(Ak)
        Sk = mu[k] ** 2 * (Qx2 @ Ai @ Qx2.T + Qy2 @ Ai @ Qy2.T) + kap[k] ** 2 * (M2 @ Ai @ M2)
        Ainv[k] = Ai
        Sinv[k] = np.linalg.inv(Sk)
    return Ainv, Sinv


def _dgemm_nt(lib, M, N, K, A, lda, sA, B, ldb, sB, s, sS, C, ldc, sC, batch, beta=0.0):
    _lib.check(lib.cutcell_dgemm_nt(M, N, K, A.data_ptr(), lda, sA, B.data_ptr(), ldb, sB,
                                    s.data_ptr() if s is not None else None, sS, beta, C.data_ptr(), ldc, sC, batch,
                                    _lib.current_stream_ptr()), "cutcell_dgemm_nt")


def mode_operators_gpu(M2, Qx2, Qy2, KN2, mu, sig, kap, a, device="cuda", timings=None):
    """The per-mode operators of FastDiagHill::build (hill_fastdiag.h:26-43)
    through one shared generalised eigenbasis instead of 2 nz dense
    inversions of nr x nr matrices (the Lynch-Rice-Thomas form of
    cpp/include/solvers/fastdiag3.h:29-92):

    * KN2 Phi = M2 Phi diag(lam), Phi^T M2 Phi = I (host LAPACK, once), so
      A_k = (mu_k + a sig_k) M2 + a mu_k KN2 = Phi^-T diag(c1 + c2 lam) Phi^-1
      and A_k^{-1} = Phi diag(d_k) Phi^T, d_k = 1 / (c1_k + c2_k lam);
    * with G = [Qx2 Phi | Qy2 Phi | M2 Phi] the Schur complement is
      S_k = G diag(mu_k^2 d_k, mu_k^2 d_k, kap_k^2 d_k) G^T;
    * modes k and nz - k share mu, sig and kap^2, so only nz/2 + 1 distinct
      modes are built.
    The products run on the device (cutcell_dgemm_nt, FP64 tensor cores);
    each S_k is inverted on the host (LAPACK, symmetric).  Returns device
    tensors Ainv, Sinv of shape (nz, nr, nr)."""
    import time

    import scipy.linalg
    import torch

    lib = _lib.load()
    dv = torch.device(device)
    f64 = torch.float64
    T = {} if timings is None else timings
    t0 = time.perf_counter()
    M2 = np.asarray(M2, dtype=float)
    KN2 = np.asarray(KN2, dtype=float)
    lam, Phi = scipy.linalg.eigh(0.5 * (KN2 + KN2.T), 0.5 * (M2 + M2.T))
    T["eigh_s"] = time.perf_counter() - t0
    nr, nz = M2.shape[0], len(mu)
    kd = np.arange(nz // 2 + 1)
    c1 = np.asarray(mu)[kd] + a * np.asarray(sig)[kd]
    c2 = a * np.asarray(mu)[kd]
    d = 1.0 / (c1[:, None] + c2[:, None] * lam[None, :])  # (K, nr)
    w = np.concatenate([(np.asarray(mu)[kd] ** 2)[:, None] * d, (np.asarray(mu)[kd] ** 2)[:, None] * d,
                        (np.asarray(kap)[kd] ** 2)[:, None] * d], axis=1)  # (K, 3 nr)
    t1 = time.perf_counter()
    up = lambda x: torch.as_tensor(np.ascontiguousarray(x), dtype=f64).to(dv)
    Phi_d, PhiT_d = up(Phi), up(Phi.T)
    G = torch.empty((nr, 3 * nr), dtype=f64, device=dv)
    for j, Op in enumerate((Qx2, Qy2, M2)):
        Od = up(Op)
        _dgemm_nt(lib, nr, nr, nr, Od, nr, 0, PhiT_d, nr, 0, None, 0, G[:, j * nr:], 3 * nr, 0, 1)
    K = kd.size
    d_d, w_d = up(d), up(w)
    Ainv = torch.empty((nz, nr, nr), dtype=f64, device=dv)
    _dgemm_nt(lib, nr, nr, nr, Phi_d, nr, 0, Phi_d, nr, 0, d_d, nr, Ainv, nr, nr * nr, K)
    S = torch.empty((K, nr, nr), dtype=f64, device=dv)
    _dgemm_nt(lib, nr, nr, 3 * nr, G, 3 * nr, 0, G, 3 * nr, 0, w_d, 3 * nr, S, nr, nr * nr, K)
    torch.cuda.synchronize(dv)
    T["device_gemm_s"] = time.perf_counter() - t1
    T["device_gemm_flop"] = 2.0 * nr * nr * nr * 3 + 2.0 * nr * nr * nr * K + 2.0 * nr * nr * 3 * nr * K
    t2 = time.perf_counter()
    Sh = S.cpu().numpy()
    Sinv = torch.empty((nz, nr, nr), dtype=f64, device=dv)
    for k in range(K):
        Sk = 0.5 * (Sh[k] + Sh[k].T)
        Sinv[k].copy_(torch.as_tensor(np.linalg.inv(Sk)))
    T["schur_inverse_s"] = time.perf_counter() - t2
    for k in range(K, nz):  # modes nz - k
        Ainv[k].copy_(Ainv[nz - k])
        Sinv[k].copy_(Sinv[nz - k])
    torch.cuda.synchronize(dv)
    T["total_s"] = time.perf_counter() - t0
    return Ainv, Sinv


class FastDiagHill:
    def __init__(self, device="cuda"):
        import torch

        self.device = torch.device(device)
        self._lib = _lib.load()
        self._ctx = None

    def build(self, M2, Qx2, Qy2, KN2, Mz_row, Sz_row, Kz_row, a, *, inverses=None, on_device: bool = False):
        """FastDiagHill::build.  ``on_device=True`` forms the per-mode
        operators through the shared eigenbasis on the device
        (mode_operators_gpu); otherwise by dense host inversion as the
        reference does.  ``inverses=(Ainv, Sinv)`` may be supplied instead."""
        import torch

        self.nr = int(M2.shape[0])
        self.nz = int(len(Mz_row))
        self.a = float(a)
        self.mu, self.sig, self.kap = z_symbols(Mz_row, Sz_row, Kz_row)
        self.build_timings = {}
        if inverses is None and on_device:
            if KN2 is None:
                raise ValueError("KN2 is needed to form the inverses")
            inverses = mode_operators_gpu(M2, Qx2, Qy2, KN2, self.mu, self.sig, self.kap, float(a), self.device,
                                          self.build_timings)
        if inverses is None:
            if KN2 is None:
                raise ValueError("KN2 is needed to form the inverses")
            inverses = mode_inverses(np.asarray(M2), np.asarray(Qx2), np.asarray(Qy2), np.asarray(KN2), self.mu, self.sig, self.kap, self.a)
        dv = self.device
        f64 = torch.float64
        t = lambda x: torch.as_tensor(x, dtype=f64).to(dv).contiguous()
        self._t = {
            "M2": t(M2), "Qx2": t(Qx2), "Qy2": t(Qy2), "mu": t(self.mu), "kap": t(self.kap),
            "Ainv": t(inverses[0]), "Sinv": t(inverses[1]),
        }
        self.close()
        ctx = C.c_void_p()
        T = self._t
        _lib.check(
            self._lib.cutcell_fastdiag_create(
                self.nr, self.nz, T["M2"].data_ptr(), T["Qx2"].data_ptr(), T["Qy2"].data_ptr(), T["mu"].data_ptr(),
                T["kap"].data_ptr(), T["Ainv"].data_ptr(), T["Sinv"].data_ptr(), C.byref(ctx),
            ),
            "cutcell_fastdiag_create",
        )
        self._ctx = ctx
        return self

    def solve_device(self, ux, uy, uz, out=None):
        import torch

        ins = [torch.as_tensor(u, dtype=torch.float64, device=self.device).contiguous() for u in (ux, uy, uz)]
        outs = out or [torch.empty_like(ins[0]) for _ in range(3)]
        _lib.check(
            self._lib.cutcell_fastdiag_solve(
                self._ctx, *(u.data_ptr() for u in ins), *(o.data_ptr() for o in outs), _lib.current_stream_ptr()
            ),
            "cutcell_fastdiag_solve",
        )
        return outs

    def solve(self, ux, uy, uz):
        """FastDiagHill::solve with host arrays in and out."""
        return [o.cpu().numpy() for o in self.solve_device(ux, uy, uz)]

    def close(self):
        if getattr(self, "_ctx", None):
            self._lib.cutcell_fastdiag_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- advection (hill_skew_conv) and the fast step (hill_fastdiag_step) ----


def z_element_tables(Vz, dVz, wz, nz):
    """Per z element: its (p+1) basis functions in periodic order and their
    values / derivatives at the element's quadrature points.

    The z quadrature nodes are grouped by element (cpp/include/cut/hill3d.h:
    153-160: element e owns nodes e*qpe .. e*qpe+qpe-1).  The band of element e
    must be the periodic run (e - s + j) mod nz, j = 0..nzb-1, with the same
    shift s for every element (uniform periodic B-splines), so that element e
    writes mode (e - s + j) mod nz in scatter round j without conflicts."""
    Vz, dVz, wz = np.asarray(Vz), np.asarray(dVz), np.asarray(wz)
    nzq = Vz.shape[0]
    qpe = nzq // nz
    if qpe * nz != nzq:
        raise ValueError("z quadrature is not a whole number of points per element")
    bands = []
    for e in range(nz):
        rows = slice(e * qpe, (e + 1) * qpe)
        cols = np.nonzero((np.abs(Vz[rows]) + np.abs(dVz[rows])).sum(0))[0]
        k = cols.size
        start = None
        for c0 in cols:
            if {int((c0 + j) % nz) for j in range(k)} == set(int(c) for c in cols):
                start = int(c0)
                break
        if start is None:
            raise ValueError(f"z element {e}: basis functions are not a periodic run")
        bands.append([(start + j) % nz for j in range(k)])
    nzb = len(bands[0])
    shifts = {(e - b[0]) % nz for e, b in enumerate(bands)}
    if any(len(b) != nzb for b in bands) or len(shifts) != 1:
        raise ValueError("z bands are not a uniform periodic shift")
    zb = np.array(bands, dtype=np.int32)
    Vl = np.stack([Vz[e * qpe : (e + 1) * qpe][:, zb[e]] for e in range(nz)])
    dVl = np.stack([dVz[e * qpe : (e + 1) * qpe][:, zb[e]] for e in range(nz)])
    wzl = wz.reshape(nz, qpe)
    return zb, Vl, dVl, wzl, qpe


def segment_tables(ptr, idx, seg_max=128, long_pattern=16, seg_max_long=32):
    """Segments of consecutive 2D points whose sample rows have the same mode
    pattern (at most seg_max points each; at most seg_max_long for patterns
    longer than long_pattern modes, which the device runs as a separate,
    smaller launch that should still spread over every SM), their patterns,
    and for every reduced mode the partial rows (segment pattern slots) that
    feed it, in segment order."""
    ptr = np.asarray(ptr, dtype=np.int64)
    idx = np.asarray(idx, dtype=np.int64)
    n2q = ptr.size - 1
    q0s, q1s, pats = [], [], []
    q = 0
    while q < n2q:
        pat = idx[ptr[q] : ptr[q + 1]]
        cap = seg_max if pat.size <= long_pattern else seg_max_long
        r = q + 1
        while r < n2q and r - q < cap and ptr[r + 1] - ptr[r] == pat.size and np.array_equal(idx[ptr[r] : ptr[r + 1]], pat):
            r += 1
        q0s.append(q)
        q1s.append(r)
        pats.append(pat)
        q = r
    seg_len = np.array([p.size for p in pats], dtype=np.int32)
    seg_pat = np.concatenate([[0], np.cumsum(seg_len)[:-1]]).astype(np.int32)
    pat_idx = np.concatenate(pats).astype(np.int32)
    order = np.argsort(pat_idx, kind="stable")  # by mode, then by partial row (segment order)
    nr = int(pat_idx.max()) + 1 if pat_idx.size else 0
    g_ptr = np.zeros(nr + 1, dtype=np.int32)
    np.add.at(g_ptr, pat_idx + 1, 1)
    g_ptr = np.cumsum(g_ptr).astype(np.int32)
    return {
        "seg_q0": np.array(q0s, np.int32), "seg_q1": np.array(q1s, np.int32), "seg_pat": seg_pat,
        "seg_len": seg_len, "pat_idx": pat_idx, "g_ptr": g_ptr, "g_ent": order.astype(np.int32),
    }


class HillAdvection:
    """Device advection of the periodic hill (hill_skew_conv of all three
    components) and the fast step, from Hill3D's sample machinery.

    ``phi, dpx, dpy``: scipy CSR (n2q x nr) sample rows on one pattern
    (sp_idx / sp_phi / sp_dpx / sp_dpy); ``w2`` (n2q); ``Vz, dVz`` (nzq x nz);
    ``wz`` (nzq); ``M2inv`` (nr x nr), ``Mzinv`` (nz x nz)."""

    def __init__(self, phi, dpx, dpy, w2, Vz, dVz, wz, M2inv, Mzinv, device="cuda", seg_max=128):
        import torch

        self._lib = _lib.load()
        self.device = torch.device(device)
        phi, dpx, dpy = phi.tocsr(), dpx.tocsr(), dpy.tocsr()
        for other in (dpx, dpy):
            if not (np.array_equal(other.indptr, phi.indptr) and np.array_equal(other.indices, phi.indices)):
                raise ValueError("phi, dpx and dpy must share one sparsity pattern")
        self.n2q, self.nr = phi.shape
        self.nz = int(np.asarray(Vz).shape[1])
        zb, Vl, dVl, wzl, qpe = z_element_tables(Vz, dVz, wz, self.nz)
        seg = segment_tables(phi.indptr, phi.indices, seg_max)
        if seg["g_ptr"].size - 1 < self.nr:
            seg["g_ptr"] = np.concatenate([seg["g_ptr"], np.full(self.nr + 1 - seg["g_ptr"].size, seg["g_ptr"][-1], np.int32)])
        self.tables = seg
        dv = self.device
        ti = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.int32)).to(dv)
        tf = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).to(dv)
        self._t = {
            **{k: ti(v) for k, v in seg.items()},
            "sp_ptr": ti(phi.indptr), "phi": tf(phi.data), "dpx": tf(dpx.data), "dpy": tf(dpy.data), "w2": tf(w2),
            "zb": ti(zb), "Vl": tf(Vl), "dVl": tf(dVl), "wzl": tf(wzl), "Mzinv": tf(Mzinv), "M2inv": tf(M2inv),
        }
        T = self._t
        desc = _lib.CutcellHillDesc(
            self.nr, self.nz, int(qpe), int(zb.shape[1]), int(seg["seg_len"].size), int(seg["seg_len"].max()),
            int(seg["pat_idx"].size), int(self.n2q),
            *(T[k].data_ptr() for k in ("seg_q0", "seg_q1", "seg_pat", "seg_len", "pat_idx", "sp_ptr", "phi", "dpx",
                                        "dpy", "w2", "zb", "Vl", "dVl", "wzl", "g_ptr", "g_ent", "Mzinv", "M2inv")),
        )
        ctx = C.c_void_p()
        _lib.check(self._lib.cutcell_hill_create(C.byref(desc), C.byref(ctx)), "cutcell_hill_create")
        self._ctx = ctx

    def _fields(self, u):
        import torch

        return [torch.as_tensor(c, dtype=torch.float64, device=self.device).contiguous() for c in u]

    def skew_conv(self, ux, uy, uz):
        """hill_skew_conv(w = u, u_c) for the three components (device tensors)."""
        import torch

        ins = self._fields((ux, uy, uz))
        outs = [torch.empty_like(ins[0]) for _ in range(3)]
        _lib.check(
            self._lib.cutcell_hill_skew_conv(self._ctx, *(t.data_ptr() for t in ins), *(o.data_ptr() for o in outs),
                                             _lib.current_stream_ptr()),
            "cutcell_hill_skew_conv",
        )
        return outs

    def step(self, fd: "FastDiagHill", u, dt: float, fx: float = 0.0):
        """hill_fastdiag_step in place on the three device fields ``u``."""
        _lib.check(
            self._lib.cutcell_hill_step(self._ctx, fd._ctx, *(t.data_ptr() for t in u), float(dt), float(fx),
                                        _lib.current_stream_ptr()),
            "cutcell_hill_step",
        )
        return u

    def close(self):
        if getattr(self, "_ctx", None):
            self._lib.cutcell_hill_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cubic_bspline(t):
    """Centred cardinal cubic B-spline and its derivative (support |t| < 2)."""
    a = np.abs(t)
    v = np.where(a < 1, 2.0 / 3.0 - a**2 + 0.5 * a**3, np.where(a < 2, (2.0 - a) ** 3 / 6.0, 0.0))
    dv = np.where(a < 1, -2.0 * a + 1.5 * a**2, np.where(a < 2, -0.5 * (2.0 - a) ** 2, 0.0)) * np.sign(t)
    return v, dv


def synthetic_machinery(nr=2345, nz=32, cells=(64, 32), pts_per_cell=196, modes_per_row=16, Lz=4.5, seed=20260629):
    """Seeded stand-in for Hill3D's sample machinery at a given size: each 2D
    cell's points share one pattern of ``modes_per_row`` reduced modes (a
    window of the mode range moving with the cell), values and weights are
    random; the z basis is the periodic cubic B-spline on nz elements with
    9 Gauss points each.  Used for timing and for device-vs-oracle checks
    where the reference machinery is not available."""
    import scipy.sparse as sp

    rng = np.random.default_rng(seed)
    ncell = cells[0] * cells[1]
    n2q = ncell * pts_per_cell
    starts = (np.arange(ncell) * (nr - modes_per_row)) // max(ncell - 1, 1)
    cols = (starts[:, None] + np.arange(modes_per_row)[None, :])
    idx = np.repeat(cols, pts_per_cell, axis=0).ravel()
    ptr = np.arange(n2q + 1) * modes_per_row
    mk = lambda scale: sp.csr_matrix((rng.standard_normal(idx.size) * scale, idx, ptr), shape=(n2q, nr))
    phi, dpx, dpy = mk(0.3), mk(2.0), mk(2.0)
    w2 = rng.uniform(0.5, 1.5, n2q) / n2q
    hz = Lz / nz
    g, gw = np.polynomial.legendre.leggauss(9)
    zq = ((np.arange(nz)[:, None] + 0.5 * (g[None, :] + 1.0)) * hz).ravel()
    wz = np.tile(0.5 * gw * hz, nz)
    d = zq[:, None] - hz * np.arange(nz)[None, :]
    d -= Lz * np.floor(d / Lz + 0.5)
    Vz, dVz = cubic_bspline(d / hz)
    dVz = dVz / hz
    A = rng.standard_normal((nr, nr)) / np.sqrt(nr)
    M2inv = np.eye(nr) + 0.1 * (A + A.T)
    Mzinv = np.eye(nz) + 0.05 * np.roll(np.eye(nz), 1, 1) + 0.05 * np.roll(np.eye(nz), -1, 1)
    return {"phi": phi, "dpx": dpx, "dpy": dpy, "w2": w2, "Vz": Vz, "dVz": dVz, "wz": wz, "M2inv": M2inv,
            "Mzinv": Mzinv, "nr": nr, "nz": nz}
