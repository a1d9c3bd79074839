"""Periodic-hill fast-diagonalisation oracle (CPU, NumPy) -- test infrastructure only.

Restates ``FastDiagHill`` (cpp/include/cut/hill_fastdiag.h:20-80):

* build (:26-43): z symbols by DFT of the circulant first rows,
  ``mu_k = sum_j Mz(0,j) cos(2 pi jk/nz)``, ``sig_k`` likewise from Sz,
  ``kap_k = sum_j Kz(0,j) sin(2 pi jk/nz)``; per mode
  ``A_k = (mu_k + a sig_k) M2 + a mu_k KN2``, ``Ainv_k = A_k^{-1}``,
  ``S_k = mu_k^2 (Qx2 Ainv_k Qx2^T + Qy2 Ainv_k Qy2^T) + kap_k^2 M2 Ainv_k M2``,
  ``Sinv_k = S_k^{-1}``;
* solve (:47-79): DFT in z (``X_k = sum_iz f(:,iz) e^{-2 pi i iz k/nz}``),
  tentative velocity ``ut = Ainv_k (mu_k M2 X_k)``, divergence
  ``mu_k (Qx2 utx + Qy2 uty) + i kap_k M2 utz``, pressure ``p = Sinv_k div``,
  correction ``u = ut - Ainv_k (mu_k Qx2^T p, mu_k Qy2^T p, -i kap_k M2 p)``,
  inverse DFT with the 1/nz factor.

Fields are (nr, nz) arrays laid out as FieldH (``v[m*nz + iz]``).
"""

from __future__ import annotations

import numpy as np


def symbols(Mz_row, Sz_row, Kz_row):
    nz = len(Mz_row)
    j = np.arange(nz)
    ang = 2 * np.pi * np.outer(np.arange(nz), j) / nz
    return np.cos(ang) @ Mz_row, np.cos(ang) @ Sz_row, np.sin(ang) @ Kz_row


def build(M2, Qx2, Qy2, KN2, mu, sig, kap, a):
    nz = len(mu)
    Ainv, Sinv = [], []
    for k in range(nz):
        A = (mu[k] + a * sig[k]) * M2 + a * mu[k] * KN2
        Ai = np.linalg.inv(A)
        S = mu[k] ** 2 * (Qx2 @ Ai @ Qx2.T + Qy2 @ Ai @ Qy2.T) + kap[k] ** 2 * (M2 @ Ai @ M2)
        Ainv.append(Ai)
        Sinv.append(np.linalg.inv(S))
    return np.array(Ainv), np.array(Sinv)


def solve(M2, Qx2, Qy2, mu, kap, Ainv, Sinv, ux, uy, uz):
    nr, nz = ux.shape
    iz = np.arange(nz)
    ang = -2 * np.pi * np.outer(iz, np.arange(nz)) / nz  # (iz, k)
    F = np.exp(1j * ang)

    def dft(f):
        return f @ F  # (nr, nz): column k

    X, Y, Z = dft(ux), dft(uy), dft(uz)
    U = [np.zeros((nr, nz), complex) for _ in range(3)]
    for k in range(nz):
        ut = [Ainv[k] @ (mu[k] * (M2 @ v[:, k])) for v in (X, Y, Z)]
        div = mu[k] * (Qx2 @ ut[0]) + mu[k] * (Qy2 @ ut[1]) + 1j * kap[k] * (M2 @ ut[2])
        p = Sinv[k] @ div
        g = [mu[k] * (Qx2.T @ p), mu[k] * (Qy2.T @ p), -1j * kap[k] * (M2 @ p)]
        for c in range(3):
            U[c][:, k] = ut[c] - Ainv[k] @ g[c]
    inv = np.exp(-1j * ang).T  # (k, iz)
    return [np.real(u @ inv) / nz for u in U]


# ---- advection and the fast step (hill3d.h:245-312,519-538; hill_fastdiag.h:83-95) ----
#
# ``S`` is the sparse reduced 2D sample matrix (n2q x nr) with the rows
# sp_phi / sp_dpx / sp_dpy on the pattern sp_idx (hill3d.h:86-93, built at
# :121-151); ``Vz``/``dVz`` (nzq x nz) the periodic z basis and derivative at
# the z quadrature nodes, ``wz`` (nzq) and ``w2`` (n2q) the weights.
# Quadrature fields are (n2q, nzq) arrays laid out like QField (v[q2*nzq+qz]).


def sample(S, c, B):
    """hill_sample / hill_grad (hill3d.h:245-285): (S c) B^T."""
    return (S @ c) @ B.T


def load(S, w2, B, wz, fq):
    """hill_load / hill_load_grad (hill3d.h:288-312): S^T diag(w2) fq diag(wz) B."""
    return S.T @ (w2[:, None] * (fq @ (B * wz[:, None])))


def mass_solve(M2inv, Mzinv, b):
    """hill_mass_solve (hill3d.h:215-220): M2^-1 per z slice, then Mz^-1 per mode."""
    return (M2inv @ b) @ Mzinv.T


def skew_conv(m, wq, ui):
    """hill_skew_conv (hill3d.h:519-538): M^-1 0.5 [load(w.grad u) - sum_d load_grad_d(w_d u)]."""
    P, Dx, Dy = m["phi"], m["dpx"], m["dpy"]
    uq = sample(P, ui, m["Vz"])
    gx, gy, gz = sample(Dx, ui, m["Vz"]), sample(Dy, ui, m["Vz"]), sample(P, ui, m["dVz"])
    wx, wy, wzq = wq
    conv = wx * gx + wy * gy + wzq * gz
    adv = load(P, m["w2"], m["Vz"], m["wz"], conv)
    div = (load(Dx, m["w2"], m["Vz"], m["wz"], wx * uq) + load(Dy, m["w2"], m["Vz"], m["wz"], wy * uq)
           + load(P, m["w2"], m["dVz"], m["wz"], wzq * uq))
    return mass_solve(m["M2inv"], m["Mzinv"], 0.5 * (adv - div))


def advect(m, u):
    wq = [sample(m["phi"], c, m["Vz"]) for c in u]
    return [-skew_conv(m, wq, c) for c in u]


def fast_step(m, fd, u, dt, fx):
    """hill_fastdiag_step (hill_fastdiag.h:83-95): SSP-RK3 skew advection,
    + dt fx on u_x, then the fast-diagonalisation solve.  ``fd`` holds
    M2, Qx2, Qy2, mu, kap, Ainv, Sinv."""
    def stage(v, L):
        return [a + dt * b for a, b in zip(v, L)]

    u1 = stage(u, advect(m, u))
    t = stage(u1, advect(m, u1))
    u2 = [0.75 * a + 0.25 * b for a, b in zip(u, t)]
    t = stage(u2, advect(m, u2))
    us = [(1.0 / 3.0) * a + (2.0 / 3.0) * b for a, b in zip(u, t)]
    if fx != 0.0:
        us[0] = us[0] + dt * fx
    return solve(fd["M2"], fd["Qx2"], fd["Qy2"], fd["mu"], fd["kap"], fd["Ainv"], fd["Sinv"], *us)


def read_reference_dump(path):
    """Parse the binary written by oracle/_ref/hill_ref (hill_ref_main.cpp)."""
    import scipy.sparse as sp

    raw = np.fromfile(path, dtype=np.float64)
    nr, nz, a, steps = int(raw[0]), int(raw[1]), raw[2], int(raw[3])
    k = 4

    def take(n):
        nonlocal k
        v = raw[k : k + n]
        k += n
        return v

    d = {"nr": nr, "nz": nz, "a": a}
    for name in ("M2", "Qx2", "Qy2", "KN2"):
        d[name] = take(nr * nr).reshape(nr, nr)
    zr = take(3 * nz)
    d["Mz_row"], d["Sz_row"], d["Kz_row"] = zr[:nz], zr[nz : 2 * nz], zr[2 * nz :]
    for name in ("mu", "sig", "kap"):
        d[name] = take(nz)
    for name in ("ux", "uy", "uz", "ox", "oy", "oz"):
        d[name] = take(nr * nz).reshape(nr, nz)
    n2q, nzq = (int(v) for v in take(2))
    nnz = int(take(1)[0])
    ptr = take(n2q + 1).astype(np.int64)
    idx = take(nnz).astype(np.int64)
    for name in ("phi", "dpx", "dpy"):
        d[name] = sp.csr_matrix((take(nnz), idx, ptr), shape=(n2q, nr))
    d["w2"] = take(n2q)
    d["Vz"] = take(nzq * nz).reshape(nzq, nz)
    d["dVz"] = take(nzq * nz).reshape(nzq, nz)
    d["wz"] = take(nzq)
    d["M2inv"] = take(nr * nr).reshape(nr, nr)
    d["Mzinv"] = take(nz * nz).reshape(nz, nz)
    for name in ("cx", "cy", "cz"):
        d[name] = take(nr * nz).reshape(nr, nz)
    if steps:
        for name in ("sx", "sy", "sz"):
            d[name] = take(nr * nz).reshape(nr, nz)
    assert k == raw.size, (k, raw.size)
    d["n2q"], d["nzq"] = n2q, nzq
    return d


def reference_dump(ne=3, nz=6, seed=99, steps=1, ref_root=None, physical=False):
    """Run the compiled reference (oracle/_ref/hill_ref; built from the
    reference's headers when the tree is present) and parse its dump.
    Returns None when the binary is unavailable."""
    import subprocess
    import tempfile
    from pathlib import Path

    exe = Path(__file__).resolve().parent / "_ref" / "hill_ref"
    if not exe.exists():
        from .build_ref import build

        try:
            build(ref_root)
        except Exception:
            return None
    if not exe.exists():
        return None
    with tempfile.TemporaryDirectory() as td:
        out = Path(td) / "h.bin"
        subprocess.run([str(exe), str(ne), str(nz), str(seed), str(out), str(steps), str(int(physical))],
                       check=True, capture_output=True)
        return read_reference_dump(out)
