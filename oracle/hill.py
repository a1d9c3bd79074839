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
