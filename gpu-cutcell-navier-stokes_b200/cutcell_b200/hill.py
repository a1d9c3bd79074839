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


class FastDiagHill:
    def __init__(self, device="cuda"):
        import torch

        self.device = torch.device(device)
        self._lib = _lib.load()
        self._ctx = None

    def build(self, M2, Qx2, Qy2, KN2, Mz_row, Sz_row, Kz_row, a, *, inverses=None):
        """Host build (FastDiagHill::build); ``inverses=(Ainv, Sinv)`` may be
        supplied (host or device arrays) instead of being formed here."""
        import torch

        self.nr = int(M2.shape[0])
        self.nz = int(len(Mz_row))
        self.a = float(a)
        self.mu, self.sig, self.kap = z_symbols(Mz_row, Sz_row, Kz_row)
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
