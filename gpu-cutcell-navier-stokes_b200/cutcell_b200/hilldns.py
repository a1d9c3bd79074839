"""Periodic-hill DNS loop on the device: the time loop of the reference's
GPU DNS driver (cpp/gpu/gpu_dns.cu:150-250) around the device fast step.

* ``HillDNS.step`` is one ``hill_fastdiag_step`` on the device (SSP-RK3 skew
  advection, body force on u_x, fast-diagonalisation solve).
* The body force is constant, or PI-controlled to hold a target bulk
  velocity (fixed Reynolds number): with e = U_target - U_b,
  integ += e dt, fx = Kp e + Ki integ, Kp = 4, Ki = 3 (gpu_dns.cu:198,235-236).
  U_b = (1/V) int u_x dV is a weighted dot product on the device
  (gpu_dns.cu:121-124): V the fluid volume, the weights a = PHI^T w2 (x-y)
  and c = Vz^T wz (z) folded once, U_b = a^T u_x c / V.
* ``StationStats``: online first and second moments at the ten reference
  stations x/H in {0.05, 0.5, 1, ..., 8}, 64 y nodes each from the wall to
  the top, z-averaged over the spanwise quadrature (stats_hill.h), their
  binary accumulator record and the hillturb_stats JSON they are written as.
* Checkpoints keep the reference's binary layout (gpu_dns.cu:128-146), so a
  run can resume from either program's file: int32 step, float64 fx,
  float64 integ, int32 NC = nr * nz, then u_x, u_y, u_z (FieldH order
  v[m * nz + iz], NC float64 each), then the statistics record (int64 n,
  then su, sv, sw, suu, svv, sww, suv, each NS x NY float64); written to
  ``path.tmp`` and renamed.
"""

from __future__ import annotations

import json
import os
import struct

import numpy as np

from .hillsetup import HillSetup, sample_rows, weak_div

KP, KI = 4.0, 3.0


class StationStats:
    NS, NY = 10, 64
    X_H = (0.05, 0.5, 1.0, 2.0, 3.0, 4.0, 5.0, 6.0, 7.0, 8.0)

    def __init__(self, hs: HillSetup, eps: float = 1e-4):
        wall = hs.wall
        Lx, Ly = wall.Lx, wall.Ly
        xs, ys = [], []
        self.yphys = np.zeros((self.NS, self.NY))
        for i, xh in enumerate(self.X_H):
            hw = float(wall.h(xh))
            yj = (hw + eps) + ((Ly - eps) - (hw + eps)) * np.arange(self.NY) / (self.NY - 1)
            self.yphys[i] = yj
            xs.append(np.full(self.NY, xh / Lx))
            ys.append(yj / Ly)
        # reduced sample rows at every (station, y) point: (NS * NY, nr)
        self.S, _, _ = sample_rows(hs.forms.basis, hs.E, np.concatenate(xs), np.concatenate(ys))
        self.Vz, self.wz, self.Lz = hs.Vz, hs.wz, hs.Lz
        self.acc = {k: np.zeros((self.NS, self.NY)) for k in ("su", "sv", "sw", "suu", "svv", "sww", "suv")}
        self.n = 0

    def accumulate(self, ux, uy, uz) -> None:
        """Add one sample of host FieldH arrays (nr, nz)."""
        q = [(self.S @ u) @ self.Vz.T for u in (ux, uy, uz)]  # (NS*NY, nzq)
        w = self.wz / self.Lz
        U, V, W = (x @ w for x in q)
        sh = (self.NS, self.NY)
        self.acc["su"] += U.reshape(sh)
        self.acc["sv"] += V.reshape(sh)
        self.acc["sw"] += W.reshape(sh)
        self.acc["suu"] += ((q[0] * q[0]) @ w).reshape(sh)
        self.acc["svv"] += ((q[1] * q[1]) @ w).reshape(sh)
        self.acc["sww"] += ((q[2] * q[2]) @ w).reshape(sh)
        self.acc["suv"] += ((q[0] * q[1]) @ w).reshape(sh)
        self.n += 1

    def save(self, f) -> None:
        f.write(struct.pack("<q", self.n))
        for k in ("su", "sv", "sw", "suu", "svv", "sww", "suv"):
            f.write(np.ascontiguousarray(self.acc[k], dtype="<f8").tobytes())

    def load(self, f) -> None:
        raw = f.read(8)
        if len(raw) < 8:
            return
        self.n = struct.unpack("<q", raw)[0]
        for k in ("su", "sv", "sw", "suu", "svv", "sww", "suv"):
            self.acc[k] = np.frombuffer(f.read(8 * self.NS * self.NY), dtype="<f8").reshape(self.NS, self.NY).copy()

    def profiles(self, u_b: float) -> list:
        """Per station: y, U, V, W (by u_b) and the Reynolds stresses uu, vv,
        ww, uv (by u_b^2), with uu = max(<u u> - U^2, 0)."""
        n = max(self.n, 1)
        ub = u_b if u_b != 0.0 else 1.0
        a = {k: v / n for k, v in self.acc.items()}
        U, V, W = a["su"], a["sv"], a["sw"]
        out = []
        for i, xh in enumerate(self.X_H):
            out.append({
                "x_over_H": xh, "y": self.yphys[i].tolist(),
                "U": (U[i] / ub).tolist(), "V": (V[i] / ub).tolist(), "W": (W[i] / ub).tolist(),
                "uu": (np.maximum(a["suu"][i] - U[i] ** 2, 0.0) / ub**2).tolist(),
                "vv": (np.maximum(a["svv"][i] - V[i] ** 2, 0.0) / ub**2).tolist(),
                "ww": (np.maximum(a["sww"][i] - W[i] ** 2, 0.0) / ub**2).tolist(),
                "uv": ((a["suv"][i] - U[i] * V[i]) / ub**2).tolist(),
            })
        return out

    def write_json(self, path: str, hs: HillSetup, u_b: float, reynolds: int, step: int, sim_time: float,
                   dt: float, u_tau: float = 0.0) -> None:
        doc = {
            "status": "gpu_dns",
            "meta": {"reynolds": reynolds, "nu": (u_b / reynolds if reynolds > 0 else 0.0), "p": hs.p, "nx": hs.nex,
                     "ny": hs.ney, "Lz": hs.Lz, "Nz": hs.nz, "n_modes": hs.nz, "dt": dt, "target_bulk": u_b,
                     "dns_source": "cutcell_b200"},
            "averaging_window": {"n_samples": self.n, "step": step, "sim_time": sim_time, "eddy_turnover_time": 9.0,
                                 "under_averaged": self.n < 200},
            "running_means": {"u_tau": u_tau, "bulk_velocity": u_b, "reynolds": float(reynolds)},
            "stations": self.profiles(u_b),
            "wall": {"x_over_H": [], "cf": [], "cp": [], "reattachment_x_over_H": None},
        }
        with open(path, "w") as f:
            json.dump(doc, f, indent=1)


class HillDNS:
    """Device DNS of the periodic-hill channel described by ``hs`` (physical
    metric): state on the device, body force constant or PI-controlled."""

    def __init__(self, hs: HillSetup, *, nu: float = 1.0 / 5600.0, dt: float = 0.02, fx0: float = 0.0,
                 target_ub: float = 0.0, device="cuda", stats: bool = False):
        import torch

        from .hill import FastDiagHill, HillAdvection

        self.hs, self.nu, self.dt = hs, float(nu), float(dt)
        self.fx, self.integ = float(fx0), 0.0
        self.target_ub = float(target_ub)
        self.device = torch.device(device)
        m = hs.machinery()
        self.adv = HillAdvection(m["phi"], m["dpx"], m["dpy"], m["w2"], m["Vz"], m["dVz"], m["wz"], m["M2inv"],
                                 m["Mzinv"], device=self.device)
        self.fd = FastDiagHill(device=self.device).build(hs.M2, hs.Qx2, hs.Qy2, hs.KN2, hs.Mz[0], hs.Sz[0], hs.Kz[0],
                                                         self.dt * self.nu, on_device=True)
        f64 = torch.float64
        self.a_w = torch.as_tensor(np.asarray(hs.phi.T @ hs.w2), dtype=f64, device=self.device)
        self.c_w = torch.as_tensor(hs.Vz.T @ hs.wz, dtype=f64, device=self.device)
        self.volume = float(hs.w2.sum() * hs.wz.sum())
        self.M2 = torch.as_tensor(hs.M2, dtype=f64, device=self.device)
        self.Mz = torch.as_tensor(hs.Mz, dtype=f64, device=self.device)
        self.u = None
        self.step_count = 0
        self.stats = StationStats(hs) if stats else None

    def set_state(self, ux, uy, uz) -> None:
        import torch

        self.u = [torch.as_tensor(np.ascontiguousarray(c), dtype=torch.float64).to(self.device).contiguous()
                  for c in (ux, uy, uz)]

    def host_state(self):
        return [c.cpu().numpy() for c in self.u]

    def bulk_velocity(self) -> float:
        """U_b = (1/V) int u_x dV (gpu_dns.cu:121-124)."""
        return float(self.a_w @ self.u[0] @ self.c_w) / self.volume

    def kinetic_energy(self) -> float:
        """hill_ke (hill3d.h:497-501): (1/2) sum_c u_c . (M2 (x) Mz) u_c."""
        return 0.5 * float(sum((c * (self.M2 @ c @ self.Mz.T)).sum() for c in self.u))

    def max_weak_div(self) -> float:
        return float(np.abs(weak_div(self.hs, *self.host_state())).max())

    def step(self) -> None:
        """Controller update from the current bulk velocity, then one fast step."""
        if self.target_ub > 0.0:
            e = self.target_ub - self.bulk_velocity()
            self.integ += e * self.dt
            self.fx = KP * e + KI * self.integ
        self.adv.step(self.fd, self.u, self.dt, self.fx)
        self.step_count += 1

    def accumulate_stats(self) -> None:
        if self.stats is not None:
            self.stats.accumulate(*self.host_state())

    # -- checkpoints (gpu_dns.cu:128-146 layout) ---------------------------
    def save_checkpoint(self, path: str) -> None:
        ux, uy, uz = self.host_state()
        nc = ux.size
        tmp = path + ".tmp"
        with open(tmp, "wb") as f:
            f.write(struct.pack("<i", self.step_count))
            f.write(struct.pack("<d", self.fx))
            f.write(struct.pack("<d", self.integ))
            f.write(struct.pack("<i", nc))
            for c in (ux, uy, uz):
                f.write(np.ascontiguousarray(c, dtype="<f8").tobytes())
            if self.stats is not None:
                self.stats.save(f)
            else:  # an unbuilt statistics record: its sample count only
                f.write(struct.pack("<q", 0))
        os.replace(tmp, path)

    def load_checkpoint(self, path: str) -> bool:
        """Resume field, controller and statistics; False if the file is
        absent or its field size differs (the reference's behaviour)."""
        if not os.path.exists(path):
            return False
        with open(path, "rb") as f:
            step = struct.unpack("<i", f.read(4))[0]
            fx = struct.unpack("<d", f.read(8))[0]
            integ = struct.unpack("<d", f.read(8))[0]
            nc = struct.unpack("<i", f.read(4))[0]
            if nc != self.hs.nr * self.hs.nz:
                return False
            shape = (self.hs.nr, self.hs.nz)
            comps = [np.frombuffer(f.read(8 * nc), dtype="<f8").reshape(shape) for _ in range(3)]
            if self.stats is not None:
                self.stats.load(f)
        self.step_count, self.fx, self.integ = step, fx, integ
        self.set_state(*comps)
        return True

    def close(self) -> None:
        self.adv.close()
        self.fd.close()
