"""Host side of the periodic-hill DNS loop (cutcell_b200.hilldns):

* the station statistics (stats_hill.h) equal a direct evaluation of the
  field at the station points (x-y basis through E, periodic z basis at the
  spanwise quadrature), z-averaged with the quadrature weights;
* the statistics record and the checkpoint keep the reference's binary
  layout (cpp/gpu/gpu_dns.cu:128-146): int32 step, float64 fx, float64
  integ, int32 NC, three NC-blocks, then int64 n and seven NS x NY blocks."""

import struct

import numpy as np

from cutcell_b200.hilldns import HillDNS, StationStats
from cutcell_b200.hillsetup import build_hill


def _setup():
    return build_hill(8, 4, 3, 8, 4.5, physical=True)


def test_station_moments_match_direct_evaluation():
    hs = _setup()
    st = StationStats(hs)
    rng = np.random.default_rng(1)
    u = [rng.standard_normal((hs.nr, hs.nz)) for _ in range(3)]
    st.accumulate(*u)
    B = hs.forms.basis
    for i in (0, 4, 9):
        for j in (0, 31, 63):
            x = st.X_H[i] / hs.wall.Lx
            y = st.yphys[i, j] / hs.wall.Ly
            rows, phi, _, _ = B.local(np.array([x]), np.array([y]))
            red = phi[0] @ hs.E[rows[0]]  # reduced basis values at the point
            vals = [(red @ c) @ hs.Vz.T for c in u]  # (nzq,)
            w = hs.wz / hs.Lz
            assert abs(st.acc["su"][i, j] - vals[0] @ w) <= 1e-12 * (1 + abs(vals[0] @ w))
            assert abs(st.acc["suv"][i, j] - (vals[0] * vals[1]) @ w) <= 1e-12 * (1 + np.abs(vals[0] * vals[1]).max())


def test_checkpoint_layout_round_trip(tmp_path):
    hs = _setup()

    class HostTensor:  # stands in for a device tensor in the checkpoint writer
        def __init__(self, a):
            self.a = a

        def cpu(self):
            return self

        def numpy(self):
            return self.a

    dns = HillDNS.__new__(HillDNS)
    dns.hs = hs
    rng = np.random.default_rng(2)
    state = [rng.standard_normal((hs.nr, hs.nz)) for _ in range(3)]
    dns.u = [HostTensor(a) for a in state]
    dns.step_count, dns.fx, dns.integ = 17, 0.125, -0.5
    dns.stats = StationStats(hs)
    dns.stats.accumulate(*state)
    path = str(tmp_path / "ck.bin")
    dns.save_checkpoint(path)
    raw = open(path, "rb").read()
    nc = hs.nr * hs.nz
    step, fx, integ, nc2 = struct.unpack_from("<iddi", raw, 0)
    assert (step, fx, integ, nc2) == (17, 0.125, -0.5, nc)
    off = struct.calcsize("<iddi")
    for c in state:
        np.testing.assert_array_equal(np.frombuffer(raw, dtype="<f8", count=nc, offset=off).reshape(c.shape), c)
        off += 8 * nc
    (n,) = struct.unpack_from("<q", raw, off)
    assert n == 1
    assert len(raw) == off + 8 + 7 * StationStats.NS * StationStats.NY * 8
    # read back into a fresh statistics record
    st2 = StationStats(hs)
    with open(path, "rb") as f:
        f.seek(off)
        st2.load(f)
    for k in st2.acc:
        np.testing.assert_array_equal(st2.acc[k], dns.stats.acc[k])
