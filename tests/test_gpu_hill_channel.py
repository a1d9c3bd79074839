"""The periodic-hill channel built here (anisotropic Hill3D::build
restatement, cutcell_b200.hillsetup) stepped on the device.

* cutcell_dgemm_nt (FP64 tensor-core batched GEMM with a diagonal scale)
  against NumPy to 1e-13 relative, ragged sizes and shared operands included;
* the per-mode operators built through the shared generalised eigenbasis on
  the device (mode_operators_gpu) against the host's dense inversions of
  FastDiagHill::build (hill_fastdiag.h:26-43) to 1e-8 relative;
* one fast step (SSP-RK3 skew advection + fast-diagonalisation solve) of the
  parabolic initial condition on an anisotropic 16 x 8 x 8 channel against
  the oracle's step (oracle/hill.py) to 1e-9, and its weak divergence within
  10x of the oracle step's (the same algorithm on the host);
* the channel configuration itself, 64 x 32 elements, nz = 32, p = 3, built
  and stepped on the device: finite, and the weak divergence of the stepped
  velocity below 1e-10 of the initial condition's (reported)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch


def test_dgemm_nt_matches_numpy(torch_cuda):
    from cutcell_b200 import _lib
    from cutcell_b200.hill import _dgemm_nt

    torch = torch_cuda
    lib = _lib.load()
    rng = np.random.default_rng(3)
    for (M, N, K, batch, shareA, scale, beta) in [(70, 33, 19, 3, False, True, 0.0), (128, 64, 64, 1, False, False, 0.0),
                                                 (5, 130, 257, 2, True, True, 0.5), (200, 200, 3, 4, True, False, 0.0)]:
        A = rng.standard_normal((1 if shareA else batch, M, K))
        B = rng.standard_normal((batch, N, K))
        s = rng.standard_normal((batch, K)) if scale else None
        C0 = rng.standard_normal((batch, M, N))
        dv = lambda x: torch.as_tensor(x).cuda()
        Ad, Bd, Cd = dv(A), dv(B), dv(C0)
        sd = dv(s) if scale else None
        _dgemm_nt(lib, M, N, K, Ad, K, 0 if shareA else M * K, Bd, K, N * K, sd, K if scale else 0, Cd, N, M * N,
                  batch, beta=beta)
        got = Cd.cpu().numpy()
        for b in range(batch):
            Ab = A[0 if shareA else b] * (s[b][None, :] if scale else 1.0)
            ref = Ab @ B[b].T + beta * C0[b]
            assert np.abs(got[b] - ref).max() <= 1e-13 * np.abs(ref).max() * np.sqrt(K), (M, N, K, b)


def test_mode_operators_on_device_match_host_inversion(torch_cuda):
    from cutcell_b200.hill import mode_inverses, mode_operators_gpu, z_symbols
    from cutcell_b200.hillsetup import build_hill

    hs = build_hill(8, 4, 3, 8, 4.5, physical=True)
    mu, sig, kap = z_symbols(hs.Mz[0], hs.Sz[0], hs.Kz[0])
    a = 0.02 / 5600
    Ah, Sh = mode_inverses(hs.M2, hs.Qx2, hs.Qy2, hs.KN2, mu, sig, kap, a)
    Ad, Sd = mode_operators_gpu(hs.M2, hs.Qx2, hs.Qy2, hs.KN2, mu, sig, kap, a)
    Ad, Sd = Ad.cpu().numpy(), Sd.cpu().numpy()
    for k in range(len(mu)):
        assert np.abs(Ad[k] - Ah[k]).max() <= 1e-8 * np.abs(Ah[k]).max(), k
        assert np.abs(Sd[k] - Sh[k]).max() <= 1e-8 * np.abs(Sh[k]).max(), k


def _device_step(hs, u, dt, fx):
    import torch

    from cutcell_b200.hill import FastDiagHill, HillAdvection, z_symbols

    m = hs.machinery()
    adv = HillAdvection(m["phi"], m["dpx"], m["dpy"], m["w2"], m["Vz"], m["dVz"], m["wz"], m["M2inv"], m["Mzinv"])
    fd = FastDiagHill().build(hs.M2, hs.Qx2, hs.Qy2, hs.KN2, hs.Mz[0], hs.Sz[0], hs.Kz[0], dt / 5600, on_device=True)
    ud = [torch.as_tensor(np.ascontiguousarray(c)).cuda() for c in u]
    adv.step(fd, ud, dt, fx)
    out = [c.cpu().numpy() for c in ud]
    adv.close()
    fd.close()
    return out


def test_anisotropic_channel_step_matches_oracle(torch_cuda):
    from cutcell_b200.hill import mode_inverses, z_symbols
    from cutcell_b200.hillsetup import build_hill, parabolic_ic, weak_div
    from oracle import hill as oh

    hs = build_hill(16, 8, 3, 8, 4.5, physical=True)
    u0 = parabolic_ic(hs)
    dt, fx = 0.02, 0.7
    got = _device_step(hs, u0, dt, fx)
    mu, sig, kap = z_symbols(hs.Mz[0], hs.Sz[0], hs.Kz[0])
    Ai, Si = mode_inverses(hs.M2, hs.Qx2, hs.Qy2, hs.KN2, mu, sig, kap, dt / 5600)
    fd = dict(M2=hs.M2, Qx2=hs.Qx2, Qy2=hs.Qy2, mu=mu, kap=kap, Ainv=Ai, Sinv=Si)
    ref = oh.fast_step(hs.machinery(), fd, [c.copy() for c in u0], dt, fx)
    for g, r in zip(got, ref):
        assert np.abs(g - r).max() <= 1e-9 * np.abs(r).max()
    div_dev = np.abs(weak_div(hs, *got)).max()
    div_ref = np.abs(weak_div(hs, *ref)).max()
    print(f"16x8x8 channel: weak divergence device {div_dev:.2e}, oracle step {div_ref:.2e}, "
          f"initial {np.abs(weak_div(hs, *u0)).max():.2e}")
    assert div_dev <= 10 * max(div_ref, 1e-16)


def test_channel_configuration_builds_and_steps(torch_cuda):
    import time

    from cutcell_b200.hillsetup import build_hill, parabolic_ic, weak_div

    t0 = time.perf_counter()
    hs = build_hill(64, 32, 3, 32, 4.5, physical=True)
    u0 = parabolic_ic(hs)
    t_host = time.perf_counter() - t0
    got = _device_step(hs, u0, 0.02, 0.0)
    assert all(np.all(np.isfinite(g)) for g in got)
    d0 = np.abs(weak_div(hs, *u0)).max()
    d1 = np.abs(weak_div(hs, *got)).max()
    print(f"64x32x32 channel: nr={hs.nr} n2q={hs.n2q} host build {t_host:.1f}s, weak divergence {d0:.2e} -> {d1:.2e}, "
          f"max|u| {max(np.abs(g).max() for g in got):.3f}")
    assert d1 <= 1e-10 * d0


def test_dns_pi_control_and_checkpoint_resume(torch_cuda, tmp_path):
    """The DNS loop on the device (cutcell_b200.hilldns): with the PI flow
    controller (Kp = 4, Ki = 3, gpu_dns.cu:198,235-236) the bulk velocity of
    the 16 x 8 x 8 channel moves towards its target; a run checkpointed and
    resumed in a fresh driver continues bit for bit like the uninterrupted run."""
    from cutcell_b200.hilldns import HillDNS
    from cutcell_b200.hillsetup import build_hill, parabolic_ic

    hs = build_hill(16, 8, 3, 8, 4.5, physical=True)
    u0 = parabolic_ic(hs, ub=0.8)
    a = HillDNS(hs, target_ub=1.0, stats=True)
    a.set_state(*u0)
    ub0 = a.bulk_velocity()
    for k in range(6):
        a.step()
        if k % 2 == 1:
            a.accumulate_stats()
    ub6 = a.bulk_velocity()
    assert abs(ub6 - 1.0) < abs(ub0 - 1.0), (ub0, ub6)
    path = str(tmp_path / "ck.bin")
    a.save_checkpoint(path)
    for _ in range(3):
        a.step()
    ref = a.host_state()
    b = HillDNS(hs, target_ub=1.0, stats=True)
    assert b.load_checkpoint(path)
    assert b.stats.n == 3 and b.step_count == 6
    for _ in range(3):
        b.step()
    for x, y in zip(b.host_state(), ref):
        np.testing.assert_array_equal(x, y)
    print(f"DNS: bulk velocity {ub0:.4f} -> {ub6:.4f} (target 1), fx {a.fx:.4f}, "
          f"max weak div {a.max_weak_div():.2e}, KE {a.kinetic_energy():.4f}")
    a.close()
    b.close()
