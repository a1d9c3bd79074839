"""The device hill step against the reference's own implementations on the
same box, on identical machinery (the restated build equals the reference's
Hill3D::build at nex = ney, tests/test_hill_setup_host.py):

* the reference's GPU step (cpp/gpu/gpu_run.cu, its kernels plus cuBLAS,
  compiled by oracle/build_ref.py into oracle/_ref/gpu_run) at ne = 16,
  nz = 2 ne = 32, physical metric, a = 0.01, dt = 0.02, fx = 2;
* this package's device step on the same configuration.
Prints both times and asserts the device step is faster than the
reference's GPU step.  Skips where the reference binary is absent."""

import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REF = Path(__file__).resolve().parents[1] / "oracle" / "_ref"


def test_device_step_beats_reference_gpu_step():
    import torch

    from cutcell_b200.hill import FastDiagHill, HillAdvection
    from cutcell_b200.hillsetup import build_hill

    exe = REF / "gpu_run"
    if not exe.exists():
        pytest.skip("reference GPU binary unavailable")
    out = subprocess.run([str(exe), "16", "12", "0"], capture_output=True, text=True, timeout=600)
    m = re.search(r"GPU ([0-9.]+) ms/step", out.stdout)
    assert m, out.stdout + out.stderr
    ref_ms = float(m.group(1))
    hs = build_hill(16, 16, 3, 32, 4.5, physical=True)
    mach = hs.machinery()
    adv = HillAdvection(mach["phi"], mach["dpx"], mach["dpy"], mach["w2"], mach["Vz"], mach["dVz"], mach["wz"],
                        mach["M2inv"], mach["Mzinv"])
    fd = FastDiagHill().build(hs.M2, hs.Qx2, hs.Qy2, hs.KN2, hs.Mz[0], hs.Sz[0], hs.Kz[0], 0.01, on_device=True)
    rng = np.random.default_rng(20260629)
    u = [torch.as_tensor(0.01 * rng.uniform(-0.5, 0.5, (hs.nr, hs.nz))).cuda() for _ in range(3)]
    adv.step(fd, u, 0.02, 2.0)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(11):
        adv.step(fd, u, 0.02, 2.0)
    e1.record()
    torch.cuda.synchronize()
    ours_ms = e0.elapsed_time(e1) / 11
    print(f"hill ne=16 nz=32 (nr={hs.nr}): device step {ours_ms:.3f} ms, reference GPU step {ref_ms:.2f} ms")
    assert np.all([torch.isfinite(c).all().item() for c in u])
    assert ours_ms < ref_ms
    adv.close()
    fd.close()
