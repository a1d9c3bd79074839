"""Learned preconditioner: device forward/backward/Adam against the CPU
oracle, and the flexible PCG that uses the trained network (needs a B200)."""

import numpy as np
import pytest
import scipy.sparse.linalg as spla

from oracle import mlp as om

from _systems import system

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch


def test_mlp_forward_and_gradients_match_oracle(torch_cuda):
    from cutcell_b200.learned import PatchMLP, init_params, split_params

    rng = np.random.default_rng(3)
    theta = init_params(5)
    theta[-64:] = rng.standard_normal(64).astype(np.float32) * 0.1  # nonzero output bias
    theta[(128 * 64 + 64 + 64 * 64 + 64):(128 * 64 + 64 + 64 * 64 + 64) + 64 * 64] *= 100.0  # make W3 visible
    X = rng.standard_normal((300, 128)).astype(np.float32)
    T = rng.standard_normal((300, 64)).astype(np.float32)
    net = PatchMLP(theta)
    Xd = torch_cuda.as_tensor(X).cuda()
    Td = torch_cuda.as_tensor(T).cuda()
    Y = net.forward(Xd).cpu().numpy()
    W, b = split_params(theta)
    Yo, _ = om.forward(X.astype(np.float64), W, [bb.astype(np.float64) for bb in b])
    assert np.abs(Y - Yo).max() <= 1e-4 * np.abs(Yo).max()
    loss = float(net.train_step(Xd, Td, 0.0).item())
    g = net.last_grad()
    lo, gW, gb = om.loss_and_grads(X.astype(np.float64), T.astype(np.float64), W, [bb.astype(np.float64) for bb in b])
    assert abs(loss - lo) <= 1e-5 * lo
    go = np.concatenate([gW[0].ravel(), gb[0], gW[1].ravel(), gb[1], gW[2].ravel(), gb[2]])
    assert np.linalg.norm(g - go) <= 1e-4 * np.linalg.norm(go)
    # one Adam step against the oracle's update with the device gradient
    net.train_step(Xd, Td, 1e-3)
    th1 = net.params()
    m = [np.zeros_like(p) for p in (theta,)]
    v = [np.zeros_like(p) for p in (theta,)]
    ref = om.adam_step([theta.astype(np.float64)], [net.last_grad().astype(np.float64)], m, v, 1, 1e-3)[0]
    assert np.abs(th1 - ref).max() <= 1e-6 + 1e-5 * np.abs(ref).max()
    net.close()


def test_patch_layout_covers_reduced_dofs_once(torch_cuda):
    from cutcell_b200.learned import patch_layout
    from cutcell_b200.operator import CutCellOperator

    prob, ext, A_full, A_red, b = system("sphere", 9, 3)
    op = CutCellOperator(prob, ext)
    lay = patch_layout(op)
    r = lay.red[lay.red >= 0]
    assert np.array_equal(np.sort(r), np.arange(ext.n_red))
    op.close()


def test_learned_fcg_converges_to_fp64_solution(torch_cuda):
    from cutcell_b200 import solve_spd
    from cutcell_b200.learned import PatchMLP, attach, generate_pairs, train
    from cutcell_b200.operator import CutCellOperator

    prob, ext, A_full, A_red, b = system("sphere", 9, 3)
    op = CutCellOperator(prob, ext)
    net = PatchMLP(seed=1)
    X, T = generate_pairs([op], 3000, seed=7)
    hist = train(net, X, T, epochs=8, batch=256, lr=2e-3)
    assert hist[-1] < hist[0]  # the network learns something
    attach(op, net)
    x, rep = solve_spd(op, b, tol=1e-9, maxiter=5000, preconditioner="jacobi+learned")
    assert rep.success, rep
    assert rep.relative_residual <= 1e-9
    xd = spla.spsolve(A_red.tocsc(), b)
    xp, rep_plain = solve_spd(op, b, tol=1e-9, maxiter=5000)
    # the same relative residual as plain FP64 Jacobi-PCG; the error against
    # the direct solution stays at the level the plain solve reaches
    err = np.linalg.norm(x - xd) / np.linalg.norm(xd)
    err_plain = np.linalg.norm(xp - xd) / np.linalg.norm(xd)
    assert err <= max(10 * err_plain, 1e-7), (err, err_plain)
    print(f"learned FCG iterations {rep.iterations} vs plain {rep_plain.iterations}; err {err:.2e} plain {err_plain:.2e}")
    op.close()
    net.close()
