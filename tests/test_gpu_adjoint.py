"""Fixed-strategy evaluation and its adjoint against FP64 central differences.

With the average strategy frozen, the root cfvalues are linear in the
opponent's weights and in the boundary values, so the loss
L = g0 . cfv0 + g1 . cfv1 has exact central differences.  The FP64 oracle
(seeded with the GPU game's cumulative strategy) evaluates L at perturbed
inputs; the step actually taken is recovered from the f32 inputs the oracle
reads, so the only error left is the GPU's f32 arithmetic.  Tolerance: 1e-4
of the largest gradient entry in each block (weights of one player, boundary
values of one player).
"""

import numpy as np
import pytest
import torch

import poker_solver_rust_b200 as ps
from poker_solver_rust_b200.autograd import fixed_strategy_values
from tests import spots

pytestmark = pytest.mark.gpu

TOL_GRAD = 1e-4  # relative to the largest |gradient| of the block
H_STEP = 1e-3


def _copy_strategy(g, o):
    for i in range(g.num_nodes()):
        info = g.node_info(i)
        if not info["player"] & (4 | 8):
            o.seed_node_storage(i, 1, g.node_storage(i, 1))


def _setup(kind, iters=30, seed=5):
    rng = np.random.default_rng(seed)
    if kind == "boundary":
        r, b, t = spots.turn_spot(9, weights=_sparse)
        t.depth_limit = 0
    else:
        r, b, t = spots.river_spot(4)
    g = spots.product_game(r, b, t)
    o = spots.oracle_game(r, b, t, fp64=True)
    B = []
    for k in range(g.num_boundary_nodes()):
        row = []
        for p in range(2):
            v = rng.normal(0, 1, g.num_private_hands(p)).astype(np.float32)
            g.set_boundary_cfvs(k, p, v)
            o.set_boundary_cfvs(k, p, v)
            row.append(v)
        B.append(row)
    for it in range(iters):
        ps.solve_step(g, it)
    _copy_strategy(g, o)
    H = [g.num_private_hands(0), g.num_private_hands(1)]
    w = [rng.random(H[p]).astype(np.float32) for p in range(2)]
    cot = [rng.normal(0, 1, H[p]).astype(np.float32) for p in range(2)]
    return g, o, B, w, cot, rng


def _sparse(rng, board):
    out = []
    for _ in range(2):
        w = rng.random(1326).astype(np.float32)
        w[rng.random(1326) < 0.9] = 0.0
        out.append(spots._mask_board(w, board))
    return out


def _loss64(o, w, cot):
    c0 = o.root_cfvalues_with_reach(0, w[1])
    c1 = o.root_cfvalues_with_reach(1, w[0])
    return float(np.dot(cot[0].astype(np.float64), c0) + np.dot(cot[1].astype(np.float64), c1))


def _fd_weight(o, w, cot, p, j):
    wp, wm = [x.copy() for x in w], [x.copy() for x in w]
    wp[p][j] = np.float32(w[p][j] + H_STEP)
    wm[p][j] = np.float32(w[p][j] - H_STEP)
    step = float(wp[p][j]) - float(wm[p][j])
    return (_loss64(o, wp, cot) - _loss64(o, wm, cot)) / step


def _fd_boundary(o, B, w, cot, k, p, j):
    def at(x):
        v = B[k][p].copy()
        v[j] = x
        o.set_boundary_cfvs(k, p, v)
        return _loss64(o, w, cot), float(np.float32(x))

    lp, xp = at(np.float32(B[k][p][j] + H_STEP))
    lm, xm = at(np.float32(B[k][p][j] - H_STEP))
    o.set_boundary_cfvs(k, p, B[k][p])
    return (lp - lm) / (xp - xm)


def _check_block(got, ref, name):
    got, ref = np.asarray(got, np.float64), np.asarray(ref, np.float64)
    scale = max(np.abs(ref).max(), 1e-30)
    err = np.abs(got - ref).max() / scale
    assert err <= TOL_GRAD, (name, err)
    return err


@pytest.mark.parametrize("kind", ["river", "boundary"])
def test_adjoint_matches_fp64_central_differences(kind):
    g, o, B, w, cot, rng = _setup(kind)
    cfv0, cfv1 = ps.eval_fixed_strategy(g, w[0], w[1])
    # forward is the root-cfvalue sweep with the given weights
    assert np.array_equal(cfv0, ps.root_cfvalues_with_reach(g, 0, w[1]))
    assert np.array_equal(cfv1, ps.root_cfvalues_with_reach(g, 1, w[0]))
    ref0 = o.root_cfvalues_with_reach(0, w[1])
    assert np.abs(cfv0 - ref0).max() <= 1e-5 * np.abs(ref0).max()
    dw0, dw1, db = ps.eval_fixed_strategy_adjoint(g, w[0], w[1], cot[0], cot[1])
    if kind == "river":  # unraked river: zero-sum, so the adjoint is minus the other sweep
        neg = -ps.root_cfvalues_with_reach(g, 0, cot[1])
        assert np.abs(dw0 - neg).max() <= 1e-5 * np.abs(neg).max()
    for p, dw in ((0, dw0), (1, dw1)):
        idx = rng.choice(len(w[p]), size=min(24, len(w[p])), replace=False)
        fd = [_fd_weight(o, w, cot, p, j) for j in idx]
        _check_block(dw[idx], fd, f"dw{p}")
    if kind == "boundary":
        assert g.num_boundary_nodes() > 0
        for p in range(2):
            picks = [(int(rng.integers(g.num_boundary_nodes())), int(rng.integers(len(w[p])))) for _ in range(24)]
            got = [db[k][p][j] for k, j in picks]
            fd = [_fd_boundary(o, B, w, cot, k, p, j) for k, j in picks]
            _check_block(got, fd, f"dB{p}")


def test_autograd_value_gradient_cross_checks_cfvalues():
    """V = w0 . cfv0 + w1 . cfv1: dV/dw0 = cfv0 + (adjoint through cfv1) and
    the boundary gradient reaches the boundary tensors; both against FD."""
    g, o, B, w, cot, rng = _setup("boundary", seed=8)
    nb = g.num_boundary_nodes()
    w0 = torch.tensor(w[0], dtype=torch.float64, requires_grad=True)
    w1 = torch.tensor(w[1], dtype=torch.float64, requires_grad=True)
    b0 = torch.tensor(np.stack([B[k][0] for k in range(nb)]), dtype=torch.float64, requires_grad=True)
    b1 = torch.tensor(np.stack([B[k][1] for k in range(nb)]), dtype=torch.float64, requires_grad=True)
    c0, c1 = fixed_strategy_values(g, w0, w1, b0, b1)
    V = (w0 * c0).sum() + (w1 * c1).sum()
    V.backward()
    # FD of V: cotangents are the weights themselves, plus the own-weight term
    c0_ref = o.root_cfvalues_with_reach(0, w[1])
    c1_ref = o.root_cfvalues_with_reach(1, w[0])
    for p in range(2):
        idx = rng.choice(len(w[p]), size=16, replace=False)
        grad = (w0 if p == 0 else w1).grad.numpy()[idx]
        own = (c0_ref if p == 0 else c1_ref)[idx]
        cross = [_fd_weight(o, w, [w[0], w[1]], p, j) for j in idx]
        # _fd_weight differentiates only the opponent's cfv term; add the own term
        fd = np.asarray(cross) + own
        _check_block(grad, fd, f"dV/dw{p}")
    picks = [(int(rng.integers(nb)), int(rng.integers(len(w[0])))) for _ in range(12)]
    fd = [_fd_boundary(o, B, w, [w[0], w[1]], k, 0, j) for k, j in picks]
    _check_block([b0.grad[k, j].item() for k, j in picks], fd, "dV/dB0")


def test_autograd_cuda_tensors_stay_on_the_device(monkeypatch):
    """CUDA tensors go through the device-pointer entry points: forward and
    backward run with every route to host memory of a tensor disabled, and
    give the same bits as the host-memory path."""
    g, o, B, w, cot, rng = _setup("boundary", seed=12)
    nb = g.num_boundary_nodes()

    def inputs(dev):
        w0 = torch.tensor(w[0], dtype=torch.float64, device=dev, requires_grad=True)
        w1 = torch.tensor(w[1], dtype=torch.float64, device=dev, requires_grad=True)
        b0 = torch.tensor(np.stack([B[k][0] for k in range(nb)]), dtype=torch.float64, device=dev,
                          requires_grad=True)
        b1 = torch.tensor(np.stack([B[k][1] for k in range(nb)]), dtype=torch.float64, device=dev,
                          requires_grad=True)
        return w0, w1, b0, b1

    def run(dev):
        t = inputs(dev)
        c0, c1 = fixed_strategy_values(g, *t)
        loss = (c0 * torch.tensor(cot[0], dtype=torch.float64, device=dev)).sum() + \
               (c1 * torch.tensor(cot[1], dtype=torch.float64, device=dev)).sum()
        loss.backward()
        return [c0.detach(), c1.detach()] + [x.grad for x in t]

    host = [x.numpy() for x in run("cpu")]

    def no_host(*a, **k):
        raise AssertionError("a CUDA tensor was copied to the host")

    with monkeypatch.context() as m:
        m.setattr(torch.Tensor, "cpu", no_host)
        m.setattr(torch.Tensor, "numpy", no_host)
        dev = run("cuda")
        torch.cuda.synchronize()
    for a, b in zip(dev, host):
        assert np.array_equal(a.to("cpu").numpy(), b)
