"""Training through solved trees (poker_solver_rust_b200.trainer).

- RiverAverage: its hand-written backward against autograd of a plain f64
  torch form of the same average.
- solve_through_loss: the gradient that reaches the network's last layer
  (on which the loss is quadratic at a fixed strategy) against central
  differences of the same loss, with the solved strategy and the boundary
  reach held fixed.  Tolerance 1e-3 of the largest gradient checked: the
  values pass through the tree in f32.
"""

import numpy as np
import pytest
import torch

import poker_solver_rust_b200 as ps
from poker_solver_rust_b200 import trainer as T
from poker_solver_rust_b200.datagen import boundary_encode
from tests import spots

pytestmark = pytest.mark.gpu


def _plain_average(y, boards, scale, reach):
    keep = T.river_keep_mask(boards, y.device).to(torch.float64)
    opp = reach.flip(1).to(torch.float64)
    W = torch.einsum("npc,nrc->npr", opp, keep)
    num = torch.einsum("npr,nrc,nprc->npc", W, keep, y.to(torch.float64))
    den = torch.einsum("npr,nrc->npc", W, keep)
    s = torch.as_tensor(scale, dtype=torch.float64, device=y.device)[:, None, None]
    return torch.where(den > 0, num / den.clamp_min(1e-300) * s, torch.zeros_like(den))


def test_river_average_backward():
    rng = np.random.default_rng(9)
    n = 3
    boards = np.stack([rng.choice(52, 4, replace=False) for _ in range(n)]).astype(np.uint8)
    scale = rng.uniform(50, 300, n).astype(np.float32)
    reach = torch.tensor(rng.random((n, 2, 1326)).astype(np.float32), device="cuda")
    y = torch.tensor(rng.normal(0, 1, (n, 2, 48, 1326)).astype(np.float32), device="cuda", requires_grad=True)
    G = torch.tensor(rng.normal(0, 1, (n, 2, 1326)), device="cuda")
    out = T.RiverAverage.apply(y, boards, scale, reach)
    ref = _plain_average(y, boards, scale, reach)
    assert torch.allclose(out.double(), ref, rtol=1e-5, atol=1e-5 * ref.abs().max().item())
    (g1,) = torch.autograd.grad((out.double() * G).sum(), y)
    (g2,) = torch.autograd.grad((ref * G).sum(), y)
    assert torch.allclose(g1.double(), g2.double(), rtol=1e-5, atol=1e-6 * g2.abs().max().item())


def test_solve_through_loss_gradient_matches_central_differences():
    sp = spots.turn_boundary_spots(3, seed=31)
    bs = ps.BatchSolver([spots.card_config(r, b) for r, b, _ in sp], [t for _, _, t in sp])
    torch.manual_seed(0)
    net = torch.nn.Sequential(torch.nn.Linear(2720, 16), torch.nn.ReLU(), torch.nn.Linear(16, 1326)).cuda().double()
    rng = np.random.default_rng(3)
    target = torch.tensor(rng.normal(0, 5, (3, 2, 1326)).astype(np.float32), device="cuda")
    ranges = np.stack([np.stack(r) for r, _, _ in sp])
    mask = torch.tensor((ranges > 0).astype(np.float32), device="cuda")
    loss = T.solve_through_loss(bs, net, target, mask, iterations=20, eval_interval=10)
    net.zero_grad()
    loss.backward()
    last = net[2]
    assert last.weight.grad.abs().sum() > 0 and net[0].weight.grad.abs().sum() > 0
    # the same loss at the solved strategy, as a function of the last layer
    items = bs.boundary_items()
    reach = bs.boundary_reach(device=True)

    def L():
        with torch.no_grad():
            B = T.boundary_values(items, reach, net)
            cfv = T.FixedStrategyRootValues.apply(bs, B)
            return T.masked_mse(cfv.double(), target.double(), mask.double()).item()

    h = 1.0  # the loss is quadratic in the last layer: central differences are exact for any step
    picks = [("bias", int(i)) for i in rng.choice(1326, 6, replace=False)] + \
            [("weight", (int(i), int(j))) for i, j in zip(rng.choice(1326, 6), rng.choice(16, 6))]
    got, fd = [], []
    for name, idx in picks:
        p = getattr(last, name)
        g = p.grad[idx].item()
        with torch.no_grad():
            p[idx] += h
        lp = L()
        with torch.no_grad():
            p[idx] -= 2 * h
        lm = L()
        with torch.no_grad():
            p[idx] += h
        got.append(g)
        fd.append((lp - lm) / (2 * h))
    got, fd = np.array(got), np.array(fd)
    assert np.abs(got - fd).max() <= 1e-3 * max(np.abs(fd).max(), 1e-12), (got, fd)
