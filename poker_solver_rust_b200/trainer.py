"""Training a boundary-value network through solved depth-limited trees.

The reference trains its BoundaryNet (cfvnet python/cfvnet/model.py) only on
supervised targets read from datagen records (python/cfvnet/train.py,
loss.py).  With the batched adjoint, the network can also be trained through
the tree it feeds: the depth-limited spots are solved with the network's
boundary values (datagen.solve_with_boundary_net), then, with that average
strategy held fixed, a loss on the spots' root cfvalues is differentiated with
respect to the network's parameters:

    rows = boundary_encode(reach)           no gradient (solver state)
    y    = net(rows)                        torch autograd
    B    = RiverAverage(y)                  device forward, torch backward
    cfv  = FixedStrategyRootValues(B)       device forward, ps_batch_adjoint backward
    loss = masked MSE(cfv, target)

`solve_through_loss` builds that graph; `loss.backward()` reaches the network.
"""

from __future__ import annotations

import numpy as np
import torch

from .datagen import boundary_encode, boundary_river_reduce, solve_with_boundary_net

_PAIRS = None


def _pairs(device):
    global _PAIRS
    if _PAIRS is None or _PAIRS.device != torch.device(device):
        p = [(a, b) for a in range(52) for b in range(a + 1, 52)]
        _PAIRS = torch.tensor(p, dtype=torch.int64, device=device)
    return _PAIRS


def river_keep_mask(boards, device):
    """[n, 48, 1326] bool: combo c holds none of river r's card, for the 48
    rivers (ascending) of each 4-card board."""
    b = torch.as_tensor(np.asarray(boards, np.int64).reshape(-1, 4), device=device)
    cards = torch.arange(52, device=device)
    free = (cards[None, :, None] != b[:, None, :]).all(dim=2)  # [n, 52]
    rivers = cards.expand(b.shape[0], 52)[free].view(-1, 48)
    pr = _pairs(device)
    return (pr[None, None, :, 0] != rivers[:, :, None]) & (pr[None, None, :, 1] != rivers[:, :, None])


class RiverAverage(torch.autograd.Function):
    """The reach-weighted 48-river average (ps_boundary_river_reduce, combo
    layout) as a function of the network outputs y [n, 2, 48, 1326]; reach
    and the scale are constants.  Backward: dB/dy[i,p,r,c] = scale_i *
    W[i,p,r] * keep[i,r,c] / sum_r' W[i,p,r'] keep[i,r',c], where W[i,p,r] is
    the opponent's reach on combos free of river r (gpu_boundary_eval.rs:146-161)."""

    @staticmethod
    def forward(ctx, y, boards, scale, reach):
        combos = torch.arange(1326, dtype=torch.int32, device=y.device)
        scale = np.asarray(scale, np.float32)
        out = boundary_river_reduce(boards, scale, np.zeros(len(scale), np.float32), y.detach(), reach, combos)
        ctx.save_for_backward(reach, torch.as_tensor(scale, device=y.device))
        ctx.boards = boards
        return out

    @staticmethod
    def backward(ctx, g):
        reach, s = ctx.saved_tensors
        keep = river_keep_mask(ctx.boards, g.device).to(torch.float64)  # [n, 48, 1326]
        opp = reach.flip(1).to(torch.float64)  # player 0 weighted by IP reach, player 1 by OOP reach
        W = torch.einsum("npc,nrc->npr", opp, keep)  # [n, 2, 48]
        den = torch.einsum("npr,nrc->npc", W, keep)  # [n, 2, 1326]
        coef = torch.where(den > 0, g.to(torch.float64) * s[:, None, None].to(torch.float64) / den.clamp_min(1e-300),
                           torch.zeros_like(den))
        gy = W[:, :, :, None] * keep[:, None, :, :] * coef[:, :, None, :]
        return gy.to(g.dtype), None, None, None


class FixedStrategyRootValues(torch.autograd.Function):
    """Boundary values [items, 2, 1326] -> root cfvalues [n, 2, 1326] of every
    spot under the batch's current average strategy (no iterations);
    backward: the batched adjoint (ps_batch_adjoint)."""

    @staticmethod
    def forward(ctx, batch, values):
        batch.set_boundary_cfvs(values)
        batch.run_iterations(0, 0, root=True)
        ctx.batch = batch
        return batch.root_cfvalues_all(device=True)

    @staticmethod
    def backward(ctx, g):
        _, dB = ctx.batch.adjoint(g.float())
        return None, dB


def boundary_values(items, reach, net, pot_source: str = "boundary", denormalize: bool = False,
                    bf16: bool = False, chunk_items: int = 512):
    """Differentiable boundary values [items, 2, 1326] from the network (the
    graph of datagen.evaluate_boundaries with autograd through the network
    and the river average)."""
    n = len(items["spot"])
    if pot_source == "root":
        pots, stacks = items["root_pots"], items["root_stacks"]
    else:
        pots, stacks = items["pots"], items["stacks"]
    scale = (pots + stacks).astype(np.float32) if denormalize else np.ones(n, np.float32)
    parts = []
    for a in range(0, n, chunk_items):
        z = slice(a, min(n, a + chunk_items))
        m = z.stop - z.start
        rows = boundary_encode(items["boards"][z], pots[z], stacks[z], reach[z], bf16=bf16)
        x = rows.view(m * 96, 2720)
        p = next(net.parameters(), None) if hasattr(net, "parameters") else None
        if p is not None and p.dtype != x.dtype:
            x = x.to(p.dtype)
        y = net(x).float().view(m, 2, 48, 1326)
        parts.append(RiverAverage.apply(y, items["boards"][z], scale[z], reach[z]))
    return torch.cat(parts)


def masked_mse(cfv, target, mask):
    """Mean squared error over the entries where mask is set."""
    d = (cfv - target) * mask
    return (d * d).sum() / mask.sum().clamp_min(1.0)


def solve_through_loss(batch, net, target, mask, iterations: int, eval_interval: int, **kw):
    """Solve the batch's depth-limited spots with the network's boundary
    values (no gradient), then return masked MSE(root cfvalues at the solved
    strategy, target) as a differentiable function of the network.  target,
    mask: [n, 2, 1326] CUDA tensors (mask 1 on the hands to fit)."""
    with torch.no_grad():
        solve_with_boundary_net(batch, net, iterations, eval_interval, **kw)
    items = batch.boundary_items()
    reach = batch.boundary_reach(device=True)
    B = boundary_values(items, reach, net, **kw)
    cfv = FixedStrategyRootValues.apply(batch, B)
    return masked_mse(cfv, target, mask)
