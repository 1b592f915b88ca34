"""torch.autograd.Function over fixed-strategy evaluation of a solved game.

With the average strategy held fixed, the root cfvalues of each player are
linear in the opponent's initial weights and in the player's depth-boundary
values.  `FixedStrategyValues` exposes that map to PyTorch: forward runs the
C-ABI evaluation (ps_eval_fixed_strategy), backward the hand-written adjoint
kernels (ps_eval_fixed_strategy_adjoint), so a boundary-value model can be
trained through a solved depth-limited tree.  Tensors may live on any device;
CUDA tensors stay on the device: the library reads and writes them through
device pointers (ps_eval_fixed_strategy_ex and its adjoint, every boundary
value in one ps_set_boundary_cfvs_all call); host tensors go through host
copies.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _native as N
from . import game as G


class FixedStrategyValues(torch.autograd.Function):
    """(w0, w1, B0, B1) -> (cfv0, cfv1).

    w_p: [H_p] initial weights in solver hand order; B_p: [n_boundary, H_p]
    boundary values of player p (ps_set_boundary_cfvs); cfv_p: [H_p] root
    cfvalues of player p under the average strategy.
    """

    @staticmethod
    def forward(ctx, game, w0, w1, b0, b1):
        if w0.is_cuda:
            return _forward_device(ctx, game, w0, w1, b0, b1)
        nb = game.num_boundary_nodes()
        for k in range(nb):
            game.set_boundary_cfvs(k, 0, b0[k].detach().cpu().numpy().astype(np.float32))
            game.set_boundary_cfvs(k, 1, b1[k].detach().cpu().numpy().astype(np.float32))
        a = w0.detach().cpu().numpy()
        b = w1.detach().cpu().numpy()
        c0, c1 = G.eval_fixed_strategy(game, a, b)
        ctx.game = game
        ctx.save_for_backward(w0, w1, b0, b1)
        dev, dt = w0.device, w0.dtype
        return torch.from_numpy(c0).to(dev, dt), torch.from_numpy(c1).to(dev, dt)

    @staticmethod
    def backward(ctx, g0, g1):
        w0, w1, b0, b1 = ctx.saved_tensors
        game = ctx.game
        if w0.is_cuda:
            return _backward_device(game, w0, w1, b0, b1, g0, g1)
        nb = game.num_boundary_nodes()
        for k in range(nb):  # the values the forward pass saw
            game.set_boundary_cfvs(k, 0, b0[k].detach().cpu().numpy().astype(np.float32))
            game.set_boundary_cfvs(k, 1, b1[k].detach().cpu().numpy().astype(np.float32))
        dw0, dw1, db = G.eval_fixed_strategy_adjoint(
            game, w0.detach().cpu().numpy(), w1.detach().cpu().numpy(),
            None if g0 is None else g0.detach().cpu().numpy(), None if g1 is None else g1.detach().cpu().numpy())
        dev, dt = w0.device, w0.dtype
        db0 = torch.from_numpy(np.stack([db[k][0] for k in range(nb)]) if nb else np.zeros((0, w0.shape[0]),
                                                                                           np.float32))
        db1 = torch.from_numpy(np.stack([db[k][1] for k in range(nb)]) if nb else np.zeros((0, w1.shape[0]),
                                                                                           np.float32))
        return (None, torch.from_numpy(dw0).to(dev, dt), torch.from_numpy(dw1).to(dev, dt), db0.to(dev, dt),
                db1.to(dev, dt))


def _f32(t):
    return t.detach().to(torch.float32).contiguous()


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _set_boundaries_device(game, b0, b1):
    """Every boundary value in one call from the device: [nb, H0 + H1] rows."""
    if game.num_boundary_nodes() == 0:
        return None
    rows = torch.cat([_f32(b0), _f32(b1)], dim=1).contiguous()
    torch.cuda.current_stream(rows.device).synchronize()
    N.check(N.lib().ps_set_boundary_cfvs_all(game._h, _ptr(rows), 1))
    return rows


def _forward_device(ctx, game, w0, w1, b0, b1):
    keep = _set_boundaries_device(game, b0, b1)
    a, b = _f32(w0), _f32(w1)
    c0 = torch.empty(game.num_private_hands(0), dtype=torch.float32, device=w0.device)
    c1 = torch.empty(game.num_private_hands(1), dtype=torch.float32, device=w0.device)
    torch.cuda.current_stream(w0.device).synchronize()
    N.check(N.lib().ps_eval_fixed_strategy_ex(game._h, _ptr(a), _ptr(b), _ptr(c0), _ptr(c1), 1))
    del keep
    ctx.game = game
    ctx.save_for_backward(w0, w1, b0, b1)
    return c0.to(w0.dtype), c1.to(w0.dtype)


def _backward_device(game, w0, w1, b0, b1, g0, g1):
    keep = _set_boundaries_device(game, b0, b1)  # the values the forward pass saw
    H0, H1, nb = game.num_private_hands(0), game.num_private_hands(1), game.num_boundary_nodes()
    a, b = _f32(w0), _f32(w1)
    ga = None if g0 is None else _f32(g0)
    gb = None if g1 is None else _f32(g1)
    dw0 = torch.empty(H0, dtype=torch.float32, device=w0.device)
    dw1 = torch.empty(H1, dtype=torch.float32, device=w0.device)
    db = torch.empty((max(nb, 1), H0 + H1), dtype=torch.float32, device=w0.device)
    torch.cuda.current_stream(w0.device).synchronize()
    N.check(N.lib().ps_eval_fixed_strategy_adjoint_ex(
        game._h, _ptr(a), _ptr(b), None if ga is None else _ptr(ga), None if gb is None else _ptr(gb),
        _ptr(dw0), _ptr(dw1), _ptr(db), 1))
    del keep
    dt = w0.dtype
    return None, dw0.to(dt), dw1.to(dt), db[:nb, :H0].to(dt), db[:nb, H0:].to(dt)


def fixed_strategy_values(game, w0, w1, b0, b1):
    """Root cfvalues (cfv0, cfv1) of `game` as a differentiable function of
    the initial weights and boundary values (see FixedStrategyValues)."""
    return FixedStrategyValues.apply(game, w0, w1, b0, b1)


class BatchSolvedValues(torch.autograd.Function):
    """Boundary values -> root cfvalues of a batch of depth-limited spots.

    Forward: the boundary values B [items, 2, 1326] (combo layout, CUDA) go
    into the batch, every spot runs `iterations` DCFR iterations from zero
    state in one launch, and the root cfvalues of both players under the
    resulting average strategy come back as [n, 2, 1326].  Backward: the
    batched adjoint (ps_batch_adjoint) with that strategy held fixed, i.e. the
    gradient of the fixed-strategy evaluation, as FixedStrategyValues gives it
    for one game.  Everything stays on the device.
    """

    @staticmethod
    def forward(ctx, batch, values, iterations):
        batch.set_boundary_cfvs(values)
        batch.reset()
        batch.run_iterations(0, int(iterations), root=True)
        ctx.batch = batch
        return batch.root_cfvalues_all(device=True).to(values.dtype)

    @staticmethod
    def backward(ctx, g):
        _, dB = ctx.batch.adjoint(g.float())
        return None, dB.to(g.dtype), None


def batch_solved_values(batch, values, iterations: int):
    """Root cfvalues [n, 2, 1326] of a BatchSolver's depth-limited spots solved
    with boundary values `values` [items, 2, 1326] (see BatchSolvedValues)."""
    return BatchSolvedValues.apply(batch, values, iterations)
