"""Device pieces of the turn-datagen boundary pipeline against host restatements.

Boundary reach: the oracle records the opponent's reach at every boundary it
evaluates; after its average-strategy passes (root_cfvalues) from the same
strategy sums it must match ps_boundary_reach.  River reduction: the oracle's f64
numpy restatement of cfvnet/src/datagen/gpu_boundary_eval.rs:207-269 on random
inputs; the device sums the per-river weights in another order, so values
agree to f32 rounding (tolerance 1e-6 relative).
"""

import numpy as np
import pytest
import torch

import poker_solver_rust_b200 as ps
from poker_solver_rust_b200.datagen import boundary_reach, boundary_river_reduce
from oracle import boundary_io as bio
from tests import spots
from tests.test_gpu_adjoint import _copy_strategy, _sparse

pytestmark = pytest.mark.gpu


def test_boundary_reach_matches_oracle():
    rng = np.random.default_rng(3)
    r, b, t = spots.turn_spot(9, weights=_sparse)
    t.depth_limit = 0
    g = spots.product_game(r, b, t)
    o = spots.oracle_game(r, b, t, fp64=True)
    for k in range(g.num_boundary_nodes()):
        for p in range(2):
            v = rng.normal(0, 1, g.num_private_hands(p)).astype(np.float32)
            g.set_boundary_cfvs(k, p, v)
            o.set_boundary_cfvs(k, p, v)
    for it in range(20):
        ps.solve_step(g, it)
    _copy_strategy(g, o)
    o.root_cfvalues(0)  # records player 1's reach at each boundary
    o.root_cfvalues(1)  # ... and player 0's
    got = boundary_reach(g)
    assert len(got) == g.num_boundary_nodes() > 0
    for k in range(len(got)):
        for p in range(2):
            ref = o.boundary_reach(k, p)
            assert np.abs(got[k][p] - ref).max() <= 1e-6 * max(1.0, np.abs(ref).max())


def test_boundary_river_reduce_matches_reference():
    rng = np.random.default_rng(11)
    n = 3
    boards = np.stack([rng.choice(52, 4, replace=False) for _ in range(n)]).astype(np.uint8)
    pots = rng.uniform(20, 200, n).astype(np.float32).round()
    stacks = rng.uniform(20, 400, n).astype(np.float32).round()
    reach = rng.random((n, 2, 1326)).astype(np.float32)
    pairs = bio.combo_pairs()
    for i in range(n):  # no reach on combos blocked by the board
        for c in range(1326):
            if set(pairs[c].tolist()) & set(boards[i].tolist()):
                reach[i, :, c] = 0.0
    net = rng.normal(0, 0.1, (n, 2, 48, 1326)).astype(np.float32)
    hands = rng.choice(1326, 200, replace=False).astype(np.int32)
    ref = bio.river_reduce(boards, pots, stacks, net, reach, hands)
    got = boundary_river_reduce(boards, pots, stacks, torch.from_numpy(net).cuda(), torch.from_numpy(reach).cuda(),
                                torch.from_numpy(hands).cuda()).cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-6 * max(1.0, np.abs(ref).max())
