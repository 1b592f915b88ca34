"""Batched depth-limited solving and the on-device boundary-network pipeline.

- Input rows: the encoding kernel against the oracle's restatement of
  boundary_evaluator.rs:27-60, bit for bit (f32, and bf16 as the rounding of
  those f32 rows).
- Batch vs single games: a batch of depth-limited turn spots given boundary
  values in the 1326-combo layout solves every spot exactly as the single game
  given the same values per hand; iteration ranges (run_iterations) continue
  the same state as solve_step, and the epilogue's boundary reach equals the
  single game's ps_boundary_reach scattered to combos.  Both sides run the same
  kernels, so the comparison is bit for bit.
- The datagen loop (solve_with_boundary_net) against the same loop composed by
  hand from single games and the separately checked device pieces.
- The factored first layer (boundary_first_layer) against the network's first
  Linear on the encoded rows, within 1e-5 of the largest output (f32; the sums
  run in another order); bf16 output as the rounding of the f32 one.
"""

import numpy as np
import pytest
import torch

import poker_solver_rust_b200 as ps
from oracle import boundary_io as bio
from poker_solver_rust_b200.datagen import (boundary_encode, boundary_first_layer, boundary_reach,
                                            boundary_river_reduce, evaluate_boundaries, solve_with_boundary_net)
from tests import spots
from tests.test_gpu_adjoint import _sparse

pytestmark = pytest.mark.gpu


def _dl_spots(n, seed):
    out = []
    for i in range(n):
        r, b, t = spots.turn_spot(seed + i, weights=_sparse if i % 2 else None)
        t.depth_limit = 0
        if i % 3 == 2:
            t.effective_stack = 60  # a second tree shape
        out.append((r, b, t))
    return out


def _batch(sp, **kw):
    return ps.BatchSolver([spots.card_config(r, b) for r, b, _ in sp], [t for _, _, t in sp], **kw)


def _combos(g, p):
    return np.array([ps.card_pair_to_index(int(a), int(b)) for a, b in g.private_cards(p)])


def _set_single(g, items, i, V):
    ks = np.nonzero(items["spot"] == i)[0]
    assert len(ks) == g.num_boundary_nodes() > 0
    for j, k in enumerate(ks):
        assert items["ordinal"][k] == j
        for p in range(2):
            g.set_boundary_cfvs(j, p, np.ascontiguousarray(V[k, p, _combos(g, p)]))
    return ks


def test_boundary_encode_bit_exact():
    rng = np.random.default_rng(17)
    n = 3
    boards = np.stack([rng.choice(52, 4, replace=False) for _ in range(n)]).astype(np.uint8)
    pots = rng.uniform(10, 300, n).astype(np.float32).round()
    stacks = rng.uniform(0, 400, n).astype(np.float32).round()
    stacks[0] = 0.0
    reach = rng.random((n, 2, 1326)).astype(np.float32)
    reach[rng.random(reach.shape) < 0.3] = 0.0
    ref = bio.encode_rows(boards, pots, stacks, reach)
    d_reach = torch.from_numpy(reach).cuda()
    got = boundary_encode(boards, pots, stacks, d_reach).cpu().numpy()
    assert got.shape == (n, 2, 48, 2720)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    got16 = boundary_encode(boards, pots, stacks, d_reach, bf16=True).cpu()
    assert torch.equal(got16.view(torch.int16), torch.from_numpy(ref).to(torch.bfloat16).view(torch.int16))


def test_batch_depth_limited_matches_single_games():
    sp = _dl_spots(5, 60)
    bs = _batch(sp)
    items = bs.boundary_items()
    rng = np.random.default_rng(1)
    V = rng.normal(0, 1, (len(items["spot"]), 2, 1326)).astype(np.float32)
    bs.set_boundary_cfvs(V)
    bs.solve(40, np.full(len(sp), -1e30, np.float32))  # no early stop
    e, it = bs.results()
    assert (it == 40).all()
    for i, (r, b, t) in enumerate(sp):
        g = spots.product_game(r, b, t)
        ks = _set_single(g, items, i, V)
        nodes = g.boundary_node_indices()
        for j, k in enumerate(ks):
            amount = g.node_info(int(nodes[j]))["amount"]
            assert items["pots"][k] == t.starting_pot + 2 * amount
            assert items["stacks"][k] == t.effective_stack - amount
            assert list(items["boards"][k]) == list(b[:4])
        assert ps.solve(g, 40, -1e30) == e[i]
        for p in range(2):
            assert np.array_equal(bs.root_cfvalues(i, p), ps.root_cfvalues(g, p))


def test_run_iterations_and_boundary_reach_match_single_games():
    sp = _dl_spots(4, 80)
    bs = _batch(sp, instances_per_cta=2)
    items = bs.boundary_items()
    rng = np.random.default_rng(2)
    V = rng.normal(0, 1, (len(items["spot"]), 2, 1326)).astype(np.float32)
    bs.set_boundary_cfvs(torch.from_numpy(V).cuda())  # device path of the setter
    bs.run_iterations(0, 7, root=False)
    bs.run_iterations(7, 15, root=True, exploitability=True)
    e, it = bs.results()
    assert (it == 15).all()
    R = bs.boundary_reach()
    Rd = bs.boundary_reach(device=True).cpu().numpy()
    assert np.array_equal(R, Rd)
    for i, (r, b, t) in enumerate(sp):
        g = spots.product_game(r, b, t)
        ks = _set_single(g, items, i, V)
        for k in range(15):
            ps.solve_step(g, k)
        assert ps.compute_exploitability(g) == e[i]
        for p in range(2):
            assert np.array_equal(bs.root_cfvalues(i, p), ps.root_cfvalues(g, p))
        br = boundary_reach(g)
        for j, k in enumerate(ks):
            for p in range(2):
                want = np.zeros(1326, np.float32)
                want[_combos(g, p)] = br[j][p]
                assert np.array_equal(R[k, p], want)
    # a reset starts again from zero state with the same boundary values
    bs.reset()
    bs.run_iterations(0, 15, root=False, exploitability=True)
    assert np.array_equal(bs.results()[0], e)


def _net():
    torch.manual_seed(0)
    return torch.nn.Sequential(torch.nn.Linear(2720, 64), torch.nn.ReLU(), torch.nn.Linear(64, 1326)).cuda()


def test_solve_with_boundary_net_composes_the_pieces():
    sp = _dl_spots(3, 90)
    net = _net()
    bs = _batch(sp)
    items = solve_with_boundary_net(bs, net, iterations=12, eval_interval=5, factored=False)
    e, it = bs.results()
    assert (it == 12).all()
    # the same loop by hand: single games, their own boundary reach, the
    # network on the rows of all items at once, the river average
    games = [spots.product_game(r, b, t) for r, b, t in sp]
    n = len(items["spot"])
    for i, g in enumerate(games):
        _set_single(g, items, i, np.zeros((n, 2, 1326), np.float32))
    combos = torch.arange(1326, dtype=torch.int32, device="cuda")
    t = 0
    while True:
        reach = np.zeros((n, 2, 1326), np.float32)
        for i, g in enumerate(games):
            br = boundary_reach(g)
            for j, k in enumerate(np.nonzero(items["spot"] == i)[0]):
                for p in range(2):
                    reach[k, p, _combos(g, p)] = br[j][p]
        d_reach = torch.from_numpy(reach).cuda()
        rows = boundary_encode(items["boards"], items["pots"], items["stacks"], d_reach)
        with torch.no_grad():
            y = net(rows.view(n * 96, 2720)).float().view(n, 2, 48, 1326)
        V = boundary_river_reduce(items["boards"], np.ones(n, np.float32), np.zeros(n, np.float32), y, d_reach,
                                  combos).cpu().numpy()
        for i, g in enumerate(games):
            _set_single(g, items, i, V)
        end = min(12, t + 5)
        for k in range(t, end):
            for g in games:
                ps.solve_step(g, k)
        t = end
        if t >= 12:
            break
    for i, g in enumerate(games):
        assert ps.compute_exploitability(g) == e[i]
        for p in range(2):
            assert np.array_equal(bs.root_cfvalues(i, p), ps.root_cfvalues(g, p))


def test_batch_adjoint_matches_single_games():
    """ps_batch_adjoint: every spot's values and gradients equal the single
    game's ps_eval_fixed_strategy(_adjoint) with the same strategy, weights
    and cotangents (which tests/test_gpu_adjoint.py holds against FP64 central
    differences)."""
    sp = _dl_spots(4, 120)
    bs = _batch(sp, instances_per_cta=2)
    items = bs.boundary_items()
    rng = np.random.default_rng(3)
    V = rng.normal(0, 1, (len(items["spot"]), 2, 1326)).astype(np.float32)
    bs.set_boundary_cfvs(V)
    bs.run_iterations(0, 20, root=True)
    cot = rng.normal(0, 1, (len(sp), 2, 1326)).astype(np.float32)
    dw, dB = bs.adjoint(cot)
    cfv = bs.root_cfvalues_all()
    dw_d, dB_d = bs.adjoint(torch.from_numpy(cot).cuda())
    assert np.array_equal(dw, dw_d.cpu().numpy()) and np.array_equal(dB, dB_d.cpu().numpy())
    assert np.array_equal(cfv, bs.root_cfvalues_all(device=True).cpu().numpy())
    for i, (r, b, t) in enumerate(sp):
        g = spots.product_game(r, b, t)
        ks = _set_single(g, items, i, V)
        for k in range(20):
            ps.solve_step(g, k)
        w = [g.initial_weights(p) for p in range(2)]
        cb = [_combos(g, p) for p in range(2)]
        c = ps.eval_fixed_strategy(g, w[0], w[1])
        d0, d1, db = ps.eval_fixed_strategy_adjoint(g, w[0], w[1], cot[i, 0, cb[0]], cot[i, 1, cb[1]])
        for p, dwp in ((0, d0), (1, d1)):
            assert np.array_equal(cfv[i, p, cb[p]], c[p])
            assert np.array_equal(dw[i, p, cb[p]], dwp)
            assert not np.delete(dw[i, p], cb[p]).any()
            for j, k in enumerate(ks):
                assert np.array_equal(dB[k, p, cb[p]], db[j][p])
                assert not np.delete(dB[k, p], cb[p]).any()


def test_batch_solved_values_autograd():
    """loss = MSE(root cfvalues, target) through BatchSolvedValues: the
    gradient reaching the boundary values is the batched adjoint of
    dL/dcfv."""
    from poker_solver_rust_b200.autograd import batch_solved_values

    sp = _dl_spots(3, 140)
    bs = _batch(sp)
    n = bs.num_boundary_items()
    rng = np.random.default_rng(4)
    B = torch.tensor(rng.normal(0, 25, (n, 2, 1326)).astype(np.float32), device="cuda", requires_grad=True)
    target = torch.tensor(rng.normal(0, 25, (len(sp), 2, 1326)).astype(np.float32), device="cuda")
    cfv = batch_solved_values(bs, B, 30)
    loss = ((cfv - target) ** 2).mean()
    loss.backward()
    cot = (2.0 / cfv.numel()) * (cfv.detach() - target)
    _, dB = bs.adjoint(cot)
    assert torch.equal(B.grad, dB)
    assert B.grad.abs().sum() > 0


def _random_items(rng, n):
    boards = np.stack([rng.choice(52, 4, replace=False) for _ in range(n)]).astype(np.uint8)
    pots = rng.uniform(10, 300, n).astype(np.float32).round()
    stacks = rng.uniform(0, 400, n).astype(np.float32).round()
    reach = rng.random((n, 2, 1326)).astype(np.float32)
    pairs = bio.combo_pairs()
    for i in range(n):
        blocked = np.isin(pairs[:, 0], boards[i]) | np.isin(pairs[:, 1], boards[i])
        reach[i, :, blocked] = 0.0
    return boards, pots, stacks, torch.from_numpy(reach).cuda()


def test_factored_first_layer_matches_dense():
    rng = np.random.default_rng(23)
    boards, pots, stacks, reach = _random_items(rng, 3)
    torch.manual_seed(1)
    lin = torch.nn.Linear(2720, 40).cuda()
    with torch.no_grad():
        dense = lin(boundary_encode(boards, pots, stacks, reach).view(-1, 2720)).view(3, 2, 48, 40)
        fact = boundary_first_layer(boards, pots, stacks, reach, lin.weight, lin.bias)
        f16 = boundary_first_layer(boards, pots, stacks, reach, lin.weight, lin.bias, bf16=True)
    scale = dense.abs().max().item()
    assert (fact - dense).abs().max().item() <= 1e-5 * scale
    assert torch.equal(f16, fact.to(torch.bfloat16))


def test_bf16_river_average_and_factored_evaluation():
    rng = np.random.default_rng(29)
    boards, pots, stacks, reach = _random_items(rng, 2)
    combos = torch.arange(1326, dtype=torch.int32, device="cuda")
    y = torch.tensor(rng.normal(0, 0.1, (2, 2, 48, 1326)).astype(np.float32), device="cuda").to(torch.bfloat16)
    a = boundary_river_reduce(boards, pots, stacks, y, reach, combos)
    b = boundary_river_reduce(boards, pots, stacks, y.float(), reach, combos)
    assert torch.equal(a, b)
    torch.manual_seed(2)
    net = torch.nn.Sequential(torch.nn.Linear(2720, 32), torch.nn.ReLU(), torch.nn.Linear(32, 1326)).cuda()
    items = {"boards": boards, "pots": pots, "stacks": stacks, "spot": np.zeros(2, np.int32)}
    fast = evaluate_boundaries(items, reach, net)
    slow = evaluate_boundaries(items, reach, net, factored=False)
    assert (fast - slow).abs().max().item() <= 1e-4 * slow.abs().max().item()
