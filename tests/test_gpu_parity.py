"""CUDA path against the oracle on the same seeded inputs (needs a B200).

Bit-exact: hand-strength orders, valid-hand lists (the device-built board
tables), tree shape.  Floating point: the device keeps regrets, strategy sums
and counterfactual values in FP32 like the reference, but sums terminal reach
in FP32 where the reference accumulates in f64, so values agree within the
tolerances below, stated per quantity.
"""

import json
import os

import numpy as np
import pytest

import poker_solver_rust_b200 as ps
from tests import spots

pytestmark = pytest.mark.gpu

# tolerances (absolute unless stated)
TOL_STRATEGY = 2e-3          # average strategy probabilities after <= 200 iterations
TOL_EXPL_REL = 2e-3          # exploitability, relative to max(|oracle|, 1e-3 * pot)
TOL_CFV_REL = 1e-4           # root cfvalues, relative to max |value|

_REPORT = {}


def _report(key, val):
    _REPORT[key] = val
    out = os.environ.get("PS_PARITY_REPORT")
    if out:
        with open(out, "w") as f:
            json.dump(_REPORT, f, indent=1, default=float)


def _decision_nodes(g):
    out = []
    for i in range(g.num_nodes()):
        info = g.node_info(i)
        if not info["player"] & (4 | 8) and info["num_children"] > 1:
            out.append(i)
    return out


def _max_strategy_diff(g, o):
    d = 0.0
    for i in _decision_nodes(g):
        d = max(d, float(np.abs(g.strategy_at_index(i) - o.strategy_at_index(i)).max()))
    return d


def _expl_close(a, b, pot):
    return abs(a - b) <= TOL_EXPL_REL * max(abs(b), 1e-3 * pot)


def test_board_tables_bit_exact():
    for r, board, tc in (spots.river_spot(2), spots.turn_spot(4)):
        g = spots.product_game(r, board, tc)
        o = spots.oracle_game(r, board, tc)
        turn = board[3]
        rivers = [board[4]] if len(board) == 5 else [c for c in range(52) if c not in board]
        for rv in rivers:
            pi = ps.card_pair_to_index(turn, rv)
            for p in range(2):
                s, i = g.hand_strength(turn, rv, p)
                so, io = o.hand_strength(pi, p)
                assert np.array_equal(s, so) and np.array_equal(i, io), (turn, rv, p)
                assert np.array_equal(g.valid_indices(turn, rv, p), o.valid_indices(2, pi, p))
        if len(board) == 4:
            for p in range(2):
                assert np.array_equal(g.valid_indices(turn, 255, p), o.valid_indices(1, turn, p))


def test_initial_exploitability():
    r, board, tc = spots.river_spot(1)
    g = spots.product_game(r, board, tc)
    o = spots.oracle_game(r, board, tc)
    e, eo = ps.compute_exploitability(g), o.compute_exploitability()
    _report("initial_expl", {"gpu": e, "oracle": eo})
    assert _expl_close(e, eo, 100)


@pytest.mark.parametrize("seed", [1, 2])
def test_river_iterations(seed):
    r, board, tc = spots.river_spot(seed)
    g = spots.product_game(r, board, tc)
    o = spots.oracle_game(r, board, tc)
    o64 = spots.oracle_game(r, board, tc, fp64=True)
    rows = []
    for t in range(200):
        ps.solve_step(g, t)
        o.solve_step(t)
        o64.solve_step(t)
        if t + 1 in (1, 10, 50, 200):
            e, eo, e64 = ps.compute_exploitability(g), o.compute_exploitability(), o64.compute_exploitability()
            sd = _max_strategy_diff(g, o)
            rows.append({"t": t + 1, "gpu": e, "oracle": eo, "fp64": e64, "strategy_maxdiff": sd,
                         "gpu_vs_fp64": abs(e - e64), "oracle_vs_fp64": abs(eo - e64)})
            assert _expl_close(e, eo, 100), rows[-1]
            assert sd <= TOL_STRATEGY, rows[-1]
    _report(f"river_iterations_{seed}", rows)


def test_river_solve_to_target():
    r, board, tc = spots.river_spot(3)
    g = spots.product_game(r, board, tc)
    o = spots.oracle_game(r, board, tc)
    target = 0.003 * 100
    e = ps.solve(g, 1000, target)
    eo = o.solve(1000, target)
    _report("solve_to_target", {"gpu": e, "oracle": eo, "iters_gpu": g.last_iterations, "iters_oracle": o.iterations_run})
    assert e <= target and eo <= target
    assert abs(g.last_iterations - o.iterations_run) <= 5
    assert _max_strategy_diff(g, o) <= 5 * TOL_STRATEGY


def test_finalize_and_queries():
    r, board, tc = spots.river_spot(4)
    g = spots.product_game(r, board, tc)
    o = spots.oracle_game(r, board, tc)
    ps.solve(g, 60, 0.0)
    o.solve(60, 0.0)
    rows = {}
    for path in ([], [1], [1, 1], [0], [0, 2]):
        g.back_to_root()
        o.back_to_root()
        for a in path:
            if g.is_terminal_node():
                break
            g.play(a)
            o.play(a)
        assert g.available_actions() == o.available_actions()
        assert g.current_node_index() == o.current_node_index()
        assert g.total_bet_amount() == o.total_bet_amount()
        g.cache_normalized_weights()
        o.cache_normalized_weights()
        for p in range(2):
            np.testing.assert_allclose(g.normalized_weights(p), o.weights(p, normalized=True), rtol=1e-5, atol=1e-6)
            ev, evo = g.expected_values(p), o.expected_values(p)
            scale = max(1.0, float(np.abs(evo).max()))
            rows[f"{path}_{p}"] = float(np.abs(ev - evo).max() / scale)
            assert np.abs(ev - evo).max() <= 1e-2 * scale
        if not g.is_terminal_node() and not g.is_chance_node():
            assert np.abs(g.strategy() - o.strategy()).max() <= 5 * TOL_STRATEGY
    _report("query_ev_rel", rows)


def test_root_cfvalues_with_reach():
    r, board, tc = spots.river_spot(5)
    g = spots.product_game(r, board, tc)
    o = spots.oracle_game(r, board, tc)
    for t in range(30):
        ps.solve_step(g, t)
        o.solve_step(t)
    rng = np.random.default_rng(9)
    for p in range(2):
        reach = rng.random(g.num_private_hands(p ^ 1)).astype(np.float32)
        v = ps.root_cfvalues_with_reach(g, p, reach)
        vo = o.root_cfvalues_with_reach(p, reach)
        err = float(np.abs(v - vo).max() / max(1e-12, np.abs(vo).max()))
        _report(f"root_cfv_rel_{p}", err)
        assert err <= 50 * TOL_CFV_REL


def test_raked_river():
    r, board, tc = spots.river_spot(6)
    tc.rake_rate, tc.rake_cap = 0.05, 3.0
    g = spots.product_game(r, board, tc)
    o = spots.oracle_game(r, board, tc)
    for t in range(40):
        ps.solve_step(g, t)
        o.solve_step(t)
    e, eo = ps.compute_exploitability(g), o.compute_exploitability()
    _report("raked", {"gpu": e, "oracle": eo})
    assert _expl_close(e, eo, 100)
    assert _max_strategy_diff(g, o) <= TOL_STRATEGY


def test_turn_spot():
    def small(rng, board):  # ~100-combo ranges keep the CPU oracle fast
        out = []
        for _ in range(2):
            w = rng.random(1326).astype(np.float32)
            w[rng.random(1326) < 0.9] = 0.0
            out.append(spots._mask_board(w, board))
        return out
    r, board, tc = spots.turn_spot(8, weights=small)
    g = spots.product_game(r, board, tc)
    o = spots.oracle_game(r, board, tc)
    for t in range(20):
        ps.solve_step(g, t)
        o.solve_step(t)
    e, eo = ps.compute_exploitability(g), o.compute_exploitability()
    _report("turn", {"gpu": e, "oracle": eo, "strategy_maxdiff": _max_strategy_diff(g, o)})
    assert _expl_close(e, eo, 100)
    assert _max_strategy_diff(g, o) <= TOL_STRATEGY


def test_depth_limited_turn_boundary():
    r, board, tc = spots.turn_spot(9)
    tc.depth_limit = 0
    g = spots.product_game(r, board, tc)
    o = spots.oracle_game(r, board, tc)
    nb = g.num_boundary_nodes()
    assert nb == o.num_boundary_nodes() > 0
    assert np.array_equal(g.boundary_node_indices(), o.boundary_node_indices())
    rng = np.random.default_rng(4)
    for k in range(nb):
        for p in range(2):
            v = rng.normal(0, 1, g.num_private_hands(p)).astype(np.float32)
            g.set_boundary_cfvs(k, p, v)
            o.set_boundary_cfvs(k, p, v)
    for t in range(30):
        ps.solve_step(g, t)
        o.solve_step(t)
    e, eo = ps.compute_exploitability(g), o.compute_exploitability()
    _report("boundary", {"gpu": e, "oracle": eo})
    assert _expl_close(e, eo, 100)
    assert _max_strategy_diff(g, o) <= TOL_STRATEGY


def test_isomorphic_turn():
    # suit-symmetric ranges on a board missing two suits: the reference skips
    # isomorphic river cards and adds their suit-swapped values
    r0 = ps.Range.from_str("AA,KK,QQ,AKs,AQs,KQo").raw_data()
    r1 = ps.Range.from_str("JJ-99,AJs,KJs,QJs,T9s").raw_data()
    board = ps.board_from_str("Kh Qh 7h 2s")
    sz = ps.BetSizeOptions("50%, a", "100%")
    tc = ps.TreeConfig(initial_state=ps.BoardState.Turn, starting_pot=100, effective_stack=150,
                       turn_bet_sizes=[sz, sz], river_bet_sizes=[sz, sz])
    r = [spots._mask_board(r0.copy(), board), spots._mask_board(r1.copy(), board)]
    o = spots.oracle_game(r, board, tc)
    assert o.isomorphism_counts(board[3])[2] > 0
    g = spots.product_game(r, board, tc)
    assert g.num_nodes() == o.num_nodes()
    for t in range(20):
        ps.solve_step(g, t)
        o.solve_step(t)
    e, eo = ps.compute_exploitability(g), o.compute_exploitability()
    _report("isomorphic", {"gpu": e, "oracle": eo})
    assert _expl_close(e, eo, 100)
    assert _max_strategy_diff(g, o) <= TOL_STRATEGY


def test_batch_matches_single_and_oracle():
    sp = spots.datagen_spots(6, seed=21)
    cc = [spots.card_config(r, b) for r, b, _ in sp]
    tcs = [t for _, _, t in sp]
    bs = ps.BatchSolver(cc, tcs)
    targets = np.array([0.003 * t.starting_pot for t in tcs], np.float32)
    bs.solve(300, targets)
    e, it = bs.results()
    rows = []
    for i, (r, b, t) in enumerate(sp):
        g = spots.product_game(r, b, t)
        es = ps.solve(g, 300, float(targets[i]))
        assert es == e[i] and g.last_iterations == it[i]  # same kernels, same arithmetic
        o = spots.oracle_game(r, b, t)
        eo = o.solve(300, float(targets[i]))
        rows.append({"gpu": float(e[i]), "oracle": eo, "it": int(it[i]), "it_o": o.iterations_run})
        assert abs(int(it[i]) - o.iterations_run) <= 5, rows[-1]
        assert _expl_close(float(e[i]), eo, t.starting_pot) or (e[i] <= targets[i] and eo <= targets[i]), rows[-1]
    _report("batch", rows)


def test_state_export_import():
    r, board, tc = spots.river_spot(7)
    g = spots.product_game(r, board, tc)
    for t in range(10):
        ps.solve_step(g, t)
    snap = g.storage_export()
    for t in range(10, 20):
        ps.solve_step(g, t)
    e1 = ps.compute_exploitability(g)
    g.storage_import(snap)
    for t in range(10, 20):
        ps.solve_step(g, t)
    assert ps.compute_exploitability(g) == e1


def test_edge_cases():
    # one hand per player, and a board that blocks every combo but one
    board = ps.board_from_str("As Ks Qs Js Ts")
    w0 = np.zeros(1326, np.float32)
    w1 = np.zeros(1326, np.float32)
    w0[ps.card_pair_to_index(ps.card_from_str("2c"), ps.card_from_str("2d"))] = 1.0
    w1[ps.card_pair_to_index(ps.card_from_str("3c"), ps.card_from_str("3d"))] = 0.5
    sz = ps.BetSizeOptions("50%, a", "")
    tc = ps.TreeConfig(initial_state=ps.BoardState.River, starting_pot=10, effective_stack=10,
                       river_bet_sizes=[sz, sz])
    g = spots.product_game([w0, w1], board, tc)
    o = spots.oracle_game([w0, w1], board, tc)
    e, eo = ps.solve(g, 50, 0.0), o.solve(50, 0.0)
    assert abs(e - eo) <= 1e-5
    # both players hold the same combo set: same-hand index path
    r = spots.uniform_ranges(np.random.default_rng(3), board)
    r[1] = r[0].copy()
    g = spots.product_game(r, board, tc)
    o = spots.oracle_game(r, board, tc)
    for t in range(20):
        ps.solve_step(g, t)
        o.solve_step(t)
    assert _expl_close(ps.compute_exploitability(g), o.compute_exploitability(), 10)
    # solve / solve_step after finalize are state errors
    with pytest.raises(ps.SolverError):
        ps.solve_step(g, 0) if ps.finalize(g) is None else None
