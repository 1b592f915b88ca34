"""CUDA path against the oracle on the same seeded inputs (needs a B200).

Bit-exact: hand-strength orders, valid-hand lists (the device-built board
tables), tree shape.  Floating point: the device keeps regrets, strategy sums
and counterfactual values in FP32 like the reference, but sums terminal reach
in FP32 where the reference accumulates in f64, so values agree within the
tolerances below, stated per quantity.

Two kinds of checks.  One-step parity: the oracle's regrets and strategy sums
after k iterations are copied into the GPU game, then one evaluation / one
iteration runs on both from the identical state - this is deterministic and
held to tight tolerances on every tree kind (river, turn with chance nodes,
isomorphic chance pruning, depth boundaries, rake).  Trajectories: whole
solves are compared on well-conditioned river spots; regret matching makes a
DCFR trajectory sensitive to the last bit where two actions' regrets tie (the
oracle's own FP32 and FP64 builds part ways at the same nodes), so long
trajectories are compared by exploitability against the FP64 oracle.
"""

import json
import os

import numpy as np
import pytest

import poker_solver_rust_b200 as ps
from tests import spots

pytestmark = pytest.mark.gpu

# tolerances (absolute unless stated).  Per-hand strategies of hands whose
# regrets sit near zero are sensitive to the last bit of a terminal sum, so the
# strategy check bounds both the worst entry and the mean over all entries.
TOL_STRATEGY = 1e-2          # max |sigma_gpu - sigma_oracle| over nodes x actions x hands
TOL_STRATEGY_MEAN = 2e-4     # mean of the same
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


def _strategy_diffs(g, o):
    diffs = [np.abs(g.strategy_at_index(i) - o.strategy_at_index(i)) for i in _decision_nodes(g)]
    allv = np.concatenate(diffs) if diffs else np.zeros(1)
    return float(allv.max()), float(allv.mean())


def _max_strategy_diff(g, o):
    mx, mean = _strategy_diffs(g, o)
    assert mean <= TOL_STRATEGY_MEAN, ("mean strategy diff", mean)
    return mx


def _expl_close(a, b, pot):
    return abs(a - b) <= TOL_EXPL_REL * max(abs(b), 1e-3 * pot)


TOL_STEP_REL = 2e-4   # one iteration from a shared state: max |dR|, |dS| relative to max |R|, |S|
TOL_EVAL_REL = 2e-5   # exploitability / root values from a shared state, relative


def _share_state(g, o):
    """Copies the oracle's cumulative strategy and regrets into the GPU game."""
    for i in range(g.num_nodes()):
        info = g.node_info(i)
        if info["player"] & (4 | 8):
            continue
        g.seed_node_storage(i, 1, o.node_storage(i, 1).astype(np.float32))
        g.seed_node_storage(i, 2, o.node_storage(i, 2).astype(np.float32))


def _state_diff(g, o, player=None):
    dr = ds = sr = ss = 0.0
    for i in range(g.num_nodes()):
        info = g.node_info(i)
        if info["player"] & (4 | 8) or (player is not None and info["player"] != player):
            continue
        for which in (1, 2):
            a, b = g.node_storage(i, which), o.node_storage(i, which)
            d = float(np.abs(a - b).max())
            m = float(np.abs(b).max())
            if which == 1:
                ds, ss = max(ds, d), max(ss, m)
            else:
                dr, sr = max(dr, d), max(sr, m)
    return dr / max(sr, 1e-30), ds / max(ss, 1e-30)


def _sparse(rng, board):  # ~130-combo ranges keep the CPU oracle fast on turn trees
    out = []
    for _ in range(2):
        w = rng.random(1326).astype(np.float32)
        w[rng.random(1326) < 0.9] = 0.0
        out.append(spots._mask_board(w, board))
    return out


def _iso_spot():
    r0 = ps.Range.from_str("AA,KK,QQ,AKs,AQs,KQo").raw_data()
    r1 = ps.Range.from_str("JJ-99,AJs,KJs,QJs,T9s").raw_data()
    board = ps.board_from_str("Kh Qh 7h 2s")
    sz = ps.BetSizeOptions("50%, a", "100%")
    tc = ps.TreeConfig(initial_state=ps.BoardState.Turn, starting_pot=100, effective_stack=150,
                       turn_bet_sizes=[sz, sz], river_bet_sizes=[sz, sz])
    return [spots._mask_board(r0.copy(), board), spots._mask_board(r1.copy(), board)], board, tc


def _spot(kind):
    if kind == "river":
        return spots.river_spot(12)
    if kind == "raked":
        r, b, t = spots.river_spot(13)
        t.rake_rate, t.rake_cap = 0.05, 3.0
        return r, b, t
    if kind == "turn":
        return spots.turn_spot(8, weights=_sparse)
    if kind == "iso":
        return _iso_spot()
    if kind == "boundary":
        r, b, t = spots.turn_spot(9)
        t.depth_limit = 0
        return r, b, t
    if kind == "datagen":
        return spots.datagen_spot(np.random.default_rng(77))
    raise ValueError(kind)


def _set_boundaries(g, o, seed=4):
    rng = np.random.default_rng(seed)
    for k in range(g.num_boundary_nodes()):
        for p in range(2):
            v = rng.normal(0, 1, g.num_private_hands(p)).astype(np.float32)
            g.set_boundary_cfvs(k, p, v)
            o.set_boundary_cfvs(k, p, v)


@pytest.mark.parametrize("kind", ["river", "raked", "turn", "iso", "boundary", "datagen"])
@pytest.mark.parametrize("k", [1, 6])
def test_one_step_parity(kind, k):
    r, board, tc = _spot(kind)
    g = spots.product_game(r, board, tc)
    o = spots.oracle_game(r, board, tc)
    if kind == "boundary":
        _set_boundaries(g, o)
    if kind == "iso":
        assert o.isomorphism_counts(board[3])[2] > 0 and g.num_nodes() == o.num_nodes()
    for t in range(k):
        o.solve_step(t)
    _share_state(g, o)
    assert _state_diff(g, o) == (0.0, 0.0)
    e, eo = ps.compute_exploitability(g), o.compute_exploitability()
    row = {"expl_gpu": e, "expl_oracle": eo}
    assert abs(e - eo) <= TOL_EVAL_REL * max(abs(eo), 1e-3 * tc.starting_pot), row
    for p in range(2):
        v, vo = ps.root_cfvalues(g, p), o.root_cfvalues(p)
        row[f"root_cfv_rel_{p}"] = float(np.abs(v - vo).max() / max(np.abs(vo).max(), 1e-30))
        assert row[f"root_cfv_rel_{p}"] <= 10 * TOL_EVAL_REL, row
    # one DCFR iteration on the GPU; the oracle replays it pass by pass.  The
    # second (IP) pass starts from the GPU's OOP update, so each pass is
    # checked from identical inputs.
    ps.solve_step(g, k)
    o.solve_pass(k, 0)
    dr0, ds0 = _state_diff(g, o, player=0)
    for i in range(g.num_nodes()):
        info = g.node_info(i)
        if not info["player"] & (4 | 8) and info["player"] == 0:
            o.seed_node_storage(i, 1, g.node_storage(i, 1))
            o.seed_node_storage(i, 2, g.node_storage(i, 2))
    o.solve_pass(k, 1)
    dr1, ds1 = _state_diff(g, o, player=1)
    row.update({"oop_pass_dR_rel": dr0, "oop_pass_dS_rel": ds0, "ip_pass_dR_rel": dr1, "ip_pass_dS_rel": ds1})
    _report(f"one_step_{kind}_{k}", row)
    assert max(dr0, ds0, dr1, ds1) <= TOL_STEP_REL, row


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
            sd, sm = _strategy_diffs(g, o)
            sd64, sm64 = _strategy_diffs(g, o64)
            so64, _ = _strategy_diffs(o, o64)
            rows.append({"t": t + 1, "gpu": e, "oracle": eo, "fp64": e64, "strategy_maxdiff": sd,
                         "strategy_meandiff": sm, "strategy_maxdiff_gpu_vs_fp64": sd64,
                         "strategy_maxdiff_oracle32_vs_fp64": so64,
                         "gpu_vs_fp64": abs(e - e64), "oracle_vs_fp64": abs(eo - e64)})
            assert sm <= TOL_STRATEGY_MEAN, rows[-1]
            assert _expl_close(e, eo, 100), rows[-1]
            assert abs(e - e64) <= max(5 * abs(eo - e64), TOL_EXPL_REL * max(e64, 0.1)), rows[-1]
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
    assert _max_strategy_diff(g, o) <= TOL_STRATEGY


@pytest.mark.parametrize("kind", ["river", "turn"])
def test_finalize_and_queries(kind):
    r, board, tc = spots.river_spot(4) if kind == "river" else spots.turn_spot(8, weights=_sparse)
    g = spots.product_game(r, board, tc)
    o = spots.oracle_game(r, board, tc)
    for t in range(30):
        o.solve_step(t)
    _share_state(g, o)
    ps.finalize(g)
    o.finalize()
    rows = {}
    paths = ([], [1], [1, 1], [0], [0, 2]) if kind == "river" else ([], [1], [1, 1], [1, 1, 5], [0, 0, 9, 1])
    for path in paths:
        g.back_to_root()
        o.back_to_root()
        for a in path:
            if g.is_terminal_node():
                break
            if g.is_chance_node():
                a = [c for c in range(52) if (g.possible_cards() >> c) & 1][a % 5]
            g.play(a)
            o.play(a)
        assert g.available_actions() == o.available_actions()
        assert g.current_node_index() == o.current_node_index()
        assert g.total_bet_amount() == o.total_bet_amount()
        g.cache_normalized_weights()
        o.cache_normalized_weights()
        for p in range(2):
            nw, nwo = g.normalized_weights(p), o.weights(p, normalized=True)
            assert np.abs(nw - nwo).max() <= 1e-5 * max(1.0, float(np.abs(nwo).max()))
            ev, evo = g.expected_values(p), o.expected_values(p)
            scale = max(1.0, float(np.abs(evo).max()))
            rows[f"{kind}{path}_{p}"] = float(np.abs(ev - evo).max() / scale)
            assert np.abs(ev - evo).max() <= 1e-4 * scale, rows
        if not g.is_terminal_node() and not g.is_chance_node():
            assert np.abs(g.strategy() - o.strategy()).max() <= 1e-6
    _report(f"query_ev_rel_{kind}", rows)


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


def test_batch_matches_single_and_oracle():
    """Batch == single game bit for bit; the state the batch stops in is a state
    of the oracle's map.

    Whole trajectories are not compared here: on datagen spots the oracle's own
    FP32 and FP64 builds part ways by whole multiples of the exploitability
    within 60 iterations (regret-matching ties), so the stopping iteration is
    compared only as a report.  Instead the oracle is seeded with the GPU's
    final regrets and strategy sums: both must then agree on the exploitability
    and on one further iteration, pass by pass.
    """
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
        assert ps.solve(g, 300, float(targets[i])) == e[i] and g.last_iterations == it[i]  # same arithmetic
        assert e[i] <= targets[i] or it[i] == 300
        # the same solve step by step, stopped before finalize so that its
        # regrets and strategy sums can be handed to the oracle
        g = spots.product_game(r, b, t)
        es, k = ps.compute_exploitability(g), 0
        while k < 300 and not es <= targets[i]:
            ps.solve_step(g, k)
            k += 1
            if k % 5 == 0 or k == 300:
                es = ps.compute_exploitability(g)
        assert es == e[i] and k == it[i]
        o = spots.oracle_game(r, b, t)
        eo = o.solve(300, float(targets[i]))
        row = {"gpu": float(e[i]), "oracle": eo, "it": int(it[i]), "it_o": o.iterations_run}
        o2 = spots.oracle_game(r, b, t)
        for n in range(g.num_nodes()):
            info = g.node_info(n)
            if not info["player"] & (4 | 8):
                o2.seed_node_storage(n, 1, g.node_storage(n, 1))
                o2.seed_node_storage(n, 2, g.node_storage(n, 2))
        row["oracle_at_gpu_state"] = o2.compute_exploitability()
        assert abs(row["oracle_at_gpu_state"] - es) <= TOL_EVAL_REL * max(abs(es), 1e-3 * t.starting_pot), row
        ps.solve_step(g, k)
        o2.solve_pass(k, 0)
        dr0, ds0 = _state_diff(g, o2, player=0)
        for n in range(g.num_nodes()):
            info = g.node_info(n)
            if not info["player"] & (4 | 8) and info["player"] == 0:
                o2.seed_node_storage(n, 1, g.node_storage(n, 1))
                o2.seed_node_storage(n, 2, g.node_storage(n, 2))
        o2.solve_pass(k, 1)
        dr1, ds1 = _state_diff(g, o2, player=1)
        row["next_step_rel"] = max(dr0, ds0, dr1, ds1)
        rows.append(row)
        assert row["next_step_rel"] <= TOL_STEP_REL, row
    _report("batch", rows)


def test_batch_node_storage_matches_single_game():
    """ps_batch_node_storage (the batch's extract_results) returns every
    decision node's strategy sums and regrets as the single game does after
    the same solve."""
    sp = spots.datagen_spots(3, seed=52)
    cc = [spots.card_config(r, b) for r, b, _ in sp]
    tcs = [t for _, _, t in sp]
    bs = ps.BatchSolver(cc, tcs)
    bs.solve(25, np.full(3, -1e30, np.float32))
    for i, (r, b, t) in enumerate(sp):
        g = spots.product_game(r, b, t)
        for k in range(25):
            ps.solve_step(g, k)
        assert bs.num_nodes(i) == g.num_nodes()
        for n in range(g.num_nodes()):
            for which in (1, 2):
                assert np.array_equal(bs.node_storage(i, n, which), g.node_storage(n, which))


def test_batch_root_cfvalues_match_single_game():
    """The batch's device-side root cfvalues equal the single game's
    root_cfvalues after the same solve (same kernels, same arithmetic)."""
    sp = spots.datagen_spots(5, seed=44)
    cc = [spots.card_config(r, b) for r, b, _ in sp]
    tcs = [t for _, _, t in sp]
    targets = np.array([0.003 * t.starting_pot for t in tcs], np.float32)
    bs = ps.BatchSolver(cc, tcs)
    bs.solve(300, targets)
    for i, (r, b, t) in enumerate(sp):
        g = spots.product_game(r, b, t)
        ps.solve(g, 300, float(targets[i]))
        for p in range(2):
            assert np.array_equal(bs.root_cfvalues(i, p), ps.root_cfvalues(g, p))


@pytest.mark.parametrize("inst", [2, 3])
def test_batch_lockstep_instances_keep_results(inst):
    """Spots of one tree shape solved in lockstep by one CTA: every spot's
    iteration count, exploitability and root values equal the one-spot-per-CTA
    solve (a spot that meets its target leaves the lockstep set)."""
    sp = spots.datagen_spots(48, seed=35)
    cc = [spots.card_config(r, b) for r, b, _ in sp]
    tcs = [t for _, _, t in sp]
    targets = np.array([0.003 * t.starting_pot for t in tcs], np.float32)
    one = ps.BatchSolver(cc, tcs)
    one.solve(300, targets)
    many = ps.BatchSolver(cc, tcs, instances_per_cta=inst)
    many.solve(300, targets)
    e0, i0 = one.results()
    e1, i1 = many.results()
    assert np.array_equal(i0, i1) and np.array_equal(e0, e1)
    for k in range(0, 48, 7):
        for p in range(2):
            assert np.array_equal(one.root_cfvalues(k, p), many.root_cfvalues(k, p))


def test_batch_autotune_keeps_results():
    """block_threads=-1 times every CTA size on a sample of the batch and keeps
    the fastest; the spots' arithmetic does not depend on the CTA size."""
    sp = spots.datagen_spots(48, seed=33)
    cc = [spots.card_config(r, b) for r, b, _ in sp]
    tcs = [t for _, _, t in sp]
    targets = np.array([0.003 * t.starting_pot for t in tcs], np.float32)
    ref = ps.BatchSolver(cc, tcs)
    ref.solve(300, targets)
    e0, it0 = ref.results()
    tuned = ps.BatchSolver(cc, tcs, block_threads=-1)
    cands = [(b, u) for b in range(128, 257, 32) for u in (max(1, b // 64), b // 32)]
    log = tuned.autotune_log()
    assert [(b, u) for b, u, _ in log] in ([], cands) and all(ms > 0 for _, _, ms in log)
    cfg = tuned.config()
    assert (cfg["block_threads"], cfg["scan_buffers"]) in cands
    if log:
        best = min(log, key=lambda x: x[2])
        assert (cfg["block_threads"], cfg["scan_buffers"]) == best[:2]
    tuned.solve(300, targets)
    e1, it1 = tuned.results()
    assert np.array_equal(it0, it1)
    assert np.allclose(e0, e1, rtol=1e-5, atol=0)


def test_grid_mode_matches_single_cta(monkeypatch):
    """A large single tree runs on every CTA of a cooperative launch; the
    arithmetic of each item does not depend on which warp runs it, so the
    state matches the one-CTA run bit for bit."""
    r, b, t = spots.turn_spot(8, weights=_sparse)
    grid = spots.product_game(r, b, t)            # default: grid mode for single trees >= 16 nodes
    assert grid.num_nodes() >= 2000
    assert grid.schedule()["mode"] == "grid"      # too wide for one cluster
    monkeypatch.setenv("PS_GRID_NODES", "0")
    one = spots.product_game(r, b, t)
    for it in range(4):
        ps.solve_step(grid, it)
        ps.solve_step(one, it)
    assert ps.compute_exploitability(grid) == ps.compute_exploitability(one)
    for i in _decision_nodes(grid)[:50]:
        assert np.array_equal(grid.node_storage(i, 2), one.node_storage(i, 2))
        assert np.array_equal(grid.node_storage(i, 1), one.node_storage(i, 1))
    e1 = ps.solve(grid, 12, 0.0)
    e2 = ps.solve(one, 12, 0.0)
    assert e1 == e2 and grid.last_iterations == one.last_iterations


@pytest.mark.parametrize("ctas", ["8", "16"])
def test_cluster_mode_matches_grid_mode(monkeypatch, ctas):
    """A single game on the CTAs of one thread-block cluster (hardware
    cluster barrier between steps) against the cooperative grid: the items'
    arithmetic is the same wherever they run, so every query matches bit for
    bit - the solve loop with its checks, single steps, finalize, root values
    and the expected values."""
    r, b, t = spots.river_spot(1)
    monkeypatch.delenv("PS_GRID_CLUSTER", raising=False)
    dflt = spots.product_game(r, b, t).schedule()  # a 33-node river game: one cluster by default
    assert dflt["mode"] == "cluster" and dflt["ctas"] == 16
    monkeypatch.setenv("PS_GRID_CLUSTER", "0")
    grid = spots.product_game(r, b, t)
    monkeypatch.setenv("PS_GRID_CLUSTER", ctas)
    clu = spots.product_game(r, b, t)
    assert grid.schedule()["mode"] == "grid"
    assert clu.schedule()["mode"] == "cluster" and clu.schedule()["ctas"] == int(ctas)
    for it in range(3):
        ps.solve_step(grid, it)
        ps.solve_step(clu, it)
    assert ps.compute_exploitability(grid) == ps.compute_exploitability(clu)
    for i in _decision_nodes(grid):
        assert np.array_equal(grid.node_storage(i, 2), clu.node_storage(i, 2))
        assert np.array_equal(grid.node_storage(i, 1), clu.node_storage(i, 1))
    e1 = ps.solve(grid, 60, 0.0)
    e2 = ps.solve(clu, 60, 0.0)
    assert e1 == e2 and grid.last_iterations == clu.last_iterations
    for p in range(2):  # solve() ended with finalize, as the reference's does
        assert np.array_equal(ps.root_cfvalues(grid, p), ps.root_cfvalues(clu, p))
    assert np.array_equal(grid.strategy_at_index(0), clu.strategy_at_index(0))
    for g in (grid, clu):
        g.cache_normalized_weights()
    for p in range(2):
        assert np.array_equal(grid.expected_values(p), clu.expected_values(p))


@pytest.mark.parametrize("case", [0, 1, 2])
def test_regret_matching_known_answers(case):
    """solver.rs:724-750 on the device: one iteration at t = 0 (gamma_0 = 0)
    leaves the strategy sum equal to the regret-matched seeded regrets."""
    from tests.test_oracle_pins import REGRET_CASES, _decision_node, _fixture_oracle, _tile

    pattern, na, expected = REGRET_CASES[case]
    r, board, tc = _fixture_oracle()
    g = spots.product_game(r, board, tc)
    idx = _decision_node(g, na, 0)
    H = g.num_private_hands(0)
    g.seed_node_storage(idx, 2, _tile(pattern, na, H))
    ps.solve_step(g, 0)
    want = np.full(na * H, 1.0 / na) if expected is None else _tile(expected, na, H)
    assert np.abs(g.node_storage(idx, 1) - want).max() < 1e-6


def test_normalized_strategy_known_answers():
    """utility.rs:1012-1036 through the product's strategy query."""
    from tests.test_oracle_pins import _decision_node, _fixture_oracle, _tile

    r, board, tc = _fixture_oracle()
    g = spots.product_game(r, board, tc)
    idx = _decision_node(g, 2, 1)
    H = g.num_private_hands(1)
    g.seed_node_storage(idx, 1, np.zeros(2 * H, np.float32))
    assert np.abs(g.strategy_at_index(idx) - 0.5).max() < 1e-6
    g.seed_node_storage(idx, 1, _tile([1.0, 3.0, 3.0, 1.0], 2, H))
    assert np.abs(g.strategy_at_index(idx) - _tile([0.25, 0.75, 0.75, 0.25], 2, H)).max() < 1e-6


def test_early_termination():
    """solver.rs:808-838: a target above the starting exploitability stops at once."""
    from tests.test_oracle_pins import _fixture_oracle

    r, board, tc = _fixture_oracle()
    g = spots.product_game(r, board, tc)
    e = ps.solve(g, 1000, 1e10)
    assert e >= 0.0 and g.last_iterations == 0


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
