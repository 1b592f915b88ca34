"""Parity at the sizes of the benchmark configurations, with every result's
error against the FP64 oracle stated (needs a B200).

config 1  one river game (1081 live combos per player, pot 100 / stack 200,
          bets 50% / 100% / all-in, raise 100%), 1000 DCFR iterations;
config 2  one turn game (1128 live combos, 48 river deals, 12,285 nodes, pot
          100 / stack 300, bets 33% / 75% / all-in, raise 60%), 500 iterations;
config 3  batched datagen river spots solved to <= 0.3% of the pot;
config 4  256 batched depth-limited turn trees, strategy frozen after 200
          iterations, adjoint against FP64 central differences (h = 1e-3) on
          512 random coordinates per tree.

Trajectories: the GPU, the oracle's FP32 build and its FP64 build run the same
iterations side by side.  DCFR is sensitive to the last bit where regret
matching meets ties, so the FP32-vs-FP64 spread of the oracle itself is the
yardstick: the GPU must sit as close to FP64 as the FP32 reference does (or
within the stated relative tolerance).  The map itself is checked at full size
from a shared state (the oracle's regrets and strategy sums copied into the
GPU, one iteration pass by pass).  Results go to the file named by
PS_SPEC_REPORT (JSON) when it is set.
"""

import json
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import poker_solver_rust_b200 as ps
from tests import spots

pytestmark = pytest.mark.gpu

TOL_EXPL_REL = 2e-3       # exploitability vs the FP32 oracle, relative to max(|oracle|, 1e-3 * pot)
TOL_EXPL_SPREAD = 5.0     # |gpu - fp64| <= 5 x |fp32 oracle - fp64| (or the relative bound above)
TOL_STRATEGY = 1e-2       # max |sigma_gpu - sigma_oracle| over every node, action and hand
TOL_STRATEGY_MEAN = 2e-4  # mean of the same
TOL_STRATEGY_SPREAD = 3.0  # chaotic trajectories: mean |sigma_gpu - sigma_fp64| <= 3 x that of the FP32 reference
TOL_STEP_REL = 2e-4       # one iteration from a shared state: max |dR|, |dS| relative to max |R|, |S|
TOL_EVAL_REL = 2e-5       # exploitability from one state, relative ...
TOL_EVAL_ULPS = 8         # ... or within 8 f32 ulps of the half pot: the reference rounds each player's
                          # best-response value (about half the pot) to f32 before the two are combined,
                          # so near convergence the result carries that rounding in absolute terms
TOL_CFV_REL = 1e-4        # root cfvalues from one state, relative to the largest |value|
TOL_GRAD_REL = 1e-4       # adjoint: per coordinate, relative to max(|fd|, floor)
GRAD_FLOOR = 1e-2         # ... floor = GRAD_FLOOR x the largest |fd| of the tree's block: a weight gradient is
                          # a sum of f32 terms up to that size, so near zero it carries their rounding (measured:
                          # at most 3.5e-7 of the block's largest), not a relative error

_REPORT = {}


def _report(key, val):
    _REPORT[key] = val
    out = os.environ.get("PS_SPEC_REPORT")
    if out:
        with open(out, "w") as f:
            json.dump(_REPORT, f, indent=1, default=float)


def _decision_nodes(g):
    return [i for i in range(g.num_nodes())
            if not g.node_info(i)["player"] & (4 | 8) and g.node_info(i)["num_children"] > 1]


def _strategy_diffs(games, nodes):
    """Max and mean |sigma_a - sigma_b| over every node, action and hand for
    the pairs (gpu, fp32), (gpu, fp64), (fp32, fp64), node by node."""
    pairs = ((0, 1), (0, 2), (1, 2))
    mx = [0.0] * 3
    tot = [0.0] * 3
    cnt = 0
    root = [None] * 3
    for i in nodes:
        s = [np.asarray(g.strategy_at_index(i), np.float64) for g in games]
        if root[0] is None:
            root = s
        for k, (a, b) in enumerate(pairs):
            d = np.abs(s[a] - s[b])
            mx[k] = max(mx[k], float(d.max()))
            tot[k] += float(d.sum())
        cnt += len(s[0])
    mean = [x / max(cnt, 1) for x in tot]
    root_err = float(np.abs(root[0] - root[2]).max()) if root[0] is not None else 0.0
    return mx, mean, root_err


def _trajectory(r, b, t, iters, checks, threads=1):
    """GPU, FP32 oracle and FP64 oracle in lockstep; rows at `checks`."""
    from oracle import oracle as O

    g = spots.product_game(r, b, t)
    o = spots.oracle_game(r, b, t)
    o64 = spots.oracle_game(r, b, t, fp64=True)
    nodes = _decision_nodes(g)
    rows = []
    O.set_chance_threads(threads)
    try:
        for it in range(iters):
            ps.solve_step(g, it)
            o.solve_step(it)
            o64.solve_step(it)
            if it + 1 in checks:
                e, e32, e64 = ps.compute_exploitability(g), o.compute_exploitability(), o64.compute_exploitability()
                mx, mean, root_err = _strategy_diffs((g, o, o64), nodes)
                rows.append({
                    "t": it + 1, "expl_gpu": e, "expl_fp32": e32, "expl_fp64": e64,
                    "expl_pct_pot_gpu": 100 * e / t.starting_pot,
                    "expl_err_gpu_vs_fp64": abs(e - e64), "expl_err_fp32_vs_fp64": abs(e32 - e64),
                    "strategy_max_gpu_vs_fp32": mx[0], "strategy_mean_gpu_vs_fp32": mean[0],
                    "strategy_max_gpu_vs_fp64": mx[1], "strategy_mean_gpu_vs_fp64": mean[1],
                    "strategy_max_fp32_vs_fp64": mx[2], "strategy_mean_fp32_vs_fp64": mean[2],
                    "root_strategy_max_gpu_vs_fp64": root_err,
                })
    finally:
        O.set_chance_threads(1)
    return g, o, o64, rows


def _check_rows(rows, pot):
    """Well-conditioned trajectories: the GPU follows the FP32 reference."""
    for row in rows:
        e, e32, e64 = row["expl_gpu"], row["expl_fp32"], row["expl_fp64"]
        assert abs(e - e32) <= TOL_EXPL_REL * max(abs(e32), 1e-3 * pot), row
        assert abs(e - e64) <= max(TOL_EXPL_SPREAD * abs(e32 - e64), TOL_EXPL_REL * max(e64, 1e-3 * pot)), row
        assert row["strategy_mean_gpu_vs_fp32"] <= TOL_STRATEGY_MEAN, row
        assert row["strategy_max_gpu_vs_fp32"] <= TOL_STRATEGY, row


def _check_rows_chaotic(rows, pot):
    """Trajectories where the reference's own FP32 and FP64 builds part ways
    (regret-matching ties at full turn size): the GPU must stay as close to
    the FP64 trajectory as the FP32 reference does - exploitability within
    TOL_EXPL_SPREAD times, mean strategy distance within TOL_STRATEGY_SPREAD
    times the FP32 build's own distance."""
    for row in rows:
        e, e32, e64 = row["expl_gpu"], row["expl_fp32"], row["expl_fp64"]
        assert abs(e - e64) <= max(TOL_EXPL_SPREAD * abs(e32 - e64), TOL_EXPL_REL * max(e64, 1e-3 * pot)), row
        assert row["strategy_mean_gpu_vs_fp64"] <= max(TOL_STRATEGY_SPREAD * row["strategy_mean_fp32_vs_fp64"],
                                                       TOL_STRATEGY_MEAN), row


def _share_state(g, o):
    for i in range(g.num_nodes()):
        if g.node_info(i)["player"] & (4 | 8):
            continue
        g.seed_node_storage(i, 1, o.node_storage(i, 1).astype(np.float32))
        g.seed_node_storage(i, 2, o.node_storage(i, 2).astype(np.float32))


def _state_diff(g, o, player):
    dr = ds = sr = ss = 0.0
    for i in range(g.num_nodes()):
        info = g.node_info(i)
        if info["player"] & (4 | 8) or info["player"] != player:
            continue
        for which in (1, 2):
            a, b = g.node_storage(i, which), o.node_storage(i, which)
            d, m = float(np.abs(a - b).max()), float(np.abs(b).max())
            if which == 1:
                ds, ss = max(ds, d), max(ss, m)
            else:
                dr, sr = max(dr, d), max(sr, m)
    return dr / max(sr, 1e-30), ds / max(ss, 1e-30)


def _one_step_from_shared_state(g, o, t, pot):
    """The oracle's state copied into the GPU game; exploitability, root
    cfvalues and one iteration (pass by pass) compared from it."""
    _share_state(g, o)
    e, eo = ps.compute_exploitability(g), o.compute_exploitability()
    floor = max(abs(eo), 1e-3 * pot, TOL_EVAL_ULPS * float(np.spacing(np.float32(0.5 * pot))) / TOL_EVAL_REL)
    row = {"expl_gpu": e, "expl_oracle": eo, "expl_abs": abs(e - eo), "expl_rel": abs(e - eo) / floor}
    for p in range(2):
        v, vo = ps.root_cfvalues(g, p), o.root_cfvalues(p)
        row[f"root_cfv_rel_{p}"] = float(np.abs(v - vo).max() / max(np.abs(vo).max(), 1e-30))
    ps.solve_step(g, t)
    o.solve_pass(t, 0)
    row["oop_pass_dR_rel"], row["oop_pass_dS_rel"] = _state_diff(g, o, 0)
    for i in range(g.num_nodes()):
        info = g.node_info(i)
        if not info["player"] & (4 | 8) and info["player"] == 0:
            o.seed_node_storage(i, 1, g.node_storage(i, 1))
            o.seed_node_storage(i, 2, g.node_storage(i, 2))
    o.solve_pass(t, 1)
    row["ip_pass_dR_rel"], row["ip_pass_dS_rel"] = _state_diff(g, o, 1)
    return row


def _check_one_step(row):
    assert row["expl_rel"] <= TOL_EVAL_REL, row
    assert max(row["root_cfv_rel_0"], row["root_cfv_rel_1"]) <= 10 * TOL_EVAL_REL, row
    assert max(row["oop_pass_dR_rel"], row["oop_pass_dS_rel"], row["ip_pass_dR_rel"],
               row["ip_pass_dS_rel"]) <= TOL_STEP_REL, row


def test_config1_river_game_1000_iterations():
    r, b, t = spots.river_spot(1)  # the bench's single river game
    g, o, o64, rows = _trajectory(r, b, t, 1000, {1, 10, 100, 250, 500, 1000})
    _report("config1_river_1000", {"nodes": g.num_nodes(), "hands": [g.num_private_hands(0),
                                                                      g.num_private_hands(1)], "rows": rows})
    _check_rows(rows, t.starting_pot)
    row = _one_step_from_shared_state(g, o, 1000, t.starting_pot)
    _report("config1_one_step_at_1000", row)
    _check_one_step(row)


def test_config2_turn_game_full_size():
    r, b, t = spots.turn_spot(2)  # the bench's single turn game: 1128 live combos, 48 river deals
    threads = os.cpu_count() or 1
    g, o, o64, rows = _trajectory(r, b, t, 500, {10, 100, 250, 500}, threads=threads)
    assert g.num_private_hands(0) == 1128 and g.num_nodes() > 12000
    _report("config2_turn_500", {"nodes": g.num_nodes(), "hands": [g.num_private_hands(0),
                                                                    g.num_private_hands(1)], "rows": rows})
    _check_rows_chaotic(rows, t.starting_pot)
    from oracle import oracle as O

    O.set_chance_threads(threads)
    try:
        row = _one_step_from_shared_state(g, o, 500, t.starting_pot)
    finally:
        O.set_chance_threads(1)
    _report("config2_one_step_at_500", row)
    _check_one_step(row)


def test_config3_batch_results_against_fp64():
    """The exploitability and root cfvalues a batch reports, against the FP64
    oracle evaluated from the same final state (the batch's regrets and
    strategy sums copied into it)."""
    n = 48
    sp = spots.datagen_spots(n, seed=7)  # the first spots of the bench's workload
    bs = ps.BatchSolver([spots.card_config(r, b) for r, b, _ in sp], [t for _, _, t in sp])
    targets = np.array([0.003 * t.starting_pot for _, _, t in sp], np.float32)
    bs.solve(300, targets)
    expl, iters = bs.results()

    def one(i):
        r, b, t = sp[i]
        o = spots.oracle_game(r, b, t, fp64=True)
        for k in range(o.num_nodes()):
            if not o.node_info(k)["player"] & (4 | 8):
                o.seed_node_storage(k, 1, bs.node_storage(i, k, 1))
                o.seed_node_storage(k, 2, bs.node_storage(i, k, 2))
        e64 = o.compute_exploitability()
        cfv = [float(np.abs(bs.root_cfvalues(i, p) - o.root_cfvalues(p)).max()
                     / max(np.abs(o.root_cfvalues(p)).max(), 1e-30)) for p in range(2)]
        return {"spot": i, "iterations": int(iters[i]), "expl_gpu": float(expl[i]), "expl_fp64": e64,
                "expl_abs": abs(float(expl[i]) - e64),
                "expl_rel": abs(float(expl[i]) - e64) / max(abs(e64), 1e-3 * t.starting_pot, TOL_EVAL_ULPS * float(
                    np.spacing(np.float32(0.5 * t.starting_pot))) / TOL_EVAL_REL),
                "root_cfv_rel": max(cfv), "solved": bool(expl[i] <= targets[i])}

    with ThreadPoolExecutor(os.cpu_count() or 1) as ex:
        rows = list(ex.map(one, range(n)))
    summary = {"spots": n, "max_expl_rel_vs_fp64": max(x["expl_rel"] for x in rows),
               "max_root_cfv_rel_vs_fp64": max(x["root_cfv_rel"] for x in rows),
               "all_solved": all(x["solved"] for x in rows), "rows": rows}
    _report("config3_batch_vs_fp64", summary)
    assert summary["all_solved"]
    assert summary["max_expl_rel_vs_fp64"] <= TOL_EVAL_REL, summary
    assert summary["max_root_cfv_rel_vs_fp64"] <= TOL_CFV_REL, summary


def test_config4_adjoint_spec_size():
    """256 depth-limited turn trees, boundary values ~N(0, (pot/4)^2), the
    strategy frozen after 200 iterations, the batched adjoint of
    L = sum_p cot_p . cfv_p against FP64 central differences on 512 random
    coordinates per tree: 128 each of the two players' weights and boundary
    values."""
    n, iters, per_block = 256, 200, 128
    sp = spots.turn_boundary_spots(n, seed=31)
    bs = ps.BatchSolver([spots.card_config(r, b) for r, b, _ in sp], [t for _, _, t in sp])
    rng = np.random.default_rng(32)
    V = spots.boundary_values(rng, bs)
    bs.set_boundary_cfvs(V)
    bs.run_iterations(0, iters)
    cot = rng.normal(0, 1, (n, 2, 1326)).astype(np.float32)
    dw, dB = bs.adjoint(cot)
    items = bs.boundary_items()
    first_item = np.searchsorted(items["spot"], np.arange(n))

    def one(i):
        r, b, t = sp[i]
        o = spots.oracle_game(r, b, t, fp64=True)
        idx = [[ps.card_pair_to_index(int(x), int(y)) for x, y in o.private_cards(p)] for p in range(2)]
        nb = o.num_boundary_nodes()
        for k in range(nb):
            for p in range(2):
                o.set_boundary_cfvs(k, p, np.ascontiguousarray(V[first_item[i] + k, p, idx[p]]))
        for k in range(o.num_nodes()):
            if not o.node_info(k)["player"] & (4 | 8):
                o.seed_node_storage(k, 1, bs.node_storage(i, k, 1))
        w = [o.initial_weights(p).astype(np.float32) for p in range(2)]
        g = [np.ascontiguousarray(cot[i, p, idx[p]]) for p in range(2)]
        lr = np.random.default_rng(1000 + i)
        coords, got, block = [], [], []
        for p in range(2):
            H = len(idx[p])
            for j in lr.choice(H, min(per_block, H), replace=False):
                coords.append((0, 0, p, int(j)))
                got.append(dw[i, p, idx[p][j]])
                block.append(p)
            for _ in range(per_block):
                k, j = int(lr.integers(nb)), int(lr.integers(H))
                coords.append((1, k, p, j))
                got.append(dB[first_item[i] + k, p, idx[p][j]])
                block.append(2 + p)
        fd = o.fd_central(w, g, coords, h=1e-3)
        got, block = np.asarray(got, np.float64), np.asarray(block)
        rel = np.zeros(len(fd))
        raw = np.zeros(len(fd))
        floored = 0
        blocks = {}
        for q in range(4):
            m = block == q
            if not m.any():
                continue
            bmax = np.abs(fd[m]).max()
            floor = GRAD_FLOOR * bmax
            rel[m] = np.abs(got[m] - fd[m]) / np.maximum(np.abs(fd[m]), max(floor, 1e-300))
            raw[m] = np.abs(got[m] - fd[m]) / np.maximum(np.abs(fd[m]), 1e-300)
            floored += int(np.sum(np.abs(fd[m]) < floor))
            worst = int(np.argmax(rel[m]))
            blocks[("dw0", "dw1", "dB0", "dB1")[q]] = {
                "max_rel": float(rel[m].max()), "abs_err_over_block_max": float(np.abs(got[m] - fd[m]).max() / bmax),
                "worst_fd_over_block_max": float(np.abs(fd[m][worst]) / bmax), "over_1e-4": int(np.sum(rel[m] > 1e-4))}
        return {"spot": i, "coords": len(fd), "max_rel": float(rel.max()), "median_rel": float(np.median(rel)),
                "max_rel_unfloored_nonzero": float(raw[np.abs(fd) > 0].max()) if np.any(np.abs(fd) > 0) else 0.0,
                "floored": floored, "zero_fd": int(np.sum(fd == 0)), "blocks": blocks}

    with ThreadPoolExecutor(os.cpu_count() or 1) as ex:
        rows = list(ex.map(one, range(n)))
    summary = {"trees": n, "iterations": iters, "coords_per_tree": 4 * per_block,
               "coords_total": int(sum(x["coords"] for x in rows)),
               "worst_rel": max(x["max_rel"] for x in rows),
               "median_rel": float(np.median([x["median_rel"] for x in rows])),
               "worst_rel_unfloored": max(x["max_rel_unfloored_nonzero"] for x in rows),
               "coords_under_floor": int(sum(x["floored"] for x in rows)),
               "rows": rows}
    _report("config4_adjoint_vs_fp64_fd", summary)
    assert summary["worst_rel"] <= TOL_GRAD_REL, {k: v for k, v in summary.items() if k != "rows"}
