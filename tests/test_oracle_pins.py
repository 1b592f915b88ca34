"""The oracle (CPU restatement of crates/range-solver) against the reference's
own known answers and golden values (tests/golden/reference_pins.json)."""

import hashlib
import os
import struct

import numpy as np
import pytest

from oracle import oracle as O
from tests import spots

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_hand_table_digest(pins):
    t = O.hand_table()
    p = pins["hand_table"]
    assert len(t) == p["len"] == 4824
    raw = b"".join(struct.pack("<i", int(v)) for v in t)
    assert hashlib.sha256(raw).hexdigest() == p["sha256_le_i32"]
    assert list(t[:5]) == p["first"] and list(t[-3:]) == p["last"]


def test_hand_category_counts(pins):
    # written by the oracle build from the exhaustive C(52,7) enumeration
    with open(os.path.join(ROOT, "oracle", "_build", "hand_counts.txt")) as f:
        vals = [int(x) for x in f.read().split()]
    assert vals[0] == 4824
    assert vals[1:] == pins["hand_category_counts"]["counts"]


def test_hand_ordering_known_answers():
    # hand.rs:168-385 style orderings: royal flush > quads > full house > ... > high card
    def c(r, s):
        return 4 * r + s
    royal = [c(12, 0), c(11, 0), c(10, 0), c(9, 0), c(8, 0), c(0, 1), c(1, 2)]
    quads = [c(5, 0), c(5, 1), c(5, 2), c(5, 3), c(12, 0), c(0, 1), c(1, 2)]
    boat = [c(5, 0), c(5, 1), c(5, 2), c(7, 3), c(7, 0), c(0, 1), c(1, 2)]
    wheel = [c(12, 0), c(0, 1), c(1, 2), c(2, 3), c(3, 0), c(8, 1), c(9, 2)]
    six_high = [c(4, 0), c(0, 1), c(1, 2), c(2, 3), c(3, 0), c(8, 1), c(9, 3)]
    high = [c(12, 0), c(10, 1), c(8, 2), c(6, 3), c(4, 0), c(2, 1), c(0, 2)]
    v = [O.hand_evaluate(x) for x in (royal, quads, boat, six_high, wheel, high)]
    assert v == sorted(v, reverse=True) and len(set(v)) == 6


def test_discount_params(pins):
    p = pins["discount_params"]
    a, b, g = O.discount_params(0)
    assert (a, b, g) == (p["t0"]["alpha"], p["t0"]["beta"], p["t0"]["gamma"])
    a, b, _ = O.discount_params(1)
    assert (a, b) == (p["t1"]["alpha"], p["t1"]["beta"])
    assert O.discount_params(4)[2] == p["t4_gamma"]
    assert abs(O.discount_params(5)[2] - p["t5_gamma"]) < 1e-6
    assert O.discount_params(100)[0] > p["t100_alpha_gt"]


def _expected(kind, args):
    f = [float(x.replace("f64::INFINITY", "inf")) for x in args] if args else []
    if kind in ("PotRelative", "PrevBetRelative"):
        return (kind, f[0], 0, 0)
    if kind == "Additive":
        return (kind, 0.0, int(f[0]), int(f[1]))
    if kind == "Geometric":
        return (kind, f[1], int(f[0]), 0)
    return (kind, 0.0, 0, 0)


def test_bet_size_parser(pins):
    for s, kind, args in pins["bet_size_from_str"]["ok"]:
        got = O.parse_bet_sizes(s, True)
        assert got == [_expected(kind, args)], s
    for s in pins["bet_size_from_str"]["errors"]:
        if s == "":
            continue  # an empty list is valid for the list parser
        with pytest.raises(ValueError):
            O.parse_bet_sizes(s, True)


def _basic_config(pins):
    import poker_solver_rust_b200 as ps
    from poker_solver_rust_b200 import BetSizeOptions as B, BoardState, TreeConfig

    e = pins["basic_example"]
    r0 = ps.Range.from_str(e["oop_range"]).raw_data()
    r1 = ps.Range.from_str(e["ip_range"]).raw_data()
    board = ps.flop_from_str(e["flop"]) + [ps.card_from_str(e["turn"])]
    sz = B(*e["bet_sizes"])
    tc = TreeConfig(initial_state=BoardState.Turn, starting_pot=e["starting_pot"],
                    effective_stack=e["effective_stack"], flop_bet_sizes=[sz, sz], turn_bet_sizes=[sz, sz],
                    river_bet_sizes=[sz, sz], river_donk_sizes=e["river_donk"],
                    add_allin_threshold=e["add_allin_threshold"],
                    force_allin_threshold=e["force_allin_threshold"], merging_threshold=e["merging_threshold"])
    return [r0, r1], board, tc


def _fmt(actions):
    return "[" + ", ".join(k if k in ("Fold", "Check", "Call") else f"{k}({a})" for k, a in actions) + "]"


def test_basic_example_oracle(pins):
    import poker_solver_rust_b200 as ps

    e = pins["basic_example"]
    r, board, tc = _basic_config(pins)
    g = spots.oracle_game(r, board, tc, allocate=False)
    assert ps.holes_to_strings(g.private_cards(0))[:10] == e["oop_first10"]
    assert g.num_private_hands(1) == e["ip_hands"]
    assert _fmt(g.available_actions()) == e["root_actions"]
    # navigate to the node after Bet(120) through the arena
    info = g.node_info(0)
    child = info["children_offset"] + 1
    ci = g.node_info(child)
    kids = [g.node_info(child + ci["children_offset"] + k) for k in range(ci["num_children"])]
    acts = [(O.ACTION_NAMES[k["prev_kind"]], k["prev_amount"]) for k in kids]
    assert _fmt(acts) == e["after_bet_actions"]


def test_oracle_solves_reference_fixture():
    # solver.rs:772-806: AA,KK,QQ,AKs vs QQ-JJ,AQs,AJs on Qs Jh 2c 8d 3s,
    # pot 100 / stack 100, "50%, a"; exploitability < 10 after 100 iterations
    import poker_solver_rust_b200 as ps
    from poker_solver_rust_b200 import BetSizeOptions as B, BoardState, TreeConfig

    r = [ps.Range.from_str("AA,KK,QQ,AKs").raw_data(), ps.Range.from_str("QQ-JJ,AQs,AJs").raw_data()]
    board = ps.flop_from_str("Qs Jh 2c") + [ps.card_from_str("8d"), ps.card_from_str("3s")]
    s = B("50%, a", "")
    tc = TreeConfig(initial_state=BoardState.River, starting_pot=100, effective_stack=100, river_bet_sizes=[s, s])
    g = spots.oracle_game(r, board, tc)
    e = g.solve(100, 0.0)
    assert 0.0 <= e < 10.0


def test_oracle_fp32_tracks_fp64():
    r, board, tc = spots.river_spot(11)
    g32 = spots.oracle_game(r, board, tc)
    g64 = spots.oracle_game(r, board, tc, fp64=True)
    for t in range(50):
        g32.solve_step(t)
        g64.solve_step(t)
    e32, e64 = g32.compute_exploitability(), g64.compute_exploitability()
    assert abs(e32 - e64) <= 1e-3 * max(1.0, abs(e64))


def test_oracle_evaluation_properties():
    # evaluation.rs:706-885: fold values signed by who folded; zero reach -> zero values
    r, board, tc = spots.river_spot(3)
    g = spots.oracle_game(r, board, tc)
    n = g.num_nodes()
    for idx in range(n):
        info = g.node_info(idx)
        if info["player"] & 24 == 24:  # fold terminal
            folded = info["player"] & 3
            for p in range(2):
                v = g.evaluate_node(idx, p, np.ones(g.num_private_hands(p ^ 1), np.float32))
                assert (v >= 0).all() if folded != p else (v <= 0).all()
                z = g.evaluate_node(idx, p, np.zeros(g.num_private_hands(p ^ 1), np.float32))
                assert (z == 0).all()


# ---- known answers of the reference's own unit tests (restated here) ----

def test_card_known_answers():
    # card.rs:418-490 (encoding, pair index round trip, strings, flop parser)
    import poker_solver_rust_b200 as ps

    assert ps.card_from_str("2c") == 0 and ps.card_from_str("As") == 51
    assert ps.card_to_string(0) == "2c" and ps.card_to_string(51) == "As"
    assert [ps.card_to_string(c) for c in (5, 10)] == ["3d", "4h"]
    with pytest.raises(ValueError):
        ps.card_to_string(52)
    k = 0
    for i in range(52):
        for j in range(i + 1, 52):
            assert ps.card_pair_to_index(i, j) == k == ps.card_pair_to_index(j, i)
            assert tuple(ps.index_to_card_pair(k)) == (i, j)
            k += 1
    assert k == 1326
    assert ps.hole_to_string((0, 5)) == "3d2c" and ps.hole_to_string((10, 51)) == "As4h"
    assert ps.holes_to_strings([(0, 5), (10, 51)]) == ["3d2c", "As4h"]
    assert list(ps.flop_from_str("2c3d4h")) == [0, 5, 10]
    assert list(ps.flop_from_str("As Ah Ks")) == [47, 50, 51]
    for bad in ("2c3d4h5s", "2c2c3d"):
        with pytest.raises(ValueError):
            ps.flop_from_str(bad)


def test_compute_average_known_answers():
    # utility.rs:1054-1064
    import poker_solver_rust_b200 as ps

    assert ps.compute_average([1.0, 2.0, 3.0], [1.0, 1.0, 1.0]) == pytest.approx(2.0, abs=1e-6)
    assert ps.compute_average([1.0, 2.0, 3.0], [0.0, 0.0, 1.0]) == pytest.approx(3.0, abs=1e-6)


def _fixture_oracle():
    import poker_solver_rust_b200 as ps
    from poker_solver_rust_b200 import BetSizeOptions as B, BoardState, TreeConfig

    r = [ps.Range.from_str("AA,KK,QQ,AKs").raw_data(), ps.Range.from_str("QQ-JJ,AQs,AJs").raw_data()]
    board = ps.flop_from_str("Qs Jh 2c") + [ps.card_from_str("8d"), ps.card_from_str("3s")]
    s = B("50%, a", "")
    tc = TreeConfig(initial_state=BoardState.River, starting_pot=100, effective_stack=100, river_bet_sizes=[s, s])
    return r, board, tc


def _decision_node(g, actions, player):
    for i in range(g.num_nodes()):
        info = g.node_info(i)
        if not info["player"] & (4 | 8) and info["num_children"] == actions and info["player"] == player:
            return i
    raise AssertionError("no such node")


# (regrets per action-major row pattern, actions, expected strategy) of
# solver.rs:724-750; the pattern covers two hands and is tiled over the node's hands
REGRET_CASES = [
    ([-1.0, -2.0, -3.0, -1.0, -2.0, -3.0], 3, None),  # all negative -> uniform
    ([1.0, 0.0, 0.0, 3.0], 2, [1.0, 0.0, 0.0, 1.0]),
    ([2.0, 2.0, 1.0, 1.0], 2, [2.0 / 3.0, 2.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0]),
]


def _tile(pattern, actions, hands):
    per = len(pattern) // actions  # hands covered by the pattern
    rows = np.asarray(pattern, np.float32).reshape(actions, per)
    return np.concatenate([np.resize(rows[a], hands) for a in range(actions)]).astype(np.float32)


@pytest.mark.parametrize("case", range(len(REGRET_CASES)))
def test_oracle_regret_matching_known_answers(case):
    # one pass at t = 0 (gamma_0 = 0) leaves the strategy sum equal to the
    # regret-matched strategy of the seeded regrets
    pattern, na, expected = REGRET_CASES[case]
    r, board, tc = _fixture_oracle()
    g = spots.oracle_game(r, board, tc)
    idx = _decision_node(g, na, 0)
    H = g.num_private_hands(0)
    g.seed_node_storage(idx, 2, _tile(pattern, na, H))
    g.solve_pass(0, 0)
    got = g.node_storage(idx, 1)
    want = np.full(na * H, 1.0 / na) if expected is None else _tile(expected, na, H)
    assert np.abs(got - want).max() < 1e-6


def test_oracle_normalized_strategy_known_answers():
    # utility.rs:1012-1036: zero sums -> uniform; [1, 3 | 3, 1] -> [.25, .75 | .75, .25]
    r, board, tc = _fixture_oracle()
    g = spots.oracle_game(r, board, tc)
    idx = _decision_node(g, 2, 1)
    H = g.num_private_hands(1)
    g.seed_node_storage(idx, 1, np.zeros(2 * H, np.float32))
    assert np.abs(g.strategy_at_index(idx) - 0.5).max() < 1e-6
    g.seed_node_storage(idx, 1, _tile([1.0, 3.0, 3.0, 1.0], 2, H))
    assert np.abs(g.strategy_at_index(idx) - _tile([0.25, 0.75, 0.75, 0.25], 2, H)).max() < 1e-6


def test_oracle_early_termination():
    # solver.rs:808-838: a target above the starting exploitability stops before any iteration
    r, board, tc = _fixture_oracle()
    g = spots.oracle_game(r, board, tc)
    e = g.solve(1000, 1e10)
    assert e >= 0.0 and g.iterations_run == 0


def test_boundary_io_known_answers():
    """The boundary-network I/O restatement against the reference's own unit
    tests: gpu_boundary_eval.rs:296-337 (zero_conflicting_hands) and
    boundary_evaluator.rs:664-678 (encode_boundary_input_from_ranges), plus the
    reduction's defining property: a network that outputs the same value for
    every row averages to that value times pot + stack."""
    from oracle import boundary_io as bio

    r = bio.zero_conflicting_hands(np.ones(1326, np.float32), 10)
    assert int((r == 0).sum()) == 51
    for c1 in range(52):
        for c2 in range(c1 + 1, 52):
            assert r[bio.card_pair_to_index(c1, c2)] == (0.0 if 10 in (c1, c2) else 1.0)
    r = bio.zero_conflicting_hands(np.full(1326, 0.5, np.float32), 0)
    assert r[bio.card_pair_to_index(1, 2)] == 0.5 and r[bio.card_pair_to_index(0, 1)] == 0.0
    row = bio.encode_row(np.full(1326, 0.5, np.float32), np.full(1326, 0.5, np.float32), [0, 4, 8, 12, 16],
                         100.0, 150.0, 0)
    assert row.shape == (2720,) and bio.POT_INDEX == 2717
    assert abs(row[bio.POT_INDEX] - 0.4) < 1e-6 and abs(row[bio.POT_INDEX + 1] - 0.6) < 1e-6
    assert row[2652:2704].sum() == 5 and row[2704:2717].sum() == 5  # five cards of five ranks
    rng = np.random.default_rng(4)
    boards = np.array([[48, 42, 33, 24]], np.uint8)
    reach = rng.random((1, 2, 1326)).astype(np.float32)
    net = np.full((1, 2, 48, 1326), 0.25, np.float32)
    hands = np.arange(0, 1326, 97)
    out = bio.river_reduce(boards, [100.0], [200.0], net, reach, hands)
    assert np.allclose(out, 0.25 * 300.0, rtol=1e-6)


def test_record_format_pins(tmp_path):
    """The record layout against the reference's storage tests
    (storage.rs:151-230: sizes, round trips, 4-card boards) and the writer's
    per-file rotation (writer.rs:30-83)."""
    from poker_solver_rust_b200 import records as R

    assert R.record_size(5) == 1 + 5 + 4 + 4 + 1 + 4 + 1326 * 4 * 3 + 1326 == 17257
    for bs in (3, 4, 5):
        assert R.record_dtype(bs).itemsize == R.record_size(bs)
    rng = np.random.default_rng(0)
    recs = np.zeros(5, R.record_dtype(4))
    recs["board_size"] = 4
    recs["board"] = [0, 4, 8, 12]
    recs["pot"] = rng.uniform(10, 200, 5).astype(np.float32)
    recs["player"] = [0, 1, 0, 1, 0]
    recs["game_value"] = -0.1
    recs["cfvs"] = rng.normal(0, 1, (5, 1326)).astype(np.float32)
    recs["valid_mask"] = rng.random((5, 1326)) < 0.5
    path = str(tmp_path / "data.bin")
    with R.RecordWriter(path, per_file=2) as w:
        w.write(recs[:3])
        w.write(recs[3:])
        assert w.count() == 5
    names = sorted(p.name for p in tmp_path.iterdir())
    assert names == ["data.bin", "data_00001.bin", "data_00002.bin"]
    back = np.concatenate([R.read_records(str(tmp_path / n), 4) for n in names])
    assert back.tobytes() == recs.tobytes()
    raw = open(path, "rb").read()
    assert raw[0] == 4 and list(raw[1:5]) == [0, 4, 8, 12]
    assert np.frombuffer(raw[5:9], "<f4")[0] == recs["pot"][0]
    assert len(raw) == 2 * R.record_size(4)


def test_sampler_restatement_pins():
    """The situation sampler's restatement against the reference's own tests:
    the 7-card value encoding orders hands as range-solver's evaluator does
    and gives the codes range_gen.rs:184-268 defines; R(S,p) ranges sum to 1,
    are non-negative, zero on the board and heavier on strong hands
    (range_gen.rs:330-438); boards, pots, stacks and SPR buckets keep their
    bounds (sampler.rs:240-420)."""
    from oracle import sampler as S

    def c(r, s):
        return 4 * r + s

    assert S.eval7([c(12, 0), c(0, 1), c(1, 2), c(2, 3), c(3, 0), c(8, 1), c(9, 2)]) == (4 << 26) | (1 << 3)
    assert S.eval7([c(12, 0), c(11, 0), c(10, 0), c(9, 0), c(8, 0), c(0, 1), c(1, 2)]) == (8 << 26) | (1 << 12)
    rng = np.random.default_rng(5)
    for _ in range(1500):
        cards = rng.choice(52, 9, replace=False)
        a = [int(x) for x in cards[:7]]
        b = [int(x) for x in cards[2:9]]
        ea, eb = S.eval7(a), S.eval7(b)
        oa, ob = O.hand_evaluate(a), O.hand_evaluate(b)
        assert np.sign(ea - eb) == np.sign(oa - ob), (a, b)
    board = [c(10, 3), c(9, 2), c(0, 0), c(6, 1), c(1, 3)]  # Qs Jh 2c 8d 3s
    vals = S.hand_values(board)
    blocked = np.array([bool(set(p) & set(board)) for p in S.PAIRS])
    assert (vals[blocked] == 0).all() and (vals[~blocked] > 0).all()
    order = sorted(np.nonzero(~blocked)[0], key=lambda i: (vals[i], i))
    top, bottom = order[len(order) * 3 // 4:], order[:len(order) // 4]
    ts = bs = 0.0
    for seed in range(60):
        r = S.rsp_range(vals, S.mix64(seed), 0)
        assert abs(float(r.sum()) - 1.0) < 1e-5 and (r >= 0).all() and not r[blocked].any()
        ts += float(r[top].sum())
        bs += float(r[bottom].sum())
    assert ts > bs
    assert np.array_equal(S.rsp_range(vals, 77, 1), S.rsp_range(vals, 77, 1))
    v4 = S.hand_values(board[:4])
    r4 = S.rsp_range(v4, 123, 0)
    assert abs(float(r4.sum()) - 1.0) < 1e-5
    pots = [[4, 20], [20, 80], [80, 200], [200, 400]]
    for i in range(800):
        b, pot, stack, _ = S.sample_board_pot(5, 200, pots, None, 42, i)
        assert len(set(b)) == 5 and max(b) < 52
        assert any(lo <= pot < hi for lo, hi in pots)
        max_stack = 200 - pot // 2
        assert stack == 5 if max_stack < 5 else 5 <= stack <= max_stack
    sprs = [[0.0, 1.0], [1.0, 3.0], [3.0, 8.0]]
    seen = set()
    for i in range(600):
        got = S.sample_board_pot(4, 400, [[4, 40], [40, 120], [120, 400]], sprs, 7, i)
        assert got is not None
        _, pot, stack, _ = got
        k = [j for j, (lo, hi) in enumerate(sprs) if lo <= stack / pot < hi]
        assert len(k) == 1 and stack >= 5
        seen.add(k[0])
    assert seen == {0, 1, 2}


def test_oracle_chance_threads_keep_results():
    """The oracle's parallel chance children (the reference's rayon split,
    solver.rs:264-326) give the same state as the sequential walk."""
    r, b, t = spots.turn_spot(4)
    out = []
    for threads in (1, 4):
        O.set_chance_threads(threads)
        try:
            o = spots.oracle_game(r, b, t)
            for it in range(2):
                o.solve_step(it)
            out.append((o.compute_exploitability(), o.root_cfvalues(0)))
        finally:
            O.set_chance_threads(1)
    assert out[0][0] == out[1][0] and np.array_equal(out[0][1], out[1][1])


def test_oracle_fd_central_matches_python_differences():
    """The oracle's C++ central differences (used at the spec's adjoint size)
    equal the loop over full loss evaluations that the small adjoint test
    runs: weights and boundary values of a depth-limited turn spot."""
    import numpy as np

    from tests import spots

    rng = np.random.default_rng(3)

    def sparse(rng, board):
        out = []
        for _ in range(2):
            w = rng.random(1326).astype(np.float32)
            w[rng.random(1326) < 0.93] = 0.0
            out.append(spots._mask_board(w, board))
        return out

    r, b, t = spots.turn_spot(9, weights=sparse)
    t.depth_limit = 0
    o = spots.oracle_game(r, b, t, fp64=True)
    nb = o.num_boundary_nodes()
    assert nb > 0
    B = [[rng.normal(0, 1, o.num_private_hands(p)).astype(np.float32) for p in range(2)] for _ in range(nb)]
    for k in range(nb):
        for p in range(2):
            o.set_boundary_cfvs(k, p, B[k][p])
    for it in range(8):
        o.solve_step(it)
    H = [o.num_private_hands(0), o.num_private_hands(1)]
    w = [rng.random(H[p]).astype(np.float32) for p in range(2)]
    cot = [rng.normal(0, 1, H[p]).astype(np.float32) for p in range(2)]

    def loss():
        c0 = o.root_cfvalues_with_reach(0, w[1])
        c1 = o.root_cfvalues_with_reach(1, w[0])
        return float(np.dot(cot[0].astype(np.float64), c0) + np.dot(cot[1].astype(np.float64), c1))

    coords, ref = [], []
    for p in range(2):
        for j in rng.choice(H[p], 4, replace=False):
            x0 = w[p][j]
            w[p][j] = np.float32(x0 + 1e-3)
            lp, xp = loss(), float(w[p][j])
            w[p][j] = np.float32(x0 - 1e-3)
            lm, xm = loss(), float(w[p][j])
            w[p][j] = x0
            coords.append((0, 0, p, j))
            ref.append((lp - lm) / (xp - xm))
        for _ in range(4):
            k, j = int(rng.integers(nb)), int(rng.integers(H[p]))
            v = B[k][p].copy()
            v[j] = np.float32(B[k][p][j] + 1e-3)
            o.set_boundary_cfvs(k, p, v)
            lp, xp = loss(), float(v[j])
            v[j] = np.float32(B[k][p][j] - 1e-3)
            o.set_boundary_cfvs(k, p, v)
            lm, xm = loss(), float(v[j])
            o.set_boundary_cfvs(k, p, B[k][p])
            coords.append((1, k, p, j))
            ref.append((lp - lm) / (xp - xm))
    got = o.fd_central(w, cot, coords)
    ref = np.asarray(ref)
    assert np.abs(got - ref).max() <= 1e-9 * max(1.0, np.abs(ref).max()), (got, ref)
