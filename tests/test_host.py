"""Host side of the product on CPU: the C-ABI library loads and exports every
symbol of include/ps_range_solver.h; trees, hand lists and host tables match
the oracle exactly; configuration errors behave like the reference."""

import hashlib
import os
import re
import struct

import numpy as np
import pytest

import poker_solver_rust_b200 as ps
from poker_solver_rust_b200 import _native as N
from oracle import oracle as O
from tests import spots
from tests.test_oracle_pins import _basic_config, _expected, _fmt

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_header_symbols():
    with open(os.path.join(ROOT, "include", "ps_range_solver.h")) as f:
        hdr = f.read()
    declared = set(re.findall(r"\b(ps_[a-z0-9_]+)\s*\(", hdr))
    L = N.lib()
    missing = [s for s in sorted(declared) if not hasattr(L, s)]
    assert not missing, missing
    assert declared == set(N.EXPORTED), sorted(declared ^ set(N.EXPORTED))


def test_hand_table_matches_reference(pins):
    t = ps.hand_table()
    raw = b"".join(struct.pack("<i", int(v)) for v in t)
    assert hashlib.sha256(raw).hexdigest() == pins["hand_table"]["sha256_le_i32"]
    assert np.array_equal(t, O.hand_table())


def test_discount_params_bit_exact():
    for t in list(range(0, 2000)) + [4095, 4096, 65535, 65536, 10 ** 6]:
        assert ps.discount_params(t) == O.discount_params(t), t


def test_bet_size_parser(pins):
    for s, kind, args in pins["bet_size_from_str"]["ok"]:
        assert ps.parse_bet_sizes(s, True) == [_expected(kind, args)], s
    for s in pins["bet_size_from_str"]["errors"]:
        if s == "":
            continue
        with pytest.raises(ps.SolverError):
            ps.parse_bet_sizes(s, True)
    assert ps.parse_bet_sizes("50c, e, a,", False) == O.parse_bet_sizes("50c, e, a,", False)
    with pytest.raises(ps.SolverError):
        ps.parse_bet_sizes("2.5x", False)  # bet_size.rs:319: relative sizes only for raises


def test_range_parser_known_answers():
    # range.rs:821-969
    eq = [("88+", "AA,KK,QQ,JJ,TT,99,88"), ("8s8h+", "AhAs,KhKs,QhQs,JhJs,ThTs,9h9s,8h8s"),
          ("98s+", "AKs,KQs,QJs,JTs,T9s,98s"), ("A8o+", "AKo,AQo,AJo,ATo,A9o,A8o"), ("88-55", "88,77,66,55")]
    for a, b in eq:
        assert ps.Range.from_str(a) == ps.Range.from_str(b)
    r = ps.Range.from_str("AA,AKs,AKo")
    assert r.get_weight_pair(12) == 1.0 and r.get_weight_suited(12, 11) == 1.0
    assert r.get_weight_offsuit(12, 11) == 1.0 and r.get_weight_suited(12, 10) == 0.0
    assert abs(ps.Range.from_str("AA:0.5").get_weight_pair(12) - 0.5) < 1e-6
    assert ps.Range.from_str("QQ-99").get_weight_pair(6) == 0.0
    for bad in ("AKQ", "AK+-AJ", "K9s.67", "88+:2.0", "98s-21s"):
        with pytest.raises(ValueError):
            ps.Range.from_str(bad)


def _compare_game(r, board, tc):
    g = spots.product_game(r, board, tc, allocate=False)
    o = spots.oracle_game(r, board, tc, allocate=False)
    assert g.num_nodes() == o.num_nodes()
    for i in range(g.num_nodes()):
        assert g.node_info(i) == o.node_info(i), i
    for p in range(2):
        assert np.array_equal(g.private_cards(p), o.private_cards(p))
        assert np.array_equal(g.initial_weights(p), o.initial_weights(p).astype(np.float32))
        assert np.array_equal(g.same_hand_index(p), o.same_hand_index(p))
    assert abs(g.num_combinations() - o.num_combinations()) <= 1e-12 * o.num_combinations()
    return g, o


@pytest.mark.parametrize("seed", range(6))
def test_river_arena_matches_oracle(seed):
    _compare_game(*spots.river_spot(seed))


@pytest.mark.parametrize("seed", range(12))
def test_datagen_arena_matches_oracle(seed):
    rng = np.random.default_rng(1000 + seed)
    _compare_game(*spots.datagen_spot(rng))


def test_turn_arena_matches_oracle():
    _compare_game(*spots.turn_spot(5))


def test_basic_example_product(pins):
    e = pins["basic_example"]
    r, board, tc = _basic_config(pins)
    g = spots.product_game(r, board, tc, allocate=False)
    assert ps.holes_to_strings(g.private_cards(0))[:10] == e["oop_first10"]
    assert g.num_private_hands(1) == e["ip_hands"]
    assert _fmt(g.available_actions()) == e["root_actions"]
    kids = g.child_indices(g.child_indices(0)[1])
    acts = [(ps.ACTION_NAMES[g.node_info(k)["prev_kind"]], g.node_info(k)["prev_amount"]) for k in kids]
    assert _fmt(acts) == e["after_bet_actions"]
    _compare_game(r, board, tc)


def test_max_bets_extension_is_noop_on_river_config():
    r, board, tc = spots.river_spot(0)
    tc3 = spots.river_spot(0, max_bets=3)[2]
    a = spots.product_game(r, board, tc, allocate=False)
    b = spots.product_game(r, board, tc3, allocate=False)
    assert a.num_nodes() == b.num_nodes()


def test_config_errors():
    r, board, tc = spots.river_spot(1)
    bad = [dict(starting_pot=0), dict(effective_stack=-5), dict(rake_rate=1.5), dict(initial_state=ps.BoardState.Turn)]
    for kw in bad:
        t2 = spots.river_spot(1)[2]
        for k, v in kw.items():
            setattr(t2, k, v)
        with pytest.raises(ps.SolverError) as ei:
            spots.product_game(r, board, t2, allocate=False)
        assert ei.value.code == N.PS_ERR_INVALID
    z = [np.zeros(1326, np.float32), r[1]]
    with pytest.raises(ps.SolverError, match="OOP range is empty"):
        spots.product_game(z, board, tc, allocate=False)
    dup = [board[0], board[0], board[2], board[3], board[4]]
    with pytest.raises(ps.SolverError):
        spots.product_game(r, dup, tc, allocate=False)
    g = spots.product_game(r, board, tc, allocate=False)
    with pytest.raises(ps.SolverError) as ei:
        ps.solve_step(g, 0)  # Game is not ready (solver.rs:114-120)
    assert ei.value.code == N.PS_ERR_STATE
    with pytest.raises(ps.SolverError) as ei:
        g.allocate_memory(True)
    assert ei.value.code == N.PS_ERR_UNSUPPORTED


def test_batch_config_packing_points_at_ranges():
    """The batch's card configs address each range's own float32 weights; a
    range held in another dtype is converted, and a wrong length is refused."""
    import ctypes as C

    from poker_solver_rust_b200 import game as G

    work = spots.datagen_spots(6, seed=3)
    cc = [spots.card_config(r, b) for r, b, _ in work]
    tcs = [t for _, _, t in work]
    cc[2].range[1].data = cc[2].range[1].data.astype(np.float64)  # converted on packing
    a, b, keep = G._pack_configs(cc, tcs)
    for i, c in enumerate(cc):
        for p in range(2):
            got = np.ctypeslib.as_array(C.cast(a[i].range[p], C.POINTER(C.c_float)), (1326,))
            assert np.array_equal(got, np.asarray(c.range[p].data, np.float32))
            if (i, p) != (2, 1):
                assert C.cast(a[i].range[p], C.c_void_p).value == c.range[p].data.ctypes.data
        assert list(a[i].flop) == list(c.flop) and a[i].turn == c.turn and a[i].river == c.river
        t, pt = tcs[i], b[i]
        menus = [s for st in (t.flop_bet_sizes, t.turn_bet_sizes, t.river_bet_sizes)
                 for q in range(2) for s in (st[q].bet, st[q].raise_)]
        assert [None if x is None else x.decode() for x in pt.bet_sizes] == menus
        assert (pt.starting_pot, pt.effective_stack) == (t.starting_pot, t.effective_stack)
        assert pt.initial_state == int(t.initial_state) and pt.max_bets == int(t.max_bets)
        assert (pt.rake_rate, pt.rake_cap) == (float(t.rake_rate), float(t.rake_cap))
    cc[0].range[0].data = np.zeros(100, np.float32)
    with pytest.raises(ValueError):
        G._pack_configs(cc, tcs)


def test_program_forms_pass_slot_replay():
    """Both tree-program forms compile and pass the compiler's slot replay
    (every read finds the vector it expects) on river, turn, depth-limited
    and isomorphic trees; the terminals-first form has one terminal step per
    pass and keeps the op counts."""
    import numpy as np

    from tests import spots

    cases = [spots.river_spot(1), spots.turn_spot(2), spots.datagen_spot(np.random.default_rng(5))]
    r, b, t = spots.turn_spot(9)
    t.depth_limit = 0
    cases.append((r, b, t))
    r0 = ps.Range.from_str("AA,KK,QQ,AKs,AQs,KQo").raw_data()
    r1 = ps.Range.from_str("JJ-99,AJs,KJs,QJs,T9s").raw_data()
    board = ps.board_from_str("Kh Qh 7h 2s")
    sz = ps.BetSizeOptions("50%, a", "100%")
    tc = ps.TreeConfig(initial_state=ps.BoardState.Turn, starting_pot=100, effective_stack=150,
                       turn_bet_sizes=[sz, sz], river_bet_sizes=[sz, sz])
    cases.append(([spots._mask_board(r0.copy(), board), spots._mask_board(r1.copy(), board)], board, tc))
    for r, b, t in cases:
        g = spots.product_game(r, b, t, allocate=False)
        base = g.program_info()
        g.set_terminals_first(True)
        tf = g.program_info()
        assert tf["node_ops"] == base["node_ops"] and tf["terminal_ops"] == base["terminal_ops"]
        assert tf["terminal_runs"] == base["terminal_runs"]
        g.set_terminals_first(False)
        assert g.program_info() == base


def test_autotune_log_stages():
    """The autotune log lists the sweep (each shape once), then the refine
    runs of the leading shapes: the first repeated shape starts the refine
    stage, and the choice is the fastest refine run."""
    from poker_solver_rust_b200.game import autotune_stages

    shapes = [(256, 4, 1, 1), (512, 8, 2, 3), (1024, 16, 3, 3), (512, 8, 2, 3), (1024, 16, 3, 3)]
    ms = [30.0, 20.2, 21.0, 510.0, 505.0]
    log = autotune_stages(shapes, ms)
    assert [r["stage"] for r in log] == ["sweep"] * 3 + ["refine"] * 2
    best = min((r for r in log if r["stage"] == "refine"), key=lambda r: r["trial_ms"])
    assert (best["block_threads"], best["spots_per_cta"], best["node_parts"]) == (1024, 3, 3)
    assert [r["stage"] for r in autotune_stages(shapes[:3], ms[:3])] == ["sweep"] * 3
