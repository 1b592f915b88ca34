"""Seeded synthetic spots shared by the tests and bench.py.

Generator: numpy PCG64 (np.random.default_rng(seed)).  The workload shapes
follow the configurations the reference's solver is benchmarked on:
  river_spot      5-card board, weights U[0,1] masked by the board (1081
                  live), pot 100 / stack 200, bets 50% / 100% / all-in,
                  raise 100%, max 3 bets per street;
  turn_spot       4-card board, pot 100 / stack 300, bets 33% / 75% / all-in
                  on turn and river, raise 60%, max 3 bets per street;
  datagen_spots   batched river spots: weights ~Beta(0.5, 0.5) with 30% of
                  the combos zeroed, pot U[20, 200], stack = round(SPR * pot)
                  with SPR ~U[0.5, 10], bet menu drawn from three menus,
                  raise {100%, all-in}; target 0.3% of the pot.
"""

from __future__ import annotations

import numpy as np

import poker_solver_rust_b200 as ps
from poker_solver_rust_b200 import BetSizeOptions as B, BoardState, TreeConfig

DATAGEN_MENUS = ("50%, a", "33%, 75%, a", "25%, 50%, 100%, 150%, a")


def _mask_board(w, board):
    for i in range(1326):
        c1, c2 = ps.index_to_card_pair(i)
        if c1 in board or c2 in board:
            w[i] = 0.0
    return w


def uniform_ranges(rng, board):
    return [_mask_board(rng.random(1326).astype(np.float32), board) for _ in range(2)]


def river_spot(seed: int, max_bets: int = 0):
    rng = np.random.default_rng(seed)
    board = [int(x) for x in rng.choice(52, 5, replace=False)]
    r = uniform_ranges(rng, board)
    sizes = B("50%, 100%, a", "100%")
    tc = TreeConfig(initial_state=BoardState.River, starting_pot=100, effective_stack=200,
                    river_bet_sizes=[sizes, sizes], max_bets=max_bets)
    return r, board, tc


def turn_spot(seed: int, max_bets: int = 0, weights=None):
    rng = np.random.default_rng(seed)
    board = [int(x) for x in rng.choice(52, 4, replace=False)]
    r = uniform_ranges(rng, board) if weights is None else weights(rng, board)
    sizes = B("33%, 75%, a", "60%")
    tc = TreeConfig(initial_state=BoardState.Turn, starting_pot=100, effective_stack=300,
                    turn_bet_sizes=[sizes, sizes], river_bet_sizes=[sizes, sizes], max_bets=max_bets)
    return r, board, tc


def datagen_spot(rng):
    board = [int(x) for x in rng.choice(52, 5, replace=False)]
    r = []
    for _ in range(2):
        w = rng.beta(0.5, 0.5, 1326).astype(np.float32)
        w[rng.random(1326) < 0.3] = 0.0
        r.append(_mask_board(w, board))
    pot = int(rng.integers(20, 201))
    spr = float(rng.uniform(0.5, 10.0))
    stack = max(1, int(round(spr * pot)))
    menu = DATAGEN_MENUS[int(rng.integers(0, 3))]
    sizes = B(menu, "100%, a")
    tc = TreeConfig(initial_state=BoardState.River, starting_pot=pot, effective_stack=stack,
                    river_bet_sizes=[sizes, sizes])
    return r, board, tc


def datagen_spots(n: int, seed: int = 7):
    rng = np.random.default_rng(seed)
    return [datagen_spot(rng) for _ in range(n)]


_PAIRS = None


def _board_blocked(board):
    global _PAIRS
    if _PAIRS is None:
        _PAIRS = np.array([ps.index_to_card_pair(i) for i in range(1326)])
    b = np.asarray(board)
    return np.isin(_PAIRS[:, 0], b) | np.isin(_PAIRS[:, 1], b)


def turn_boundary_spot(rng):
    """Depth-limited turn spot: the turn settings of turn_spot (bets 33% / 75%
    / all-in, raise 60%) with a depth boundary at every non-fold turn
    terminal, and the range / pot / stack distributions of datagen_spot."""
    board = [int(x) for x in rng.choice(52, 4, replace=False)]
    blocked = _board_blocked(board)
    r = []
    for _ in range(2):
        w = rng.beta(0.5, 0.5, 1326).astype(np.float32)
        w[rng.random(1326) < 0.3] = 0.0
        w[blocked] = 0.0
        r.append(w)
    pot = int(rng.integers(20, 201))
    stack = max(1, int(round(float(rng.uniform(0.5, 10.0)) * pot)))
    sizes = B("33%, 75%, a", "60%")
    tc = TreeConfig(initial_state=BoardState.Turn, starting_pot=pot, effective_stack=stack,
                    turn_bet_sizes=[sizes, sizes], river_bet_sizes=[sizes, sizes], depth_limit=0)
    return r, board, tc


def turn_boundary_spots(n: int, seed: int = 11):
    rng = np.random.default_rng(seed)
    return [turn_boundary_spot(rng) for _ in range(n)]


def boundary_values(rng, batch, scale=0.25):
    """Seeded boundary values [items, 2, 1326] ~ N(0, (scale * pot)^2) of a
    batch's boundary items, zero on board-blocked combos."""
    items = batch.boundary_items()
    n = len(items["spot"])
    v = rng.normal(0.0, 1.0, (n, 2, 1326)).astype(np.float32)
    v *= (scale * batch.starting_pots[items["spot"]])[:, None, None]
    for k in range(n):
        v[k, :, _board_blocked(items["boards"][k])] = 0.0
    return v


def card_config(ranges, board):
    turn = board[3] if len(board) > 3 else ps.NOT_DEALT
    river = board[4] if len(board) > 4 else ps.NOT_DEALT
    return ps.CardConfig([ps.Range(ranges[0]), ps.Range(ranges[1])], board[:3], turn, river)


def product_game(ranges, board, tc, allocate=True):
    g = ps.PostFlopGame.with_config(card_config(ranges, board), ps.ActionTree(tc))
    if allocate:
        g.allocate_memory(False)
    return g


def oracle_game(ranges, board, tc, fp64=False, allocate=True):
    from oracle.oracle import OracleGame

    d = tc.to_dict()
    if tc.max_bets:
        raise ValueError("the oracle restates the reference, which has no bet cap")
    g = OracleGame(ranges, board, d, fp64=fp64)
    if allocate:
        g.allocate_memory()
    return g
