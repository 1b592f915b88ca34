"""ORACLE — test infrastructure only.

numpy restatements of the boundary-network input/output steps of the
reference's GPU turn datagen (crates/cfvnet):

- ``zero_conflicting_hands``: datagen/gpu_boundary_eval.rs:35-47;
- ``encode_rows``: the input rows of every (item, player, river card),
  eval/boundary_evaluator.rs:27-60 for one row, rows ordered as
  datagen/gpu_boundary_eval.rs:164-185;
- ``river_reduce``: the reach-weighted average over the 48 river cards with
  card blocking, datagen/gpu_boundary_eval.rs:146-161 (weights) and :207-269
  (reduction), in f64.

Only ``tests/`` may import this module, as the checker of the device kernels.
"""

from __future__ import annotations

import numpy as np

NUM_COMBOS = 1326
INPUT_SIZE = 2 * NUM_COMBOS + 52 + 13 + 3  # network.rs:21
POT_INDEX = 2 * NUM_COMBOS + 52 + 13  # network.rs:24


def combo_pairs() -> np.ndarray:
    """[1326, 2] cards (c1 < c2) of each combo index, card.rs:50-55 order."""
    out = np.zeros((NUM_COMBOS, 2), np.int32)
    k = 0
    for c1 in range(52):
        for c2 in range(c1 + 1, 52):
            out[k] = (c1, c2)
            k += 1
    return out


_PAIRS = combo_pairs()


def card_pair_to_index(c1: int, c2: int) -> int:
    """card.rs:50-55."""
    a, b = min(c1, c2), max(c1, c2)
    return a * (101 - a) // 2 + b - 1


def zero_conflicting_hands(reach: np.ndarray, card: int) -> np.ndarray:
    """Copy of a [1326] reach row with every combo holding `card` set to 0."""
    r = np.array(reach, np.float32, copy=True)
    r[(_PAIRS[:, 0] == card) | (_PAIRS[:, 1] == card)] = 0.0
    return r


def encode_row(oop: np.ndarray, ip: np.ndarray, board, pot: float, stack: float, player: int) -> np.ndarray:
    """One input row (boundary_evaluator.rs:27-60), f32 arithmetic throughout."""
    pot, stack = np.float32(pot), np.float32(stack)
    total = np.float32(pot + stack)
    norm = total if total > np.float32(0) else np.float32(1)
    row = np.zeros(INPUT_SIZE, np.float32)
    row[:NUM_COMBOS] = oop
    row[NUM_COMBOS:2 * NUM_COMBOS] = ip
    for c in board:
        row[2 * NUM_COMBOS + c] = 1.0
        row[2 * NUM_COMBOS + 52 + c // 4] = 1.0
    row[POT_INDEX] = np.float32(pot / norm)
    row[POT_INDEX + 1] = np.float32(stack / norm)
    row[POT_INDEX + 2] = np.float32(player)
    return row


def encode_rows(boards, pots, stacks, reach) -> np.ndarray:
    """Rows for n items: [n, 2 (player), 48 (river), 2720]; reach [n, 2, 1326]
    holds (OOP, IP) reach at the item's boundary."""
    boards = np.asarray(boards).reshape(-1, 4)
    n = boards.shape[0]
    out = np.zeros((n, 2, 48, INPUT_SIZE), np.float32)
    for i in range(n):
        board = [int(c) for c in boards[i]]
        rivers = [c for c in range(52) if c not in board]
        for p in range(2):
            for ri, rv in enumerate(rivers):
                oop = zero_conflicting_hands(reach[i, 0], rv)
                ip = zero_conflicting_hands(reach[i, 1], rv)
                out[i, p, ri] = encode_row(oop, ip, board + [rv], pots[i], stacks[i], p)
    return out


def river_reduce(boards, pots, stacks, net, reach, hands) -> np.ndarray:
    """[n, 2, H]: per item and player, the opponent-reach-weighted average of
    the network outputs over the rivers that do not touch the hand, times
    pot + stack (player 0 weighted by IP reach, player 1 by OOP reach)."""
    boards = np.asarray(boards).reshape(-1, 4)
    n = boards.shape[0]
    hands = np.asarray(hands)
    out = np.zeros((n, 2, len(hands)))
    for i in range(n):
        rivers = [c for c in range(52) if c not in set(int(x) for x in boards[i])]
        denorm = float(np.float32(np.float32(pots[i]) + np.float32(stacks[i])))
        for p in range(2):
            opp = reach[i, 1 - p].astype(np.float64)
            w = np.array([opp[~((_PAIRS[:, 0] == rv) | (_PAIRS[:, 1] == rv))].sum() for rv in rivers])
            for hi, combo in enumerate(hands):
                c0, c1 = _PAIRS[combo]
                keep = np.array([rv not in (c0, c1) for rv in rivers])
                num = float(np.dot(w[keep], net[i, p, keep, combo].astype(np.float64)))
                den = float(w[keep].sum())
                out[i, p, hi] = num / den * denorm if den > 0 else 0.0
    return out.astype(np.float32)
