"""ORACLE — test infrastructure only.

Python restatement of the situation sampler: cfvnet datagen/sampler.rs:30-60
(situation), :142-160 (board), :165-205 (pot / stack by SPR bucket), and
datagen/range_gen.rs:18-56 (hand strengths), :120-167 (R(S,p) ranges),
:184-290 (the 7-card value encoding), drawing from the same counter-based
SplitMix64 stream as the device sampler (the reference draws from rand's
ChaCha8, a third-party crate; the distributions are the same, the numbers are
not).  Only ``tests/`` may import this module, as the checker of the device
sampler.
"""

from __future__ import annotations

import math

import numpy as np

M64 = (1 << 64) - 1
GOLDEN = 0x9E3779B97F4A7C15


def mix64(z: int) -> int:
    z &= M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def draw(key: int, ctr: int) -> int:
    return mix64(key + (ctr + 1) * GOLDEN)


def draw_int(key: int, ctr: int, n: int) -> int:
    return ((draw(key, ctr) >> 32) * n) >> 32


def draw_unit(key: int, ctr: int) -> float:
    return float(draw(key, ctr) >> 11) * 2.0 ** -53


def _top_bits(x: int, n: int) -> int:
    r = 0
    for _ in range(n):
        if not x:
            break
        b = 1 << (x.bit_length() - 1)
        r |= b
        x ^= b
    return r


def _straight_top(ranks: int) -> int:
    run = ranks & (ranks << 1) & (ranks << 2) & (ranks << 3) & (ranks << 4)
    if run:
        return _top_bits(run, 1)
    return 1 << 3 if ranks & 0x100F == 0x100F else 0


def eval7(cards) -> int:
    """Category << 26 | deciding ranks (range_gen.rs:184-268)."""
    allr = 0
    suited = [0, 0, 0, 0]
    cnt = [0] * 13
    for c in cards:
        allr |= 1 << (c >> 2)
        suited[c & 3] |= 1 << (c >> 2)
        cnt[c >> 2] += 1
    by = [0] * 5
    for r in range(13):
        by[cnt[r]] |= 1 << r
    flush = -1
    for s in range(4):
        if bin(suited[s]).count("1") >= 5:
            flush = s
    if flush >= 0:
        sf = _straight_top(suited[flush])
        return (8 << 26) | sf if sf else (5 << 26) | _top_bits(suited[flush], 5)
    if by[4]:
        return (7 << 26) | (by[4] << 13) | _top_bits(allr ^ by[4], 1)
    if bin(by[3]).count("1") == 2:
        t = _top_bits(by[3], 1)
        return (6 << 26) | (t << 13) | (by[3] ^ t)
    if by[3] and by[2]:
        return (6 << 26) | (by[3] << 13) | _top_bits(by[2], 1)
    st = _straight_top(allr)
    if st:
        return (4 << 26) | st
    if by[3]:
        return (3 << 26) | (by[3] << 13) | _top_bits(by[1], 2)
    if bin(by[2]).count("1") >= 2:
        two = _top_bits(by[2], 2)
        return (2 << 26) | (two << 13) | _top_bits(allr ^ two, 1)
    if by[2]:
        return (1 << 26) | (by[2] << 13) | _top_bits(by[1], 3)
    return _top_bits(allr, 5)


PAIRS = [(a, b) for a in range(52) for b in range(a + 1, 52)]


def hand_values(board) -> np.ndarray:
    """range_gen.rs:18-56 before the ordinal step: the value on a 5-card board,
    its mean over the 46 rivers on a 4-card board, 0 for blocked combos."""
    bm = 0
    for c in board:
        bm |= 1 << c
    out = np.zeros(1326)
    for i, (c1, c2) in enumerate(PAIRS):
        hm = (1 << c1) | (1 << c2)
        if hm & bm:
            continue
        if len(board) == 5:
            out[i] = float(eval7([c1, c2, *board]))
        else:
            vals = [eval7([c1, c2, *board, r]) for r in range(52) if not ((bm | hm) >> r) & 1]
            out[i] = float(sum(vals)) / float(len(vals))
    return out


def rsp_range(values, key: int, r: int) -> np.ndarray:
    """R(S,p) over the valid combos in ascending (value, index) order; the
    split of the node covering positions [lo, hi) draws at counter
    ((r + 1) << 32) | lo << 12 | hi."""
    valid = [i for i in range(1326) if values[i] > 0.0]
    order = sorted(valid, key=lambda i: (values[i], i))
    n = len(order)
    out = np.zeros(1326, np.float32)
    for k, c in enumerate(order):
        lo, hi, p = 0, n, 1.0
        while hi - lo > 1 and p > 0.0:
            u = draw_unit(key, ((r + 1) << 32) | (lo << 12) | hi)
            d = u * p
            rem = p - d
            mid = lo + (hi - lo) // 2
            if k >= mid:
                p, lo = max(d, rem), mid
            else:
                p, hi = min(d, rem), mid
        out[c] = np.float32(p) if p > 0.0 else np.float32(0.0)
    return out


def _round_half_away(x: float) -> float:
    f = math.floor(x)
    return f + 1.0 if x - f >= 0.5 else f


def sample_board_pot(board_size, initial_stack, pot_intervals, spr_intervals, seed: int, idx: int):
    """(board, pot, stack, key) of situation idx, or None when the SPR
    rejection gives up."""
    key = mix64(seed + (idx + 1) * GOLDEN)
    used, ctr, board = 0, 0, []
    for _ in range(board_size):
        while True:
            c = draw_int(key, ctr, 52)
            ctr += 1
            if not (used >> c) & 1 or ctr >= 4096:
                break
        if (used >> c) & 1:
            return None
        used |= 1 << c
        board.append(c)
    pc = 1 << 16
    if not spr_intervals:
        lo, hi = pot_intervals[draw_int(key, pc, len(pot_intervals))]
        pot = lo + draw_int(key, pc + 1, hi - lo)
        max_stack = initial_stack - pot // 2
        stack = 5 if max_stack < 5 else 5 + draw_int(key, pc + 2, max_stack - 5 + 1)
    else:
        sf = float(initial_stack)
        pot = stack = None
        for _ in range(10000):
            slo, shi = spr_intervals[draw_int(key, pc, len(spr_intervals))]
            spr = slo + draw_unit(key, pc + 1) * (shi - slo)
            pc += 2
            pmin = math.ceil(5.0 / spr) if spr > 0.0 else math.ceil(2.0 * (sf - 5.0))
            pmax = sf / (spr + 0.5)
            flo, fhi = int(min(max(pmin, 1.0), 1.0e9)), int(pmax)
            if flo > fhi:
                continue
            buckets = [(max(a, flo), min(b, fhi + 1)) for a, b in pot_intervals if max(a, flo) < min(b, fhi + 1)]
            if not buckets:
                continue
            blo, bhi = buckets[draw_int(key, pc, len(buckets))]
            p = blo + draw_int(key, pc + 1, bhi - blo)
            pc += 2
            max_stack = initial_stack - p // 2
            if max_stack < 5:
                continue
            s = min(max(int(min(_round_half_away(spr * p), 2.0e9)), 5), max_stack)
            if slo <= s / p < shi:
                pot, stack = p, s
                break
        if pot is None:
            return None
    return board, pot, stack, key


def sample_situation(board_size, initial_stack, pot_intervals, spr_intervals, seed: int, idx: int):
    """(board [5], pot, stack, ranges [2, 1326]) of situation idx, or None when
    the SPR rejection gives up."""
    got = sample_board_pot(board_size, initial_stack, pot_intervals, spr_intervals, seed, idx)
    if got is None:
        return None
    board, pot, stack, key = got
    values = hand_values(board)
    ranges = np.stack([rsp_range(values, key, r) for r in range(2)])
    return board + [0] * (5 - board_size), pot, stack, ranges
