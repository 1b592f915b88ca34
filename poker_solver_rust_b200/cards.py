"""Cards, hole-card pairs and ranges (crates/range-solver/src/card.rs, range.rs).

Card id = 4 * rank + suit (rank 2..A -> 0..12, suit c d h s -> 0..3); a range
is the reference's raw data: 1326 weights in ``card_pair_to_index`` order.
"""

from __future__ import annotations

import math
import re

import numpy as np

NOT_DEALT = 255
_RANKS = "23456789TJQKA"
_SUITS = "cdhs"


def card_pair_to_index(c1: int, c2: int) -> int:  # card.rs:50-55
    if c1 > c2:
        c1, c2 = c2, c1
    return c1 * (101 - c1) // 2 + c2 - 1


def index_to_card_pair(index: int):  # card.rs:61-65
    c1 = (103 - math.ceil(math.sqrt(103.0 * 103.0 - 8.0 * index))) // 2
    c2 = index - c1 * (101 - c1) // 2 + 1
    return c1, c2


def _rank(c: str) -> int:
    i = _RANKS.find(c.upper())
    if i < 0:
        raise ValueError(f"Expected rank character: {c}")
    return i


def _suit(c: str) -> int:
    i = _SUITS.find(c)
    if i < 0:
        raise ValueError(f"Expected suit character: {c}")
    return i


def card_from_str(s: str) -> int:  # card.rs:339-348
    if len(s) != 2:
        raise ValueError("Expected exactly two characters")
    return (_rank(s[0]) << 2) | _suit(s[1])


def card_to_string(card: int) -> str:  # card.rs:300-305
    if not 0 <= card < 52:
        raise ValueError(f"Invalid card: {card}")
    return _RANKS[card >> 2] + _SUITS[card & 3]


def hole_to_string(hole) -> str:  # card.rs:311-319
    a, b = max(hole), min(hole)
    return card_to_string(a) + card_to_string(b)


def holes_to_strings(holes):
    return [hole_to_string((int(h[0]), int(h[1]))) for h in holes]


def flop_from_str(s: str):  # card.rs:361-377
    t = s.replace(" ", "")
    if len(t) != 6:
        raise ValueError("Expected exactly three cards")
    cards = sorted(card_from_str(t[i:i + 2]) for i in (0, 2, 4))
    if cards[0] == cards[1] or cards[1] == cards[2]:
        raise ValueError("Cards must be unique")
    return cards


def board_from_str(s: str):
    t = s.replace(" ", "")
    return [card_from_str(t[i:i + 2]) for i in range(0, len(t), 2)]


# ---------------------------------------------------------------------------
# Range strings (range.rs:49-752)
# ---------------------------------------------------------------------------
_COMBO = r"(?:(?:[AaKkQqJjTt2-9]{2}[os]?)|(?:(?:[AaKkQqJjTt2-9][cdhs]){2}))"
_WEIGHT = r"(?:(?:[01](\.\d*)?)|(?:\.\d+))"
_RANGE_RE = re.compile(rf"^(?P<range>{_COMBO}(?:\+|(?:-{_COMBO}))?)(?::(?P<weight>{_WEIGHT}))?$")
_TRIM_RE = re.compile(r"\s*([-:,])\s*")


def _pair_idx(r):
    return [card_pair_to_index(4 * r + i, 4 * r + j) for i in range(4) for j in range(i + 1, 4)]


def _nonpair_idx(r1, r2):
    return [card_pair_to_index(4 * r1 + i, 4 * r2 + j) for i in range(4) for j in range(4)]


def _suited_idx(r1, r2):
    return [card_pair_to_index(4 * r1 + i, 4 * r2 + i) for i in range(4)]


def _offsuit_idx(r1, r2):
    return [card_pair_to_index(4 * r1 + i, 4 * r2 + j) for i in range(4) for j in range(4) if i != j]


def _indices(r1, r2, suited):
    if r1 == r2:
        if suited == "all":
            return _pair_idx(r1)
        if isinstance(suited, tuple):
            return [card_pair_to_index(4 * r1 + suited[0], 4 * r1 + suited[1])]
        raise ValueError("invalid suitedness with a pair")
    if suited == "s":
        return _suited_idx(r1, r2)
    if suited == "o":
        return _offsuit_idx(r1, r2)
    if suited == "all":
        return _nonpair_idx(r1, r2)
    return [card_pair_to_index(4 * r1 + suited[0], 4 * r2 + suited[1])]


def _parse_singleton(combo: str):
    if len(combo) == 4:
        r1, s1, r2, s2 = _rank(combo[0]), _suit(combo[1]), _rank(combo[2]), _suit(combo[3])
        if r1 < r2:
            raise ValueError(f"The first rank must be equal or higher than the second rank: {combo}")
        if r1 == r2 and s1 == s2:
            raise ValueError(f"Duplicate cards are not allowed: {combo}")
        return r1, r2, (s1, s2)
    r1, r2 = _rank(combo[0]), _rank(combo[1])
    suited = "all"
    if len(combo) > 2:
        suited = {"s": "s", "o": "o"}.get(combo[2])
        if suited is None:
            raise ValueError(f"Invalid suitedness: {combo}")
    if r1 < r2:
        raise ValueError(f"The first rank must be equal or higher than the second rank: {combo}")
    if r1 == r2 and suited != "all":
        raise ValueError(f"A pair with suitedness is not allowed: {combo}")
    return r1, r2, suited


class Range:
    """A player's range: 1326 weights in [0, 1] (range.rs:38-39)."""

    def __init__(self, data=None):
        self.data = np.zeros(1326, np.float32) if data is None else np.asarray(data, np.float32).copy()

    @classmethod
    def ones(cls):
        return cls(np.ones(1326, np.float32))

    @classmethod
    def from_raw_data(cls, data):  # range.rs:215-228
        a = np.asarray(data, np.float32)
        if a.shape != (1326,):
            raise ValueError("Expected exactly 1326 elements")
        if not np.all((a >= 0.0) & (a <= 1.0)):
            raise ValueError("Invalid weight")
        return cls(a)

    def raw_data(self):
        return self.data

    def is_empty(self):
        return not np.any(self.data != 0.0)

    def _set(self, idx, w):
        self.data[idx] = w

    @classmethod
    def from_str(cls, s: str):  # range.rs:721-752
        s = _TRIM_RE.sub(r"\1", s).strip()
        parts = s.split(",")
        if parts and parts[-1] == "":
            parts.pop()
        r = cls()
        for part in reversed(parts):
            m = _RANGE_RE.match(part)
            if not m:
                raise ValueError(f"Failed to parse range: {part}")
            rng = m.group("range")
            w = np.float32(m.group("weight")) if m.group("weight") else np.float32(1.0)
            if not 0.0 <= w <= 1.0:
                raise ValueError(f"Invalid weight: {w}")
            if "-" in rng:
                r._dash(rng, w)
            elif "+" in rng:
                r._plus(rng, w)
            else:
                r1, r2, su = _parse_singleton(rng)
                r._set(_indices(r1, r2, su), w)
        return r

    def _plus(self, rng, w):  # range.rs:471-487
        r1, r2, su = _parse_singleton(rng[:-1])
        gap = r1 - r2
        if gap <= 1:
            for i in range(r1, 13):
                self._set(_indices(i, i - gap, su), w)
        else:
            for i in range(r2, r1):
                self._set(_indices(r1, i, su), w)

    def _dash(self, rng, w):  # range.rs:490-525
        a, b = rng.split("-")
        r11, r12, s1 = _parse_singleton(a)
        r21, r22, s2 = _parse_singleton(b)
        gap, gap2 = r11 - r12, r21 - r22
        if s1 != s2:
            raise ValueError(f"Suitedness does not match: {rng}")
        if gap == gap2:
            if r11 > r21:
                for i in range(r21, r11 + 1):
                    self._set(_indices(i, i - gap, s1), w)
            else:
                raise ValueError(f"Range must be in descending order: {rng}")
        elif r11 == r21:
            if r12 > r22:
                for i in range(r22, r12 + 1):
                    self._set(_indices(r11, i, s1), w)
            else:
                raise ValueError(f"Range must be in descending order: {rng}")
        else:
            raise ValueError(f"Invalid range: {rng}")

    def get_weight_pair(self, rank):
        return float(np.float32(np.mean(self.data[_pair_idx(rank)].astype(np.float64))))

    def get_weight_suited(self, r1, r2):
        return float(np.float32(np.mean(self.data[_suited_idx(r1, r2)].astype(np.float64))))

    def get_weight_offsuit(self, r1, r2):
        return float(np.float32(np.mean(self.data[_offsuit_idx(r1, r2)].astype(np.float64))))

    def __eq__(self, other):
        return isinstance(other, Range) and np.array_equal(self.data, other.data)
