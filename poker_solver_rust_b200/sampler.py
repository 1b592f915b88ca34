"""Datagen situations drawn on the device (ps_sample_situations): boards,
pot / stack and two R(S,p) ranges per situation, with the distributions of
cfvnet datagen/sampler.rs and datagen/range_gen.rs."""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _native as N


@dataclass
class SamplerConfig:
    """cfvnet DatagenConfig fields the sampler reads (config.rs:72, :150-160)."""
    board_size: int = 5
    initial_stack: int = 200
    pot_intervals: List[List[int]] = field(default_factory=lambda: [[4, 20], [20, 80], [80, 200], [200, 400]])
    spr_intervals: Optional[List[List[float]]] = None
    seed: int = 0

    def to_c(self):
        pot = np.ascontiguousarray(self.pot_intervals, np.int32).reshape(-1, 2)
        spr = np.ascontiguousarray(self.spr_intervals if self.spr_intervals else np.zeros((0, 2)),
                                   np.float64).reshape(-1, 2)
        c = N.PsSamplerConfig(self.board_size, self.initial_stack, pot.shape[0],
                            pot.ctypes.data_as(C.POINTER(C.c_int32)), spr.shape[0],
                            spr.ctypes.data_as(C.POINTER(C.c_double)) if spr.size else None,
                            int(self.seed) & (2 ** 64 - 1))
        c._keep = (pot, spr)
        return c


def sample_situations(cfg: SamplerConfig, first: int, n: int, device="cuda"):
    """Situations first .. first + n - 1 of cfg's stream as CUDA tensors:
    boards [n, 5] uint8 (slots past board_size are 0), pots [n], stacks [n]
    int32, ranges [n, 2, 1326] float32 (OOP, IP); plus board_size."""
    import torch

    boards = torch.zeros((n, 5), dtype=torch.uint8, device=device)
    pots = torch.zeros(n, dtype=torch.int32, device=device)
    stacks = torch.zeros(n, dtype=torch.int32, device=device)
    ranges = torch.zeros((n, 2, 1326), dtype=torch.float32, device=device)
    if n:
        c = cfg.to_c()
        torch.cuda.current_stream(boards.device).synchronize()
        N.check(N.lib().ps_sample_situations(
            C.byref(c), int(first), int(n), C.c_void_p(boards.data_ptr()), C.c_void_p(pots.data_ptr()),
            C.c_void_p(stacks.data_ptr()), C.c_void_p(ranges.data_ptr()),
            C.c_void_p(torch.cuda.current_stream(boards.device).cuda_stream)))
    return {"boards": boards, "pots": pots, "stacks": stacks, "ranges": ranges, "board_size": cfg.board_size}


def to_spot_configs(situations, tree_config):
    """Host CardConfig / TreeConfig lists for a BatchSolver from sampled
    situations; tree_config(pot, stack) gives each spot's TreeConfig."""
    from .cards import NOT_DEALT, Range
    from .game import CardConfig

    b = situations["boards"].cpu().numpy()
    pots = situations["pots"].cpu().numpy()
    stacks = situations["stacks"].cpu().numpy()
    rg = situations["ranges"].cpu().numpy()
    river_dealt = situations["board_size"] == 5
    cards, trees = [], []
    for i in range(len(b)):
        river = int(b[i, 4]) if river_dealt else NOT_DEALT
        cards.append(CardConfig([Range(rg[i, 0]), Range(rg[i, 1])], [int(x) for x in b[i, :3]], int(b[i, 3]), river))
        trees.append(tree_config(int(pots[i]), int(stacks[i])))
    return cards, trees
