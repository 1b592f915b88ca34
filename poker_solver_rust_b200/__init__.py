"""B200-native range solver: the DCFR hot path of tjennings/poker_solver_rust
(`crates/range-solver`) as hand-written sm_100a CUDA kernels behind a C ABI
(include/ps_range_solver.h), with a Python mirror of the reference API."""

from .cards import (NOT_DEALT, Range, board_from_str, card_from_str, card_pair_to_index, card_to_string,
                    flop_from_str, hole_to_string, holes_to_strings, index_to_card_pair)
from .game import (ACTION_NAMES, ActionTree, BatchSolver, BetSizeOptions, BoardState, CardConfig, PostFlopGame,
                   TreeConfig, compute_average, compute_exploitability, discount_params, eval_fixed_strategy,
                   eval_fixed_strategy_adjoint, finalize, hand_table, parse_bet_sizes, root_cfvalues,
                   root_cfvalues_with_reach, solve, solve_step)
from ._native import SolverError

__all__ = [
    "NOT_DEALT", "Range", "board_from_str", "card_from_str", "card_pair_to_index", "card_to_string",
    "flop_from_str", "hole_to_string", "holes_to_strings", "index_to_card_pair", "ACTION_NAMES", "ActionTree",
    "BatchSolver", "BetSizeOptions", "BoardState", "CardConfig", "PostFlopGame", "TreeConfig", "compute_average",
    "compute_exploitability", "discount_params", "eval_fixed_strategy", "eval_fixed_strategy_adjoint", "finalize",
    "hand_table", "parse_bet_sizes", "root_cfvalues", "root_cfvalues_with_reach", "solve", "solve_step", "SolverError",
]
