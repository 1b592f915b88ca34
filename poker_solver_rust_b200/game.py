"""Python mirror of the reference's game / solve API (crates/range-solver).

Names follow the reference: ``TreeConfig`` / ``BetSizeOptions`` /
``ActionTree`` (action_tree.rs, bet_size.rs), ``CardConfig`` (card.rs),
``PostFlopGame`` with ``with_config`` / ``allocate_memory`` and the query
methods (game/interpreter.rs, game/query.rs), and the solver functions
``solve``, ``solve_step``, ``compute_exploitability``, ``finalize``,
``root_cfvalues``, ``root_cfvalues_with_reach`` (solver.rs, utility.rs).
Every call goes through the C ABI of ``_lib/libps_b200.so``; there is no
Python or CPU fallback for any of the compute.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from enum import IntEnum
from typing import Optional, Sequence

import numpy as np

from . import _native as N
from .cards import NOT_DEALT, Range

ACTION_NAMES = ["None", "Fold", "Check", "Call", "Bet", "Raise", "AllIn", "Chance"]


class BoardState(IntEnum):  # action_tree.rs:76-84
    Flop = 0
    Turn = 1
    River = 2


@dataclass
class BetSizeOptions:
    """Bet and raise size strings exactly as the reference parses them
    (bet_size.rs:82-112), e.g. ``BetSizeOptions("50%, 100%, a", "100%")``."""

    bet: str = ""
    raise_: str = ""


@dataclass
class TreeConfig:  # action_tree.rs:130-192
    initial_state: BoardState = BoardState.Flop
    starting_pot: int = 0
    effective_stack: int = 0
    rake_rate: float = 0.0
    rake_cap: float = 0.0
    flop_bet_sizes: Sequence[BetSizeOptions] = field(default_factory=lambda: [BetSizeOptions(), BetSizeOptions()])
    turn_bet_sizes: Sequence[BetSizeOptions] = field(default_factory=lambda: [BetSizeOptions(), BetSizeOptions()])
    river_bet_sizes: Sequence[BetSizeOptions] = field(default_factory=lambda: [BetSizeOptions(), BetSizeOptions()])
    turn_donk_sizes: Optional[str] = None
    river_donk_sizes: Optional[str] = None
    add_allin_threshold: float = 0.0
    force_allin_threshold: float = 0.0
    merging_threshold: float = 0.0
    depth_limit: Optional[int] = None
    max_bets: int = 0  # extension (0 = no cap, as the reference)

    def to_c(self) -> N.PsTreeConfig:
        c = N.PsTreeConfig()
        c.initial_state = int(self.initial_state)
        c.starting_pot = int(self.starting_pot)
        c.effective_stack = int(self.effective_stack)
        c.depth_limit = -1 if self.depth_limit is None else int(self.depth_limit)
        c.rake_rate = float(self.rake_rate)
        c.rake_cap = float(self.rake_cap)
        c.add_allin_threshold = float(self.add_allin_threshold)
        c.force_allin_threshold = float(self.force_allin_threshold)
        c.merging_threshold = float(self.merging_threshold)
        c.max_bets = int(self.max_bets)
        keep = []
        for si, street in enumerate((self.flop_bet_sizes, self.turn_bet_sizes, self.river_bet_sizes)):
            for p in range(2):
                for k, s in enumerate((street[p].bet, street[p].raise_)):
                    b = s.encode()
                    keep.append(b)
                    c.bet_sizes[si * 4 + p * 2 + k] = b
        for k, d in enumerate((self.turn_donk_sizes, self.river_donk_sizes)):
            if d is not None:
                b = d.encode()
                keep.append(b)
                c.donk_sizes[k] = b
        c._keep = keep
        return c

    def to_dict(self) -> dict:
        """Plain form used to feed the same configuration to the oracle."""
        def ms(street):
            return [(street[p].bet, street[p].raise_) for p in range(2)]
        return {
            "initial_state": ["flop", "turn", "river"][int(self.initial_state)],
            "starting_pot": self.starting_pot,
            "effective_stack": self.effective_stack,
            "rake_rate": self.rake_rate,
            "rake_cap": self.rake_cap,
            "flop_bet_sizes": ms(self.flop_bet_sizes),
            "turn_bet_sizes": ms(self.turn_bet_sizes),
            "river_bet_sizes": ms(self.river_bet_sizes),
            "turn_donk_sizes": self.turn_donk_sizes,
            "river_donk_sizes": self.river_donk_sizes,
            "add_allin_threshold": self.add_allin_threshold,
            "force_allin_threshold": self.force_allin_threshold,
            "merging_threshold": self.merging_threshold,
            "depth_limit": self.depth_limit,
        }


class ActionTree:
    """The abstract betting tree of a TreeConfig (action_tree.rs:326-334).
    The tree itself is built inside the library when the game is created."""

    def __init__(self, config: TreeConfig):
        self.config = config

    @classmethod
    def new(cls, config: TreeConfig):
        return cls(config)


@dataclass
class CardConfig:  # card.rs:19-32
    range: Sequence[Range]
    flop: Sequence[int]
    turn: int = NOT_DEALT
    river: int = NOT_DEALT

    def to_c(self) -> N.PsCardConfig:
        c = N.PsCardConfig()
        r0 = np.ascontiguousarray(self.range[0].raw_data(), np.float32)
        r1 = np.ascontiguousarray(self.range[1].raw_data(), np.float32)
        c.range[0] = r0.ctypes.data_as(C.POINTER(C.c_float))
        c.range[1] = r1.ctypes.data_as(C.POINTER(C.c_float))
        for i in range(3):
            c.flop[i] = int(self.flop[i])
        c.turn = int(self.turn)
        c.river = int(self.river)
        c._keep = (r0, r1)
        return c


def _f32(n):
    return np.zeros(n, np.float32)


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class PostFlopGame:
    """A subgame on the GPU (game/mod.rs PostFlopGame)."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def with_config(cls, card_config: CardConfig, action_tree: ActionTree) -> "PostFlopGame":
        L = N.lib()
        cc = card_config.to_c()
        tc = action_tree.config.to_c()
        h = C.c_void_p()
        N.check(L.ps_game_new(C.byref(cc), C.byref(tc), C.byref(h)))
        return cls(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            N.lib().ps_game_free(h)
            self._h = None

    # ---- construction ----
    def memory_usage(self) -> int:
        v = C.c_uint64()
        N.check(N.lib().ps_game_memory_usage(self._h, C.byref(v)))
        return int(v.value)

    def set_terminals_first(self, enable: bool) -> None:
        """Chooses the tree program before allocate_memory
        (ps_game_set_terminals_first): every terminal of a pass in one step
        (True) or each depth's terminals in that depth's step (False)."""
        N.check(N.lib().ps_game_set_terminals_first(self._h, int(enable)))

    def program_info(self) -> dict:
        """The compiled tree program's shape (ps_game_program_info; host-side,
        no GPU needed): working slots and their stride, steps / node ops /
        terminal ops / terminal runs per traverser, S (sum over decision edges
        of the acting player's hands) and the number of boards."""
        v = (C.c_int64 * 12)()
        N.check(N.lib().ps_game_program_info(self._h, v))
        return {"slots": int(v[0]), "slot_stride": int(v[1]), "steps": [int(v[2]), int(v[3])],
                "node_ops": [int(v[4]), int(v[5])], "terminal_ops": [int(v[6]), int(v[7])],
                "terminal_runs": [int(v[8]), int(v[9])], "S": int(v[10]), "boards": int(v[11])}

    def schedule(self) -> dict:
        """The launch shape of the game's solves (ps_game_schedule): grid mode
        runs the game on every SM (cooperative grid, "grid") or on the CTAs of
        one thread-block cluster ("cluster")."""
        v = (C.c_int32 * 8)()
        N.check(N.lib().ps_game_schedule(self._h, v))
        return {"block_threads": int(v[1]), "ctas": int(v[2]),
                "mode": {0: "one CTA", 1: "grid", 2: "cluster"}[int(v[7])]}

    def allocate_memory(self, enable_compression: bool = False) -> None:
        N.check(N.lib().ps_game_allocate_memory(self._h, int(enable_compression)))

    def num_private_hands(self, player: int) -> int:
        return N.check(N.lib().ps_num_private_hands(self._h, player))

    def private_cards(self, player: int) -> np.ndarray:
        n = self.num_private_hands(player)
        out = np.zeros(2 * n, np.uint8)
        N.check(N.lib().ps_private_cards(self._h, player, out.ctypes.data_as(C.POINTER(C.c_uint8))))
        return out.reshape(n, 2)

    def initial_weights(self, player: int) -> np.ndarray:
        out = _f32(self.num_private_hands(player))
        N.check(N.lib().ps_initial_weights(self._h, player, _fp(out)))
        return out

    def num_combinations(self) -> float:
        return float(N.lib().ps_num_combinations(self._h))

    def num_nodes(self) -> int:
        return int(N.lib().ps_num_nodes(self._h))

    def node_info(self, idx: int) -> dict:
        out = np.zeros(8, np.int32)
        N.check(N.lib().ps_node_info(self._h, idx, out.ctypes.data_as(C.POINTER(C.c_int32))))
        keys = ("player", "amount", "turn", "river", "num_children", "children_offset", "prev_kind", "prev_amount")
        return dict(zip(keys, (int(x) for x in out)))

    def child_indices(self, idx: int):
        out = np.zeros(64, np.int64)
        n = N.check(N.lib().ps_child_indices(self._h, idx, out.ctypes.data_as(C.POINTER(C.c_int64)), 64))
        return [int(x) for x in out[:n]]

    def same_hand_index(self, player: int) -> np.ndarray:
        out = np.zeros(self.num_private_hands(player), np.uint16)
        N.check(N.lib().ps_same_hand_index(self._h, player, out.ctypes.data_as(C.POINTER(C.c_uint16))))
        return out

    def hand_strength(self, turn: int, river: int, player: int):
        s = np.zeros(2000, np.uint16)
        i = np.zeros(2000, np.uint16)
        n = N.check(N.lib().ps_hand_strength(self._h, turn, river, player, s.ctypes.data_as(C.POINTER(C.c_uint16)),
                                             i.ctypes.data_as(C.POINTER(C.c_uint16))))
        return s[:n].copy(), i[:n].copy()

    def valid_indices(self, turn: int, river: int, player: int) -> np.ndarray:
        out = np.zeros(2000, np.uint16)
        n = N.check(N.lib().ps_valid_indices(self._h, turn, river, player, out.ctypes.data_as(C.POINTER(C.c_uint16))))
        return out[:n].copy()

    def strategy_at_index(self, idx: int) -> np.ndarray:
        out = _f32(200000)
        n = N.check(N.lib().ps_strategy_at_index(self._h, idx, _fp(out)))
        return out[:n].copy()

    def node_storage(self, idx: int, which: int) -> np.ndarray:
        out = _f32(200000)
        n = N.check(N.lib().ps_node_storage(self._h, idx, which, _fp(out)))
        return out[:n].copy()

    def seed_node_storage(self, idx: int, which: int, values) -> None:
        """Writes a decision node's cumulative strategy (1) or regrets (2)."""
        v = np.ascontiguousarray(values, np.float32)
        N.check(N.lib().ps_seed_node_storage(self._h, idx, which, _fp(v), len(v)))

    # ---- depth boundary ----
    def num_boundary_nodes(self) -> int:
        return int(N.lib().ps_num_boundary_nodes(self._h))

    def boundary_node_indices(self):
        n = self.num_boundary_nodes()
        out = np.zeros(max(n, 1), np.int64)
        N.check(N.lib().ps_boundary_node_indices(self._h, out.ctypes.data_as(C.POINTER(C.c_int64))))
        return out[:n].copy()

    def set_boundary_cfvs(self, ordinal: int, player: int, cfvs) -> None:
        v = np.ascontiguousarray(cfvs, np.float32)
        N.check(N.lib().ps_set_boundary_cfvs(self._h, ordinal, player, _fp(v), len(v)))

    # ---- navigation / queries ----
    def back_to_root(self):
        N.check(N.lib().ps_back_to_root(self._h))

    def play(self, action: int):
        N.check(N.lib().ps_play(self._h, action))

    def available_actions(self):
        k = np.zeros(256, np.int32)
        a = np.zeros(256, np.int32)
        n = N.check(N.lib().ps_available_actions(self._h, k.ctypes.data_as(C.POINTER(C.c_int32)),
                                                 a.ctypes.data_as(C.POINTER(C.c_int32)), 256))
        return [(ACTION_NAMES[k[i]], int(a[i])) for i in range(n)]

    def is_terminal_node(self) -> bool:
        return bool(N.check(N.lib().ps_is_terminal_node(self._h)))

    def is_chance_node(self) -> bool:
        return bool(N.check(N.lib().ps_is_chance_node(self._h)))

    def current_player(self) -> int:
        return N.check(N.lib().ps_current_player(self._h))

    def current_node_index(self) -> int:
        return int(N.lib().ps_current_node_index(self._h))

    def possible_cards(self) -> int:
        return int(N.lib().ps_possible_cards(self._h))

    def strategy(self) -> np.ndarray:
        out = _f32(200000)
        n = N.check(N.lib().ps_strategy(self._h, _fp(out)))
        return out[:n].copy()

    def cache_normalized_weights(self):
        N.check(N.lib().ps_cache_normalized_weights(self._h))

    def weights(self, player: int) -> np.ndarray:
        out = _f32(self.num_private_hands(player))
        N.check(N.lib().ps_weights(self._h, player, 0, _fp(out)))
        return out

    def normalized_weights(self, player: int) -> np.ndarray:
        out = _f32(self.num_private_hands(player))
        N.check(N.lib().ps_weights(self._h, player, 1, _fp(out)))
        return out

    def expected_values(self, player: int) -> np.ndarray:
        out = _f32(200000)
        n = N.check(N.lib().ps_expected_values(self._h, player, 0, _fp(out)))
        return out[:n].copy()

    def expected_values_detail(self, player: int) -> np.ndarray:
        out = _f32(200000)
        n = N.check(N.lib().ps_expected_values(self._h, player, 1, _fp(out)))
        return out[:n].copy()

    def total_bet_amount(self):
        out = np.zeros(2, np.int32)
        N.check(N.lib().ps_total_bet_amount(self._h, out.ctypes.data_as(C.POINTER(C.c_int32))))
        return [int(out[0]), int(out[1])]

    # ---- checkpoint ----
    def storage_export(self) -> bytes:
        need = C.c_uint64()
        N.check(N.lib().ps_state_export(self._h, None, 0, C.byref(need)))
        buf = C.create_string_buffer(need.value)
        N.check(N.lib().ps_state_export(self._h, buf, need.value, C.byref(need)))
        return buf.raw

    def storage_import(self, data: bytes):
        N.check(N.lib().ps_state_import(self._h, data, len(data)))

    @property
    def last_iterations(self) -> int:
        v = C.c_uint32()
        N.check(N.lib().ps_last_iterations(self._h, C.byref(v)))
        return int(v.value)


# ---- solver functions (solver.rs, utility.rs) ----
def solve(game: PostFlopGame, max_num_iterations: int, target_exploitability: float, print_progress: bool = False) -> float:
    e = C.c_float()
    N.check(N.lib().ps_solve(game._h, max_num_iterations, target_exploitability, int(print_progress), C.byref(e)))
    return float(e.value)


def solve_step(game: PostFlopGame, current_iteration: int) -> None:
    N.check(N.lib().ps_solve_step(game._h, current_iteration))


def compute_exploitability(game: PostFlopGame) -> float:
    e = C.c_float()
    N.check(N.lib().ps_compute_exploitability(game._h, C.byref(e)))
    return float(e.value)


def finalize(game: PostFlopGame) -> None:
    N.check(N.lib().ps_finalize(game._h))


def root_cfvalues_with_reach(game: PostFlopGame, player: int, opp_reach) -> np.ndarray:
    r = None if opp_reach is None else np.ascontiguousarray(opp_reach, np.float32)
    out = _f32(game.num_private_hands(player))
    N.check(N.lib().ps_root_cfvalues_with_reach(game._h, player, None if r is None else _fp(r), _fp(out)))
    return out


def root_cfvalues(game: PostFlopGame, player: int) -> np.ndarray:
    return root_cfvalues_with_reach(game, player, None)


def eval_fixed_strategy(game: PostFlopGame, w0, w1):
    """Root cfvalues of both players under the average strategy, with initial
    weights w0, w1 (solver hand order) in place of the game's: (cfv0, cfv1),
    where cfv0 depends on w1 and the boundary values, cfv1 on w0."""
    a = np.ascontiguousarray(w0, np.float32)
    b = np.ascontiguousarray(w1, np.float32)
    c0, c1 = _f32(game.num_private_hands(0)), _f32(game.num_private_hands(1))
    N.check(N.lib().ps_eval_fixed_strategy(game._h, _fp(a), _fp(b), _fp(c0), _fp(c1)))
    return c0, c1


def eval_fixed_strategy_adjoint(game: PostFlopGame, w0, w1, g0, g1):
    """Vector-Jacobian product of eval_fixed_strategy for cotangents g0, g1 on
    (cfv0, cfv1): returns (dw0, dw1, dbcfv) with dbcfv[k][p] the gradient with
    respect to the boundary values of ordinal k, player p."""
    a = np.ascontiguousarray(w0, np.float32)
    b = np.ascontiguousarray(w1, np.float32)
    ga = None if g0 is None else np.ascontiguousarray(g0, np.float32)
    gb = None if g1 is None else np.ascontiguousarray(g1, np.float32)
    H0, H1 = game.num_private_hands(0), game.num_private_hands(1)
    nb = game.num_boundary_nodes()
    dw0, dw1 = _f32(H0), _f32(H1)
    db = _f32(max(1, nb * (H0 + H1)))
    N.check(N.lib().ps_eval_fixed_strategy_adjoint(game._h, _fp(a), _fp(b), None if ga is None else _fp(ga),
                                                   None if gb is None else _fp(gb), _fp(dw0), _fp(dw1), _fp(db)))
    dbcfv = [[db[k * (H0 + H1):k * (H0 + H1) + H0].copy(), db[k * (H0 + H1) + H0:(k + 1) * (H0 + H1)].copy()]
             for k in range(nb)]
    return dw0, dw1, dbcfv


def compute_average(values, weights) -> float:  # utility.rs:127-136
    v = np.asarray(values, np.float64)
    w = np.asarray(weights, np.float64)
    return float(np.float32((v * w).sum() / w.sum()))


def discount_params(t: int):
    out = np.zeros(3, np.float32)
    N.check(N.lib().ps_discount_params(t, _fp(out)))
    return float(out[0]), float(out[1]), float(out[2])


BET_KINDS = ["PotRelative", "PrevBetRelative", "Additive", "Geometric", "AllIn"]


def parse_bet_sizes(sizes: str, is_raise: bool):
    """BetSizeOptions::try_from for one list: [(kind, float, int, cap)]."""
    k = np.zeros(64, np.int32)
    f = np.zeros(64)
    i = np.zeros(64, np.int32)
    c = np.zeros(64, np.int32)
    n = N.check(N.lib().ps_parse_bet_sizes(sizes.encode(), int(is_raise), k.ctypes.data_as(C.POINTER(C.c_int32)),
                                           f.ctypes.data_as(C.POINTER(C.c_double)),
                                           i.ctypes.data_as(C.POINTER(C.c_int32)),
                                           c.ctypes.data_as(C.POINTER(C.c_int32)), 64))
    return [(BET_KINDS[k[j]], float(f[j]), int(i[j]), int(c[j])) for j in range(n)]


def hand_table() -> np.ndarray:
    out = np.zeros(8192, np.int32)
    n = N.lib().ps_hand_table(out.ctypes.data_as(C.POINTER(C.c_int32)), 8192)
    return out[:n].copy()


# ---- batched datagen path ----
def _pack_configs(card_configs, tree_configs):
    """ps_card_config / ps_tree_config arrays for n spots, filled column by
    column through numpy views at the structs' field offsets: the range
    pointers address the ranges' own float32 arrays (a range held in another
    form is converted once), and every distinct bet-size string is encoded
    once. Returns the two ctypes arrays and the objects they point into."""
    n = len(card_configs)
    cc = (N.PsCardConfig * n)()
    tc = (N.PsTreeConfig * n)()
    f32 = np.dtype(np.float32)
    addrs, converted = [], []
    for c in card_configs:
        for r in c.range:
            d = r.raw_data()
            if type(d) is not np.ndarray or d.dtype != f32 or d.shape != (1326,) or not d.flags.c_contiguous:
                d = np.ascontiguousarray(d, np.float32)
                if d.shape != (1326,):
                    raise ValueError("a range holds 1326 weights")
                converted.append(d)
            addrs.append(d.__array_interface__["data"][0])
    craw = np.frombuffer(cc, np.uint8).reshape(n, C.sizeof(N.PsCardConfig))
    traw = np.frombuffer(tc, np.uint8).reshape(n, C.sizeof(N.PsTreeConfig))

    def col(raw, struct, field, dtype, count=1):
        off = getattr(struct, field).offset
        return raw[:, off:off + np.dtype(dtype).itemsize * count].view(dtype)

    if n:
        col(craw, N.PsCardConfig, "range", np.uint64, 2)[:] = np.asarray(addrs, np.uint64).reshape(n, 2)
    cards = np.array([[c.flop[0], c.flop[1], c.flop[2], c.turn, c.river] for c in card_configs], np.uint8)
    col(craw, N.PsCardConfig, "flop", np.uint8, 3)[:] = cards[:, :3]
    col(craw, N.PsCardConfig, "turn", np.uint8)[:, 0] = cards[:, 3]
    col(craw, N.PsCardConfig, "river", np.uint8)[:, 0] = cards[:, 4]

    strings = {}  # str -> bytes, kept alive with the arrays

    def addr(sv):
        if sv is None:
            return 0
        b = strings.get(sv)
        if b is None:
            b = strings[sv] = C.create_string_buffer(sv.encode())
        return C.addressof(b)

    T = tree_configs
    col(traw, N.PsTreeConfig, "initial_state", np.int32)[:, 0] = [int(t.initial_state) for t in T]
    col(traw, N.PsTreeConfig, "starting_pot", np.int32)[:, 0] = [int(t.starting_pot) for t in T]
    col(traw, N.PsTreeConfig, "effective_stack", np.int32)[:, 0] = [int(t.effective_stack) for t in T]
    col(traw, N.PsTreeConfig, "depth_limit", np.int32)[:, 0] = [-1 if t.depth_limit is None else int(t.depth_limit)
                                                               for t in T]
    for f in ("rake_rate", "rake_cap", "add_allin_threshold", "force_allin_threshold", "merging_threshold"):
        col(traw, N.PsTreeConfig, f, np.float64)[:, 0] = [float(getattr(t, f)) for t in T]
    col(traw, N.PsTreeConfig, "max_bets", np.int32)[:, 0] = [int(t.max_bets) for t in T]
    sizes = col(traw, N.PsTreeConfig, "bet_sizes", np.uint64, 12)
    menus = {}  # menu strings of a spot -> their 12 addresses (spots share a few menus)
    rows = []
    for t in T:
        f, u, r = t.flop_bet_sizes, t.turn_bet_sizes, t.river_bet_sizes
        f0, f1, u0, u1, r0, r1 = f[0], f[1], u[0], u[1], r[0], r[1]
        key = (f0.bet, f0.raise_, f1.bet, f1.raise_, u0.bet, u0.raise_, u1.bet, u1.raise_,
               r0.bet, r0.raise_, r1.bet, r1.raise_)  # street-major, then player, then bet / raise
        row = menus.get(key)
        if row is None:
            row = menus[key] = [addr(s) for s in key]
        rows.append(row)
    if n:
        sizes[:] = np.asarray(rows, np.uint64)
    donk = col(traw, N.PsTreeConfig, "donk_sizes", np.uint64, 2)
    donk[:, 0] = [addr(t.turn_donk_sizes) for t in T]
    donk[:, 1] = [addr(t.river_donk_sizes) for t in T]
    return cc, tc, (card_configs, converted, strings, menus, T)


def _is_cuda_tensor(x) -> bool:
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


def autotune_stages(shapes, trial_ms):
    """Trial records of an autotune log (ps_batch_autotune_trials): shapes are
    (threads per CTA, scan-buffer warps, spots per CTA, node-op parts).  The
    log lists the sweep (every shape once) and then the refine runs, so the
    first shape that repeats starts the refine stage."""
    out, seen, stage = [], set(), "sweep"
    for k, ms in zip(shapes, trial_ms):
        if k in seen:
            stage = "refine"
        seen.add(k)
        out.append({"block_threads": k[0], "scan_buffers": k[1], "spots_per_cta": k[2], "node_parts": k[3],
                    "trial_ms": ms, "stage": stage})
    return out


class BatchSolver:
    """Thousands of independent subgames solved by one persistent launch
    (replaces the per-spot GpuBatchSolver launches of the reference's GPU
    datagen, crates/cfvnet/src/datagen/domain/pipeline.rs:232-343)."""

    def __init__(self, card_configs: Sequence[CardConfig], tree_configs: Sequence[TreeConfig],
                 block_threads: int = 0, ctas_per_sm: int = 0, sort_by_cost: bool = True,
                 stage_tables: int = -1, scan_buffers: int = 0, instances_per_cta: int = 0,
                 scheduler: int = 0, flow_threads: int = 0, flow_spots_per_cta: int = 0, node_parts: int = 0):
        """Options as ps_batch_opts (include/ps_range_solver.h).  scheduler:
        0 = default (dataflow for batches of more spots than SMs), 1 =
        step-synchronous (one barrier per step), 2 = dataflow; flow_threads,
        flow_spots_per_cta, node_parts shape the dataflow launch (0 = default,
        or autotuned with block_threads = -1)."""
        n = len(card_configs)
        cc, tc, keep = _pack_configs(card_configs, tree_configs)
        opts = N.PsBatchOpts(block_threads, ctas_per_sm, int(sort_by_cost), stage_tables, scan_buffers,
                             instances_per_cta, scheduler, flow_threads, flow_spots_per_cta, node_parts)
        h = C.c_void_p()
        N.check(N.lib().ps_batch_new(cc, tc, n, C.byref(opts), C.byref(h)))
        self._h = h
        self.n = n
        self.starting_pots = np.array([t.starting_pot for t in tree_configs], np.float32)
        self.effective_stacks = np.array([t.effective_stack for t in tree_configs], np.float32)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and N is not None and N.lib is not None:
            N.lib().ps_batch_free(h)
            self._h = None

    def solve(self, max_num_iterations: int, target_exploitability) -> None:
        t = np.ascontiguousarray(np.broadcast_to(np.asarray(target_exploitability, np.float32), (self.n,)))
        N.check(N.lib().ps_batch_solve(self._h, max_num_iterations, _fp(t)))

    def results(self):
        e = _f32(self.n)
        it = np.zeros(self.n, np.int32)
        N.check(N.lib().ps_batch_results(self._h, _fp(e), it.ctypes.data_as(C.POINTER(C.c_int32))))
        return e, it

    def root_strategy(self, spot: int) -> np.ndarray:
        out = _f32(200000)
        n = N.check(N.lib().ps_batch_root_strategy(self._h, spot, _fp(out)))
        return out[:n].copy()

    def num_nodes(self, spot: int) -> int:
        return int(N.check(N.lib().ps_batch_num_nodes(self._h, spot)))

    def node_storage(self, spot: int, node: int, which: int) -> np.ndarray:
        """[A * H_actor] rows of a decision node of one spot: which = 1
        strategy sums, 2 regrets (PostFlopGame.node_storage for a batch)."""
        out = _f32(16 * 1326)
        n = N.check(N.lib().ps_batch_node_storage(self._h, spot, node, which, _fp(out)))
        return out[:n].copy()

    def root_cfvalues(self, spot: int, player: int) -> np.ndarray:
        """Root cfvalues of `player` under the average strategy after the last
        solve (computed on the device at the end of the spot's solve)."""
        out = np.zeros(1326, np.float32)
        n = N.check(N.lib().ps_batch_root_cfvalues(self._h, spot, player, _fp(out)))
        return out[:n].copy()

    def last_timing(self):
        a, b = C.c_float(), C.c_float()
        N.check(N.lib().ps_batch_last_timing(self._h, C.byref(a), C.byref(b)))
        return float(a.value), float(b.value)

    def iteration_bytes(self, spot: int) -> float:
        return float(N.lib().ps_batch_iteration_bytes(self._h, spot))

    def io_bytes(self):
        a, b = C.c_uint64(), C.c_uint64()
        N.check(N.lib().ps_batch_io_bytes(self._h, C.byref(a), C.byref(b)))
        return int(a.value), int(b.value)

    def autotune_log(self):
        """[(threads per CTA, scan-buffer warps, trial ms)] of the autotune run by
        block_threads=-1."""
        b = (C.c_int32 * 32)()
        u = (C.c_int32 * 32)()
        t = (C.c_float * 32)()
        n = N.check(N.lib().ps_batch_autotune_log(self._h, b, u, t, 32))
        return [(int(b[i]), int(u[i]), float(t[i])) for i in range(min(n, 32))]

    def autotune_trials(self):
        """Every trial of the last autotune: dicts of threads per CTA,
        scan-buffer warps, spots per CTA and node-op parts (0 for a
        step-synchronous trial), the trial's device ms and its stage: "sweep"
        for the trials of every shape on one wave of spots, "refine" for the
        re-runs of the leading shapes that the first fresh solve makes on a
        larger sample with its own targets (the library lists them after the
        sweep, so a shape's second entry is its refine run); the choice is the
        fastest refine run, or the fastest sweep trial when there was none."""
        cap = 256
        shape = (C.c_int32 * (4 * cap))()
        t = (C.c_float * cap)()
        n = min(N.check(N.lib().ps_batch_autotune_trials(self._h, shape, t, cap)), cap)
        return autotune_stages([tuple(int(shape[4 * i + j]) for j in range(4)) for i in range(n)],
                               [float(t[i]) for i in range(n)])

    def config(self):
        """The launch shape of the batch's solves (ps_batch_schedule)."""
        v = (C.c_int32 * 8)()
        N.check(N.lib().ps_batch_schedule(self._h, v))
        return {"scheduler": "dataflow" if v[0] == N.PS_SCHED_FLOW else "step-synchronous",
                "block_threads": int(v[1]), "grid": int(v[2]), "ctas_per_sm": int(v[3]),
                "scan_buffers": int(v[4]), "spots_per_cta": int(v[5]), "node_parts": int(v[6]),
                "grid_mode": bool(v[7])}

    # ---- depth-limited spots: iteration ranges and boundary values
    #      (gpu-range-solver batch.rs:279-585) ----

    def run_iterations(self, start: int, end: int, root: bool = True, exploitability: bool = False) -> None:
        """DCFR iterations [start, end) of every spot from the current state in
        one launch, with no exploitability checks (batch.rs:414
        run_iterations).  root: afterwards compute the root cfvalues and the
        boundary reach under the average strategy; exploitability: also the
        exploitability of every spot (results())."""
        epi = (N.PS_EPI_ROOT if root else 0) | (N.PS_EPI_EXPL if exploitability else 0)
        N.check(N.lib().ps_batch_run_iterations(self._h, start, end, epi))

    def reset(self) -> None:
        """The next run_iterations starts from zero regrets and strategy sums."""
        N.check(N.lib().ps_batch_reset(self._h))

    def num_boundary_items(self) -> int:
        return int(N.lib().ps_batch_num_boundary_items(self._h))

    def boundary_items(self) -> dict:
        """Per boundary item (one depth boundary of one spot, spot by spot):
        spot, ordinal, 4-card board, the boundary's pot and the stack behind it,
        and the spot's starting pot and effective stack."""
        n = self.num_boundary_items()
        spot = np.zeros(n, np.int32)
        ordinal = np.zeros(n, np.int32)
        boards = np.zeros((n, 4), np.uint8)
        pots = np.zeros(n, np.float32)
        stacks = np.zeros(n, np.float32)
        if n:
            N.check(N.lib().ps_batch_boundary_items(
                self._h, spot.ctypes.data_as(C.POINTER(C.c_int32)), ordinal.ctypes.data_as(C.POINTER(C.c_int32)),
                boards.ctypes.data_as(C.POINTER(C.c_uint8)), _fp(pots), _fp(stacks)))
        return {"spot": spot, "ordinal": ordinal, "boards": boards, "pots": pots, "stacks": stacks,
                "root_pots": self.starting_pots[spot], "root_stacks": self.effective_stacks[spot]}

    def set_boundary_cfvs(self, values) -> None:
        """Boundary values of every item, [items, 2, 1326] in the 1326-combo
        layout (numpy array or CUDA tensor); each spot takes its own hands'
        entries, with the semantics of PostFlopGame.set_boundary_cfvs."""
        n = self.num_boundary_items()
        if _is_cuda_tensor(values):
            import torch

            v = values.detach().to(torch.float32).contiguous()
            assert tuple(v.shape) == (n, 2, 1326), v.shape
            torch.cuda.current_stream(v.device).synchronize()
            N.check(N.lib().ps_batch_set_boundary_cfvs(self._h, C.c_void_p(v.data_ptr()), 1))
        else:
            v = np.ascontiguousarray(values, np.float32)
            assert v.shape == (n, 2, 1326), v.shape
            N.check(N.lib().ps_batch_set_boundary_cfvs(self._h, C.c_void_p(v.ctypes.data), 0))

    def root_cfvalues_all(self, device: bool = False):
        """Both players' root cfvalues of every spot under the average strategy
        (last root epilogue, solve or adjoint), [n, 2, 1326] in the combo
        layout (numpy, or a CUDA tensor when device=True)."""
        if device:
            import torch

            out = torch.empty((self.n, 2, 1326), dtype=torch.float32, device="cuda")
            torch.cuda.current_stream().synchronize()
            N.check(N.lib().ps_batch_root_cfvalues_all(self._h, C.c_void_p(out.data_ptr()), 1))
            return out
        out = np.zeros((self.n, 2, 1326), np.float32)
        N.check(N.lib().ps_batch_root_cfvalues_all(self._h, C.c_void_p(out.ctypes.data), 0))
        return out

    def adjoint(self, cotangent):
        """Batched adjoint of the fixed-strategy evaluation (ps_batch_adjoint):
        cotangent [n, 2, 1326] = dL/d(root cfvalues) -> (dL/d(initial weights)
        [n, 2, 1326], dL/d(boundary values) [items, 2, 1326]), as CUDA tensors
        for a CUDA cotangent, numpy arrays otherwise."""
        ni = self.num_boundary_items()
        if _is_cuda_tensor(cotangent):
            import torch

            g = cotangent.detach().to(torch.float32).contiguous()
            assert tuple(g.shape) == (self.n, 2, 1326), g.shape
            dw = torch.empty_like(g)
            dB = torch.empty((ni, 2, 1326), dtype=torch.float32, device=g.device)
            torch.cuda.current_stream(g.device).synchronize()
            N.check(N.lib().ps_batch_adjoint(self._h, C.c_void_p(g.data_ptr()), C.c_void_p(dw.data_ptr()),
                                             C.c_void_p(dB.data_ptr()), 1))
            return dw, dB
        g = np.ascontiguousarray(cotangent, np.float32)
        assert g.shape == (self.n, 2, 1326), g.shape
        dw = np.zeros_like(g)
        dB = np.zeros((ni, 2, 1326), np.float32)
        N.check(N.lib().ps_batch_adjoint(self._h, C.c_void_p(g.ctypes.data), C.c_void_p(dw.ctypes.data),
                                         C.c_void_p(dB.ctypes.data), 0))
        return dw, dB

    def records(self) -> np.ndarray:
        """Training records of every spot, packed on the device in the
        reference's binary format (poker_solver_rust_b200.records): two per
        spot, player 0 then 1, from the root cfvalues of the last solve."""
        from . import records as R

        nbytes = N.check(N.lib().ps_batch_record_bytes(self._h))
        out = np.zeros(nbytes, np.uint8)
        N.check(N.lib().ps_batch_records(self._h, C.c_void_p(out.ctypes.data), 0))
        return out.view(R.record_dtype(int(out[0])))

    def boundary_reach(self, device: bool = False):
        """Each player's reach at every boundary under the average strategy as
        of the last root epilogue, [items, 2, 1326] (numpy, or a CUDA tensor
        when device=True)."""
        n = self.num_boundary_items()
        if device:
            import torch

            out = torch.empty((n, 2, 1326), dtype=torch.float32, device="cuda")
            torch.cuda.current_stream().synchronize()
            if n:
                N.check(N.lib().ps_batch_boundary_reach(self._h, C.c_void_p(out.data_ptr()), 1))
            return out
        out = np.zeros((n, 2, 1326), np.float32)
        if n:
            N.check(N.lib().ps_batch_boundary_reach(self._h, C.c_void_p(out.ctypes.data), 0))
        return out
