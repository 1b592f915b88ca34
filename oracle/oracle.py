"""ORACLE — test infrastructure only.

ctypes front end of the C++ restatement of the reference's
``crates/range-solver`` (built by ``oracle/Makefile`` into ``oracle/_build``).
Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this module, and only as the checker / the timed CPU
baseline; the product never routes through it.

Method names follow the reference API (``PostFlopGame::with_config``,
``solve``, ``solve_step``, ``compute_exploitability``, ``finalize``,
``root_cfvalues_with_reach``, the query methods of ``game/query.rs``).
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")
_LIB_PATH = os.path.join(_BUILD, "liboracle.so")
_TABLE_PATH = os.path.join(_BUILD, "hand_table.bin")
_lock = threading.Lock()
_lib = None

# action_tree.rs:26-51 variant order
ACTION_NAMES = ["None", "Fold", "Check", "Call", "Bet", "Raise", "AllIn", "Chance"]


def build() -> None:
    """Compile the oracle (library + exhaustive hand table) if needed."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


class OrcTreeConfig(C.Structure):
    _fields_ = [
        ("initial_state", C.c_int32),
        ("starting_pot", C.c_int32),
        ("effective_stack", C.c_int32),
        ("depth_limit", C.c_int32),
        ("rake_rate", C.c_double),
        ("rake_cap", C.c_double),
        ("add_allin_threshold", C.c_double),
        ("force_allin_threshold", C.c_double),
        ("merging_threshold", C.c_double),
        ("sizes", C.c_char_p * 12),
        ("donk", C.c_char_p * 2),
    ]


def lib():
    global _lib
    with _lock:
        if _lib is None:
            if not (os.path.exists(_LIB_PATH) and os.path.exists(_TABLE_PATH)):
                build()
            L = C.CDLL(_LIB_PATH)
            vp, i32, i64, u32, f32, f64 = C.c_void_p, C.c_int32, C.c_int64, C.c_uint32, C.c_float, C.c_double
            P = C.POINTER
            sig = {
                "orc_last_error": (C.c_char_p, []),
                "orc_set_hand_table_path": (None, [C.c_char_p]),
                "orc_set_chance_threads": (None, [i32]),
                "orc_hand_table_exhaustive": (i32, [P(i32), i32, P(C.c_uint64)]),
                "orc_hand_table": (i32, [P(i32), i32]),
                "orc_hand_evaluate_internal": (i32, [P(i32)]),
                "orc_hand_evaluate": (i32, [P(i32)]),
                "orc_discount_params": (None, [u32, P(f32)]),
                "orc_action_tree_root": (i32, [P(OrcTreeConfig), P(i32), P(i32), i32]),
                "orc_parse_bet_sizes": (i32, [C.c_char_p, i32, P(i32), P(f64), P(i32), P(i32), i32]),
                "orc_game_new": (vp, [P(f32), P(f32), P(C.c_uint8), P(OrcTreeConfig), i32]),
                "orc_game_free": (None, [vp]),
                "orc_allocate_memory": (i32, [vp]),
                "orc_num_private_hands": (i64, [vp, i32]),
                "orc_private_cards": (i32, [vp, i32, P(C.c_uint8)]),
                "orc_initial_weights": (i32, [vp, i32, P(f64)]),
                "orc_num_combinations": (f64, [vp]),
                "orc_num_nodes": (i64, [vp]),
                "orc_node_info": (i32, [vp, i64, P(i32)]),
                "orc_same_hand_index": (i32, [vp, i32, P(C.c_uint16)]),
                "orc_valid_indices": (i32, [vp, i32, i32, i32, P(C.c_uint16)]),
                "orc_hand_strength": (i32, [vp, i32, i32, P(C.c_uint16), P(C.c_uint16)]),
                "orc_isomorphism_counts": (i32, [vp, i32, P(i32)]),
                "orc_solve": (f32, [vp, u32, f32, i32, P(u32)]),
                "orc_solve_step": (i32, [vp, u32]),
                "orc_exploitability": (f32, [vp]),
                "orc_solve_pass": (i32, [vp, u32, i32]),
                "orc_seed_node_storage": (i32, [vp, i64, i32, P(f32), i64]),
                "orc_mes_ev": (i32, [vp, P(f32)]),
                "orc_current_ev": (i32, [vp, P(f32)]),
                "orc_finalize": (i32, [vp]),
                "orc_root_cfvalues_with_reach": (i32, [vp, i32, P(f32), P(f64)]),
                "orc_node_storage": (i64, [vp, i64, i32, P(f64)]),
                "orc_strategy_at_index": (i64, [vp, i64, P(f64)]),
                "orc_num_boundary_nodes": (i64, [vp]),
                "orc_boundary_node_indices": (i32, [vp, P(i64)]),
                "orc_set_boundary_cfvs": (i32, [vp, i64, i32, P(f32), i64]),
                "orc_boundary_reach": (i32, [vp, i64, i32, P(f64)]),
                "orc_fd_central": (i32, [vp, P(f32), P(f32), P(f32), P(f32), i32, P(i32), P(i32), P(i32),
                                         P(i32), f64, P(f64)]),
                "orc_evaluate_node": (i32, [vp, i64, i32, P(f32), P(f64)]),
                "orc_back_to_root": (i32, [vp]),
                "orc_play": (i32, [vp, i64]),
                "orc_available_actions": (i32, [vp, P(i32), P(i32), i32]),
                "orc_is_terminal_node": (i32, [vp]),
                "orc_is_chance_node": (i32, [vp]),
                "orc_current_player": (i32, [vp]),
                "orc_possible_cards": (C.c_uint64, [vp]),
                "orc_current_node_index": (i64, [vp]),
                "orc_strategy": (i64, [vp, P(f64)]),
                "orc_cache_normalized_weights": (i32, [vp]),
                "orc_weights": (i32, [vp, i32, i32, P(f64)]),
                "orc_expected_values": (i64, [vp, i32, i32, P(f64)]),
                "orc_total_bet_amount": (i32, [vp, P(i32)]),
                "orc_lock_current_strategy": (i32, [vp, P(f32)]),
            }
            for name, (res, args) in sig.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            L.orc_set_hand_table_path(_TABLE_PATH.encode())
            _lib = L
        return _lib


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def _err():
    return lib().orc_last_error().decode()


def discount_params(t: int):
    out = np.zeros(3, np.float32)
    lib().orc_discount_params(t, _p(out, C.c_float))
    return float(out[0]), float(out[1]), float(out[2])


def hand_table() -> np.ndarray:
    out = np.zeros(8192, np.int32)
    n = lib().orc_hand_table(_p(out, C.c_int32), 8192)
    return out[:n].copy()


def set_chance_threads(n: int) -> None:
    """Threads for the chance children of solve passes, as the reference's
    rayon parallelism (solver.rs:264-326); results do not depend on it."""
    lib().orc_set_chance_threads(int(n))


def hand_evaluate_internal(cards) -> int:
    c = np.asarray(cards, np.int32)
    return int(lib().orc_hand_evaluate_internal(_p(c, C.c_int32)))


def hand_evaluate(cards) -> int:
    c = np.asarray(cards, np.int32)
    return int(lib().orc_hand_evaluate(_p(c, C.c_int32)))


def make_tree_config(cfg: dict) -> OrcTreeConfig:
    """``cfg`` keys mirror the reference TreeConfig (action_tree.rs:130-192);
    bet sizes are the reference's strings: ``sizes[street][player] = (bet, raise)``."""
    c = OrcTreeConfig()
    c.initial_state = {"flop": 0, "turn": 1, "river": 2}[cfg.get("initial_state", "river")]
    c.starting_pot = int(cfg["starting_pot"])
    c.effective_stack = int(cfg["effective_stack"])
    dl = cfg.get("depth_limit")
    c.depth_limit = -1 if dl is None else int(dl)
    c.rake_rate = float(cfg.get("rake_rate", 0.0))
    c.rake_cap = float(cfg.get("rake_cap", 0.0))
    c.add_allin_threshold = float(cfg.get("add_allin_threshold", 0.0))
    c.force_allin_threshold = float(cfg.get("force_allin_threshold", 0.0))
    c.merging_threshold = float(cfg.get("merging_threshold", 0.0))
    keep = []
    for si, street in enumerate(("flop", "turn", "river")):
        per = cfg.get(street + "_bet_sizes", [("", ""), ("", "")])
        for p in range(2):
            for k in range(2):
                s = per[p][k].encode()
                keep.append(s)
                c.sizes[si * 4 + p * 2 + k] = s
    for k, key in enumerate(("turn_donk_sizes", "river_donk_sizes")):
        v = cfg.get(key)
        if v is not None:
            s = v.encode()
            keep.append(s)
            c.donk[k] = s
    c._keep = keep
    return c


BET_KINDS = ["PotRelative", "PrevBetRelative", "Additive", "Geometric", "AllIn"]


def parse_bet_sizes(s: str, is_raise: bool):
    """(kind, float, int, cap) per entry, or raises ValueError (bet_size.rs)."""
    k = np.zeros(64, np.int32)
    f = np.zeros(64)
    i = np.zeros(64, np.int32)
    c = np.zeros(64, np.int32)
    n = lib().orc_parse_bet_sizes(s.encode(), int(is_raise), _p(k, C.c_int32), _p(f, C.c_double),
                                  _p(i, C.c_int32), _p(c, C.c_int32), 64)
    if n < 0:
        raise ValueError(_err())
    return [(BET_KINDS[k[j]], float(f[j]), int(i[j]), int(c[j])) for j in range(n)]


def action_tree_root(cfg: dict):
    c = make_tree_config(cfg)
    kinds = np.zeros(64, np.int32)
    amounts = np.zeros(64, np.int32)
    n = lib().orc_action_tree_root(C.byref(c), _p(kinds, C.c_int32), _p(amounts, C.c_int32), 64)
    if n < 0:
        raise ValueError(_err())
    return [(ACTION_NAMES[kinds[i]], int(amounts[i])) for i in range(n)]


class OracleGame:
    """One restated ``PostFlopGame`` (f32 parity build, or FP64 with ``fp64=True``)."""

    def __init__(self, ranges, board, tree_config: dict, fp64: bool = False):
        L = lib()
        r0 = np.ascontiguousarray(ranges[0], np.float32)
        r1 = np.ascontiguousarray(ranges[1], np.float32)
        b = list(board) + [255] * (5 - len(board))
        b5 = np.asarray(b, np.uint8)
        self._cfg = make_tree_config(tree_config)
        self.h = L.orc_game_new(_p(r0, C.c_float), _p(r1, C.c_float), _p(b5, C.c_uint8),
                                C.byref(self._cfg), int(fp64))
        if not self.h:
            raise ValueError(_err())
        self.fp64 = fp64

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_game_free(self.h)
            self.h = None

    def _check(self, rc):
        if rc < 0:
            raise RuntimeError(_err())
        return rc

    # ---- construction / solve ----
    def allocate_memory(self):
        self._check(lib().orc_allocate_memory(self.h))

    def num_private_hands(self, p):
        return int(lib().orc_num_private_hands(self.h, p))

    def private_cards(self, p):
        n = self.num_private_hands(p)
        out = np.zeros(2 * n, np.uint8)
        lib().orc_private_cards(self.h, p, _p(out, C.c_uint8))
        return out.reshape(n, 2)

    def initial_weights(self, p):
        out = np.zeros(self.num_private_hands(p))
        lib().orc_initial_weights(self.h, p, _p(out, C.c_double))
        return out

    def num_combinations(self):
        return float(lib().orc_num_combinations(self.h))

    def num_nodes(self):
        return int(lib().orc_num_nodes(self.h))

    def node_info(self, idx):
        out = np.zeros(8, np.int32)
        lib().orc_node_info(self.h, idx, _p(out, C.c_int32))
        keys = ("player", "amount", "turn", "river", "num_children", "children_offset",
                "prev_kind", "prev_amount")
        return dict(zip(keys, (int(x) for x in out)))

    def same_hand_index(self, p):
        out = np.zeros(self.num_private_hands(p), np.uint16)
        lib().orc_same_hand_index(self.h, p, _p(out, C.c_uint16))
        return out

    def valid_indices(self, kind, key, p):
        out = np.zeros(2000, np.uint16)
        n = lib().orc_valid_indices(self.h, kind, key, p, _p(out, C.c_uint16))
        return out[:n].copy()

    def hand_strength(self, pair_index, p):
        s = np.zeros(2000, np.uint16)
        i = np.zeros(2000, np.uint16)
        n = lib().orc_hand_strength(self.h, pair_index, p, _p(s, C.c_uint16), _p(i, C.c_uint16))
        return s[:n].copy(), i[:n].copy()

    def isomorphism_counts(self, turn=255):
        out = np.zeros(3, np.int32)
        lib().orc_isomorphism_counts(self.h, turn, _p(out, C.c_int32))
        return [int(x) for x in out]

    def solve(self, max_iter, target, print_progress=False):
        it = C.c_uint32(0)
        e = lib().orc_solve(self.h, max_iter, target, int(print_progress), C.byref(it))
        if e < 0 and _err():
            raise RuntimeError(_err())
        self.iterations_run = int(it.value)
        return float(e)

    def solve_step(self, t):
        self._check(lib().orc_solve_step(self.h, t))

    def solve_pass(self, t, player):
        self._check(lib().orc_solve_pass(self.h, t, player))

    def seed_node_storage(self, idx, which, values):
        v = np.ascontiguousarray(values, np.float32)
        self._check(lib().orc_seed_node_storage(self.h, idx, which, _p(v, C.c_float), len(v)))

    def compute_exploitability(self):
        return float(lib().orc_exploitability(self.h))

    def mes_ev(self):
        out = np.zeros(2, np.float32)
        self._check(lib().orc_mes_ev(self.h, _p(out, C.c_float)))
        return out

    def current_ev(self):
        out = np.zeros(2, np.float32)
        self._check(lib().orc_current_ev(self.h, _p(out, C.c_float)))
        return out

    def finalize(self):
        self._check(lib().orc_finalize(self.h))

    def root_cfvalues_with_reach(self, p, opp_reach):
        r = np.ascontiguousarray(opp_reach, np.float32)
        out = np.zeros(self.num_private_hands(p))
        self._check(lib().orc_root_cfvalues_with_reach(self.h, p, _p(r, C.c_float), _p(out, C.c_double)))
        return out

    def root_cfvalues(self, p):
        return self.root_cfvalues_with_reach(p, self.initial_weights(p ^ 1).astype(np.float32))

    def node_storage(self, idx, which):
        out = np.zeros(200000)
        n = lib().orc_node_storage(self.h, idx, which, _p(out, C.c_double))
        return out[:n].copy()

    def strategy_at_index(self, idx):
        out = np.zeros(200000)
        n = self._check(lib().orc_strategy_at_index(self.h, idx, _p(out, C.c_double)))
        return out[:n].copy()

    def num_boundary_nodes(self):
        return int(lib().orc_num_boundary_nodes(self.h))

    def boundary_node_indices(self):
        n = self.num_boundary_nodes()
        out = np.zeros(max(n, 1), np.int64)
        lib().orc_boundary_node_indices(self.h, _p(out, C.c_int64))
        return out[:n].copy()

    def set_boundary_cfvs(self, ordinal, p, cfvs):
        v = np.ascontiguousarray(cfvs, np.float32)
        lib().orc_set_boundary_cfvs(self.h, ordinal, p, _p(v, C.c_float), len(v))

    def fd_central(self, w, cot, coords, h=1e-3):
        """FP64 central differences of L = cot0 . cfv0 + cot1 . cfv1 under the
        game's current average strategy (cfv_p from the opponent's weights
        w[1-p]) at coords: rows (kind, ordinal, player, hand), kind 0 = weight
        of player `player`, 1 = boundary value.  Each perturbed input is
        rounded to f32 and the step actually taken is used (orc_fd_central)."""
        c = np.ascontiguousarray(np.asarray(coords, np.int32).reshape(-1, 4))
        cols = [np.ascontiguousarray(c[:, k]) for k in range(4)]
        w = [np.ascontiguousarray(x, np.float32) for x in w]
        cot = [np.ascontiguousarray(x, np.float32) for x in cot]
        out = np.zeros(len(c), np.float64)
        self._check(lib().orc_fd_central(self.h, _p(w[0], C.c_float), _p(w[1], C.c_float), _p(cot[0], C.c_float),
                                         _p(cot[1], C.c_float), len(c), *[_p(x, C.c_int32) for x in cols],
                                         float(h), _p(out, C.c_double)))
        return out

    def boundary_reach(self, ordinal, p):
        out = np.zeros(2000)
        n = lib().orc_boundary_reach(self.h, ordinal, p, _p(out, C.c_double))
        return out[:n].copy()

    def evaluate_node(self, idx, p, cfreach):
        r = np.ascontiguousarray(cfreach, np.float32)
        out = np.zeros(self.num_private_hands(p))
        self._check(lib().orc_evaluate_node(self.h, idx, p, _p(r, C.c_float), _p(out, C.c_double)))
        return out

    # ---- queries (game/query.rs) ----
    def back_to_root(self):
        self._check(lib().orc_back_to_root(self.h))

    def play(self, action):
        self._check(lib().orc_play(self.h, action))

    def available_actions(self):
        k = np.zeros(256, np.int32)
        a = np.zeros(256, np.int32)
        n = lib().orc_available_actions(self.h, _p(k, C.c_int32), _p(a, C.c_int32), 256)
        return [(ACTION_NAMES[k[i]], int(a[i])) for i in range(n)]

    def is_terminal_node(self):
        return bool(lib().orc_is_terminal_node(self.h))

    def is_chance_node(self):
        return bool(lib().orc_is_chance_node(self.h))

    def current_player(self):
        return int(lib().orc_current_player(self.h))

    def possible_cards(self):
        return int(lib().orc_possible_cards(self.h))

    def current_node_index(self):
        return int(lib().orc_current_node_index(self.h))

    def strategy(self):
        out = np.zeros(200000)
        n = self._check(lib().orc_strategy(self.h, _p(out, C.c_double)))
        return out[:n].copy()

    def cache_normalized_weights(self):
        self._check(lib().orc_cache_normalized_weights(self.h))

    def weights(self, p, normalized=False):
        out = np.zeros(self.num_private_hands(p))
        lib().orc_weights(self.h, p, int(normalized), _p(out, C.c_double))
        return out

    def expected_values(self, p, detail=False):
        out = np.zeros(200000)
        n = self._check(lib().orc_expected_values(self.h, p, int(detail), _p(out, C.c_double)))
        return out[:n].copy()

    def total_bet_amount(self):
        out = np.zeros(2, np.int32)
        lib().orc_total_bet_amount(self.h, _p(out, C.c_int32))
        return [int(out[0]), int(out[1])]

    def lock_current_strategy(self, strategy):
        s = np.ascontiguousarray(strategy, np.float32)
        self._check(lib().orc_lock_current_strategy(self.h, _p(s, C.c_float)))
