"""ctypes binding of the in-tree C-ABI library (include/ps_range_solver.h)."""

from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libps_b200.so")
_lock = threading.Lock()
_lib = None

PS_OK = 0
PS_ERR_INVALID = -1
PS_ERR_STATE = -2
PS_ERR_CUDA = -3
PS_ERR_UNSUPPORTED = -4
PS_ERR_DEVICE = -5


class PsTreeConfig(C.Structure):
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
        ("bet_sizes", C.c_char_p * 12),
        ("donk_sizes", C.c_char_p * 2),
        ("max_bets", C.c_int32),
        ("reserved", C.c_int32),
    ]


class PsSamplerConfig(C.Structure):
    _fields_ = [("board_size", C.c_int32), ("initial_stack", C.c_int32), ("num_pot_intervals", C.c_int32),
                ("pot_intervals", C.POINTER(C.c_int32)), ("num_spr_intervals", C.c_int32),
                ("spr_intervals", C.POINTER(C.c_double)), ("seed", C.c_uint64)]


class PsCardConfig(C.Structure):
    _fields_ = [
        ("range", C.POINTER(C.c_float) * 2),
        ("flop", C.c_uint8 * 3),
        ("turn", C.c_uint8),
        ("river", C.c_uint8),
        ("reserved", C.c_uint8 * 3),
    ]


class PsBatchOpts(C.Structure):
    _fields_ = [
        ("block_threads", C.c_int32),
        ("ctas_per_sm", C.c_int32),
        ("sort_by_cost", C.c_int32),
        ("stage_tables", C.c_int32),
        ("scan_buffers", C.c_int32),
        ("instances_per_cta", C.c_int32),
        ("scheduler", C.c_int32),
        ("flow_threads", C.c_int32),
        ("flow_spots_per_cta", C.c_int32),
        ("node_parts", C.c_int32),
    ]


PS_SCHED_DEFAULT, PS_SCHED_STEP, PS_SCHED_FLOW = 0, 1, 2


# name -> (restype, argtypes)
_SIGS = {}


def _sig(name, res, *args):
    _SIGS[name] = (res, list(args))


vp, i32, i64, u32, u64, f32, f64 = C.c_void_p, C.c_int32, C.c_int64, C.c_uint32, C.c_uint64, C.c_float, C.c_double
P = C.POINTER
_sig("ps_last_error", C.c_char_p)
_sig("ps_hand_table", i32, P(i32), i32)
_sig("ps_discount_params", i32, u32, P(f32))
_sig("ps_debug_grid_barrier_timeout", i32, i32, i32, i64, i32, P(i32), P(i32), P(f32))
_sig("ps_game_program_info", i32, vp, P(i64))
_sig("ps_game_set_terminals_first", i32, vp, i32)
_sig("ps_game_schedule", i32, vp, P(i32))
_sig("ps_eval_fixed_strategy_ex", i32, vp, vp, vp, vp, vp, i32)
_sig("ps_eval_fixed_strategy_adjoint_ex", i32, vp, vp, vp, vp, vp, vp, vp, vp, i32)
_sig("ps_set_boundary_cfvs_all", i32, vp, vp, i32)
_sig("ps_parse_bet_sizes", i32, C.c_char_p, i32, P(i32), P(f64), P(i32), P(i32), i32)
_sig("ps_game_new", i32, P(PsCardConfig), P(PsTreeConfig), P(vp))
_sig("ps_game_free", None, vp)
_sig("ps_game_memory_usage", i32, vp, P(u64))
_sig("ps_game_allocate_memory", i32, vp, i32)
_sig("ps_solve", i32, vp, u32, f32, i32, P(f32))
_sig("ps_last_iterations", i32, vp, P(u32))
_sig("ps_solve_step", i32, vp, u32)
_sig("ps_compute_exploitability", i32, vp, P(f32))
_sig("ps_compute_exploitability_noalloc", i32, vp, P(f32))
_sig("ps_finalize", i32, vp)
_sig("ps_root_cfvalues_with_reach", i32, vp, i32, P(f32), P(f32))
_sig("ps_eval_fixed_strategy", i32, vp, P(f32), P(f32), P(f32), P(f32))
_sig("ps_boundary_reach", i32, vp, P(f32))
_sig("ps_boundary_river_reduce", i32, i32, P(C.c_uint8), P(f32), P(f32), vp, i32, vp, vp, i32, vp, vp)
_sig("ps_boundary_first_layer", i32, i32, P(C.c_uint8), P(f32), P(f32), vp, vp, vp, vp, i32, vp, i32, vp)
_sig("ps_eval_fixed_strategy_adjoint", i32, vp, P(f32), P(f32), P(f32), P(f32), P(f32), P(f32), P(f32))
_sig("ps_num_private_hands", i32, vp, i32)
_sig("ps_private_cards", i32, vp, i32, P(C.c_uint8))
_sig("ps_initial_weights", i32, vp, i32, P(f32))
_sig("ps_num_combinations", f64, vp)
_sig("ps_num_nodes", i64, vp)
_sig("ps_node_info", i32, vp, i64, P(i32))
_sig("ps_child_indices", i32, vp, i64, P(i64), i32)
_sig("ps_strategy_at_index", i32, vp, i64, P(f32))
_sig("ps_node_storage", i64, vp, i64, i32, P(f32))
_sig("ps_seed_node_storage", i32, vp, i64, i32, P(f32), i64)
_sig("ps_same_hand_index", i32, vp, i32, P(C.c_uint16))
_sig("ps_hand_strength", i32, vp, i32, i32, i32, P(C.c_uint16), P(C.c_uint16))
_sig("ps_valid_indices", i32, vp, i32, i32, i32, P(C.c_uint16))
_sig("ps_num_boundary_nodes", i64, vp)
_sig("ps_boundary_node_indices", i32, vp, P(i64))
_sig("ps_set_boundary_cfvs", i32, vp, i64, i32, P(f32), i64)
_sig("ps_back_to_root", i32, vp)
_sig("ps_play", i32, vp, i64)
_sig("ps_available_actions", i32, vp, P(i32), P(i32), i32)
_sig("ps_is_terminal_node", i32, vp)
_sig("ps_is_chance_node", i32, vp)
_sig("ps_current_player", i32, vp)
_sig("ps_current_node_index", i64, vp)
_sig("ps_possible_cards", u64, vp)
_sig("ps_strategy", i32, vp, P(f32))
_sig("ps_cache_normalized_weights", i32, vp)
_sig("ps_weights", i32, vp, i32, i32, P(f32))
_sig("ps_expected_values", i32, vp, i32, i32, P(f32))
_sig("ps_total_bet_amount", i32, vp, P(i32))
_sig("ps_state_export", i32, vp, vp, u64, P(u64))
_sig("ps_state_import", i32, vp, vp, u64)
_sig("ps_batch_new", i32, P(PsCardConfig), P(PsTreeConfig), i32, P(PsBatchOpts), P(vp))
_sig("ps_batch_free", None, vp)
_sig("ps_batch_solve", i32, vp, u32, P(f32))
_sig("ps_batch_results", i32, vp, P(f32), P(i32))
_sig("ps_batch_root_strategy", i32, vp, i32, P(f32))
_sig("ps_batch_root_cfvalues", i32, vp, i32, i32, P(f32))
_sig("ps_batch_num_nodes", i64, vp, i32)
_sig("ps_batch_node_storage", i64, vp, i32, i64, i32, P(f32))
_sig("ps_batch_last_timing", i32, vp, P(f32), P(f32))
_sig("ps_batch_iteration_bytes", f64, vp, i32)
_sig("ps_batch_config", i32, vp, P(i32), P(i32), P(i32))
_sig("ps_batch_autotune_log", i32, vp, P(i32), P(i32), P(f32), i32)
_sig("ps_batch_scan_buffers", i32, vp)
_sig("ps_batch_schedule", i32, vp, P(i32))
_sig("ps_batch_autotune_trials", i32, vp, P(i32), P(f32), i32)
_sig("ps_batch_io_bytes", i32, vp, P(u64), P(u64))
_sig("ps_batch_run_iterations", i32, vp, u32, u32, i32)
_sig("ps_batch_reset", i32, vp)
_sig("ps_batch_num_boundary_items", i64, vp)
_sig("ps_batch_boundary_items", i32, vp, P(i32), P(i32), P(C.c_uint8), P(f32), P(f32))
_sig("ps_batch_set_boundary_cfvs", i32, vp, vp, i32)
_sig("ps_batch_boundary_reach", i32, vp, vp, i32)
_sig("ps_batch_root_cfvalues_all", i32, vp, vp, i32)
_sig("ps_batch_adjoint", i32, vp, vp, vp, vp, i32)
_sig("ps_sample_situations", i32, P(PsSamplerConfig), i64, i32, vp, vp, vp, vp, vp)
_sig("ps_batch_record_bytes", i64, vp)
_sig("ps_batch_records", i32, vp, vp, i32)
_sig("ps_boundary_encode", i32, i32, P(C.c_uint8), P(f32), P(f32), vp, vp, i32, vp)

PS_EPI_ROOT = 1
PS_EPI_EXPL = 2

EXPORTED = sorted(_SIGS)


def lib(build_if_missing: bool = True):
    """Loads the library (building it first if it is missing)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                if not build_if_missing:
                    raise OSError(f"{LIB_PATH} is missing; run poker_solver_rust_b200.build.build()")
                from . import build as _b

                _b.build()
            L = C.CDLL(LIB_PATH)
            for name, (res, args) in _SIGS.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
        return _lib


class SolverError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def check(rc: int) -> int:
    if rc < 0:
        raise SolverError(rc, lib().ps_last_error().decode())
    return rc
