"""The allocation-free exploitability entry point against the allocating one.

ps_compute_exploitability_noalloc runs the same kernel as
ps_compute_exploitability with its working slots in the library's fixed
device array.  Both are called through the C ABI on the same game state and
must agree within the tolerance the one-step parity tests use for
exploitability; the fixed array keeps the previous call's contents, so each
game is evaluated twice in a row and games of different sizes alternate.
"""

import ctypes as C

import pytest

import poker_solver_rust_b200 as ps
from poker_solver_rust_b200 import _native as N
from tests import spots

pytestmark = pytest.mark.gpu

TOL_EVAL_REL = 2e-5  # exploitability from one state, relative (as in the parity tests)


def _expl(name, g):
    out = C.c_float()
    N.check(getattr(N.lib(), name)(g._h, C.byref(out)))
    return out.value


def _check(g, pot):
    ref = _expl("ps_compute_exploitability", g)
    first = _expl("ps_compute_exploitability_noalloc", g)
    second = _expl("ps_compute_exploitability_noalloc", g)
    for v in (first, second):
        assert abs(v - ref) <= TOL_EVAL_REL * max(abs(ref), 1e-3 * pot), (v, ref)
    return ref


def test_noalloc_matches_allocating_path():
    r, b, t = spots.river_spot(3)
    small = spots.product_game(r, b, t)
    r2, b2, t2 = spots.river_spot(11)
    t2.effective_stack *= 3  # deeper tree: more slots than the first game
    big = spots.product_game(r2, b2, t2)
    for it in range(5):
        ps.solve_step(small, it)
        ps.solve_step(big, it)
    _check(small, t.starting_pot)
    _check(big, t2.starting_pot)
    for it in range(5, 12):
        ps.solve_step(small, it)
    _check(small, t.starting_pot)


def test_noalloc_rejects_games_beyond_the_fixed_array():
    r, b, t = spots.turn_spot(4)
    g = spots.product_game(r, b, t)
    ps.solve_step(g, 0)
    out = C.c_float()
    rc = N.lib().ps_compute_exploitability_noalloc(g._h, C.byref(out))
    assert rc == -1 and b"fixed array" in N.lib().ps_last_error()
    assert _expl("ps_compute_exploitability", g) > 0  # the allocating path still serves it
