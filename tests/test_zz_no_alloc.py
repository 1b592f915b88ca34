"""The allocation-free exploitability entry point against the allocating one.

Some callers of this library may not allocate GPU memory when they evaluate a
game: an engine that reserves the device's memory for its own pool at start-up
and hands each plug-in a fixed share, or a caller on a latency-bound thread
where cudaMalloc's implicit device synchronisation is not allowed.
ps_compute_exploitability_noalloc serves them: it runs the same kernel as
ps_compute_exploitability with its working slots in the library's fixed
device array.  Both are called through the C ABI on the same game state and
must agree within the tolerance the one-step parity tests use for
exploitability; the fixed array keeps the previous call's contents, so each
game is evaluated twice in a row and games of different sizes alternate.
The entry point's one promise - it allocates nothing - is checked through the
driver's free-memory count, and a device reset between calls (a new CUDA
context, in which the array has a new address) in a child process.
"""

import ctypes as C
import os
import subprocess
import sys
import textwrap

import pytest

import poker_solver_rust_b200 as ps
from poker_solver_rust_b200 import _native as N
from tests import spots

pytestmark = pytest.mark.gpu

TOL_EVAL_REL = 2e-5  # exploitability from one state, relative (as in the parity tests)
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


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


def test_noalloc_allocates_nothing():
    import torch

    r, b, t = spots.river_spot(6)
    g = spots.product_game(r, b, t)
    for it in range(3):
        ps.solve_step(g, it)
    ref = _check(g, t.starting_pot)  # first calls: the kernel's launch resources exist from here on
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    vals = [_expl("ps_compute_exploitability_noalloc", g) for _ in range(8)]
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert all(abs(v - ref) <= TOL_EVAL_REL * max(abs(ref), 0.1) for v in vals)


_RESET_CHILD = textwrap.dedent("""
    import ctypes as C, sys
    sys.path.insert(0, {root!r})
    import poker_solver_rust_b200 as ps
    from poker_solver_rust_b200 import _native as N
    from tests import spots

    def values():
        r, b, t = spots.river_spot(3)
        g = spots.product_game(r, b, t)
        for it in range(4):
            ps.solve_step(g, it)
        out = []
        for name in ("ps_compute_exploitability", "ps_compute_exploitability_noalloc",
                     "ps_compute_exploitability_noalloc"):
            x = C.c_float()
            N.check(getattr(N.lib(), name)(g._h, C.byref(x)))
            out.append(x.value)
        return out

    before = values()
    # the CUDA runtime the library itself loaded (one instance per process)
    path = [l.split()[-1] for l in open("/proc/self/maps") if "libcudart.so" in l][0]
    assert C.CDLL(path).cudaDeviceReset() == 0
    after = values()
    print(repr((before, after)))
""")


def test_noalloc_after_device_reset():
    """A device reset ends the CUDA context the fixed array's address was
    looked up in; the next call must look it up again (and the library's other
    per-device caches must follow), or it would launch on a stale address."""
    res = subprocess.run([sys.executable, "-c", _RESET_CHILD.format(root=ROOT)], capture_output=True, text=True,
                         timeout=300, cwd=ROOT)
    assert res.returncode == 0, res.stderr[-2000:]
    before, after = eval(res.stdout.strip().splitlines()[-1])
    ref = before[0]
    for v in before[1:] + after:
        assert abs(v - ref) <= TOL_EVAL_REL * max(abs(ref), 0.1), (before, after)
    assert after[0] == before[0]  # the same game from scratch: the same bits
