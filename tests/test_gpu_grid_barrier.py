"""The bounded wait of the grid barrier (single-game grid mode) on the GPU.

A grid-mode launch ends each step in a grid barrier across its cooperative
CTAs.  If a CTA never arrives, the waiting CTAs must give up after a bounded
time, report the wait error (bit 4 of the launch's error word) and abort the
launch: every later barrier returns at once, so the kernel ends instead of
timing out once per remaining barrier.  The test hook launches CTAs of which
only CTA 0 enters the barriers; nothing else sets the generation word, so the
first wait runs out on purpose, within its 20 ms limit.
"""

import ctypes as C

import pytest

from poker_solver_rust_b200 import _native as N

ERR_WAIT = 4


@pytest.mark.gpu
@pytest.mark.parametrize("ctas", [2, 8])
def test_grid_barrier_gives_up_and_aborts(ctas):
    err, passed, ms = C.c_int32(), C.c_int32(), C.c_float()
    rounds, wait_ns = 1000, 20_000_000
    N.check(N.lib().ps_debug_grid_barrier_timeout(ctas, rounds, wait_ns, 0, C.byref(err), C.byref(passed),
                                                  C.byref(ms)))
    assert err.value == ERR_WAIT
    assert passed.value == 0  # the first barrier failed, and the 999 after it returned at once
    # one wait of 20 ms, not 1000 of them
    assert 15.0 <= ms.value <= 500.0, ms.value


def test_grid_barrier_hook_rejects_unbounded_waits():  # argument check only: no GPU needed
    err, passed, ms = C.c_int32(), C.c_int32(), C.c_float()
    rc = N.lib().ps_debug_grid_barrier_timeout(2, 1, 2_000_000_000, 0, C.byref(err), C.byref(passed), C.byref(ms))
    assert rc == -1


@pytest.mark.gpu
def test_grid_barrier_cost_when_every_cta_joins():
    """Every CTA (one per SM) joins every barrier: none times out, all pass,
    and the time per barrier is reported for the grid-mode step cost."""
    import torch

    nsm = torch.cuda.get_device_properties(0).multi_processor_count
    err, passed, ms = C.c_int32(), C.c_int32(), C.c_float()
    rounds = 2000
    N.check(N.lib().ps_debug_grid_barrier_timeout(nsm, rounds, 1_000_000_000, 1, C.byref(err), C.byref(passed),
                                                  C.byref(ms)))
    assert err.value == 0 and passed.value == rounds
    us = 1e3 * ms.value / rounds
    print(f"grid barrier over {nsm} CTAs: {us:.2f} us")
    assert us < 50.0
