"""Batches built while another batch solves (needs a B200).

A datagen job builds batch k + 1 on one host thread while batch k solves on
another.  The build then runs beside a kernel that holds every SM: its device
buffers come from the library's stream-ordered pool, its stream and events
from the stream pool, and its uploads from pinned staging.  These tests check
that a batch built that way, and the batch solving meanwhile, give exactly the
results of batches built and solved one at a time.
"""

import threading

import numpy as np
import pytest

import poker_solver_rust_b200 as ps
from tests import spots

pytestmark = pytest.mark.gpu


def _inputs(n, seed):
    sp = spots.datagen_spots(n, seed=seed)
    cc = [spots.card_config(r, b) for r, b, _ in sp]
    tcs = [t for _, _, t in sp]
    targets = np.array([0.003 * t.starting_pot for t in tcs], np.float32)
    return cc, tcs, targets


def _results(bs):
    e, it = bs.results()
    return e, it, bs.root_cfvalues_all()


def test_batch_built_while_another_solves_matches_serial():
    # more spots than SMs: the dataflow kernel, which holds every SM while it runs
    cc, tcs, targets = _inputs(600, seed=41)
    ref = ps.BatchSolver(cc, tcs)
    ref.solve(300, targets)
    want = _results(ref)
    del ref

    running = ps.BatchSolver(cc, tcs)
    errors = []

    def solve_running():
        try:
            running.solve(300, targets)
        except Exception as ex:  # surfaced on the main thread below
            errors.append(ex)

    for _ in range(3):  # later rounds reuse pooled streams, events and buffers
        th = threading.Thread(target=solve_running)
        th.start()
        built = ps.BatchSolver(cc, tcs)  # built while `running` solves
        th.join()
        assert not errors, errors
        for got in (_results(running), None):
            if got is None:
                built.solve(300, targets)
                got = _results(built)
            assert np.array_equal(got[0], want[0])
            assert np.array_equal(got[1], want[1])
            assert np.array_equal(got[2], want[2])
        del built


def test_boundary_batch_built_while_another_solves_reads_zero_boundaries():
    """Depth-limited spots built beside a running solve: their boundary region
    is still cleared before use (unset boundary values read as zero)."""
    r, b, t = spots.turn_spot(9)
    t.depth_limit = 0
    cc_b, tcs_b = [spots.card_config(r, b)] * 4, [t] * 4
    ref = ps.BatchSolver(cc_b, tcs_b)
    ref.run_iterations(0, 10, root=True)
    want = ref.root_cfvalues_all()
    del ref

    cc, tcs, targets = _inputs(600, seed=42)
    running = ps.BatchSolver(cc, tcs)
    th = threading.Thread(target=lambda: running.solve(300, targets))
    th.start()
    built = ps.BatchSolver(cc_b, tcs_b)
    th.join()
    built.run_iterations(0, 10, root=True)
    assert np.array_equal(built.root_cfvalues_all(), want)
