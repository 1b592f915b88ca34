"""The dataflow batched solve (k_flow) against the step-synchronous one (k_solve).

Both run every item (a terminal run, a node op or one of its column blocks)
with the same arithmetic; only which warp runs it and when differs.  So the
results must be the same bits: per-spot exploitability and iteration count,
root cfvalues, regrets and strategy sums, and for depth-limited spots the
boundary reach - for every launch shape (threads per CTA, spots per CTA,
node-op parts, scan buffers), for solves to a target and for fixed iteration
ranges with their epilogues.
"""

import numpy as np
import pytest

import poker_solver_rust_b200 as ps
from tests import spots

pytestmark = pytest.mark.gpu

STEP, FLOW = 1, 2


def _batch(sp, **kw):
    return ps.BatchSolver([spots.card_config(r, b) for r, b, _ in sp], [t for _, _, t in sp], **kw)


def _state(bs, n, picks):
    out = []
    for i in picks:
        for k in range(bs.num_nodes(i)):
            for which in (1, 2):
                v = bs.node_storage(i, k, which)
                if len(v):
                    out.append(v)
    return np.concatenate(out)


@pytest.fixture(scope="module")
def datagen():
    sp = spots.datagen_spots(320, seed=41)
    targets = np.array([0.003 * t.starting_pot for _, _, t in sp], np.float32)
    ref = _batch(sp, scheduler=STEP)
    assert ref.config()["scheduler"] == "step-synchronous"
    ref.solve(300, targets)
    picks = [0, 7, 100, 319]
    return sp, targets, ref.results(), ref.root_cfvalues_all(), _state(ref, len(sp), picks), picks


@pytest.mark.parametrize("threads,lanes,parts,bufs", [(256, 1, 1, 0), (512, 2, 1, 0), (512, 2, 2, 16),
                                                      (1024, 4, 2, 0), (1024, 8, 3, 16), (128, 3, 1, 2)])
def test_flow_solve_matches_step_synchronous(datagen, threads, lanes, parts, bufs):
    sp, targets, (e_ref, it_ref), cfv_ref, st_ref, picks = datagen
    bs = _batch(sp, scheduler=FLOW, flow_threads=threads, flow_spots_per_cta=lanes, node_parts=parts,
                scan_buffers=bufs)
    cfg = bs.config()
    assert cfg["scheduler"] == "dataflow" and cfg["spots_per_cta"] == lanes and cfg["node_parts"] == parts
    bs.solve(300, targets)
    e, it = bs.results()
    assert np.array_equal(it, it_ref)
    assert np.array_equal(e, e_ref)
    assert np.array_equal(bs.root_cfvalues_all(), cfv_ref)
    assert np.array_equal(_state(bs, len(sp), picks), st_ref)
    # a second solve of the same batch from a fresh state gives the same again
    bs.solve(300, targets)
    assert np.array_equal(bs.results()[1], it_ref)


def test_flow_is_the_default_for_large_batches(datagen):
    sp = datagen[0]
    assert _batch(sp).config()["scheduler"] == "dataflow"
    assert _batch(sp[:8]).config()["scheduler"] == "step-synchronous"


def test_flow_raked_spots_match():
    sp = spots.datagen_spots(200, seed=43)
    for _, _, t in sp:
        t.rake_rate, t.rake_cap = 0.05, 0.5 * t.starting_pot
    targets = np.array([0.003 * t.starting_pot for _, _, t in sp], np.float32)
    ref = _batch(sp, scheduler=STEP)
    ref.solve(120, targets)
    bs = _batch(sp, scheduler=FLOW, flow_threads=512, flow_spots_per_cta=3, node_parts=2)
    bs.solve(120, targets)
    assert np.array_equal(bs.results()[1], ref.results()[1])
    assert np.array_equal(bs.results()[0], ref.results()[0])
    assert np.array_equal(bs.root_cfvalues_all(), ref.root_cfvalues_all())


def test_flow_iteration_ranges_with_boundaries_match():
    """Depth-limited turn spots: boundary values set, iterations [0, 20) with
    the root epilogue (root cfvalues and boundary reach) and the closing
    exploitability, then [20, 32) continuing from that state."""
    sp = spots.turn_boundary_spots(200, seed=44)
    rng = np.random.default_rng(45)
    out = []
    for kw in ({"scheduler": STEP}, {"scheduler": FLOW, "flow_threads": 512, "flow_spots_per_cta": 2},
               {"scheduler": FLOW, "flow_threads": 1024, "flow_spots_per_cta": 4, "node_parts": 2}):
        bs = _batch(sp, **kw)
        if not out:
            V = spots.boundary_values(rng, bs)
        bs.set_boundary_cfvs(V)
        bs.run_iterations(0, 20, root=True, exploitability=True)
        r1 = (bs.results(), bs.root_cfvalues_all(), bs.boundary_reach())
        bs.run_iterations(20, 32, root=True, exploitability=False)
        r2 = (bs.root_cfvalues_all(), bs.boundary_reach(), _state(bs, len(sp), [0, 199]))
        out.append((r1, r2))
    (a1, a2) = out[0]
    for b1, b2 in out[1:]:
        assert np.array_equal(a1[0][0], b1[0][0]) and np.array_equal(a1[0][1], b1[0][1])
        for x, y in zip(a1[1:], b1[1:]):
            assert np.array_equal(x, y)
        for x, y in zip(a2, b2):
            assert np.array_equal(x, y)


def test_flow_autotune_keeps_results_and_picks_the_fastest(datagen):
    sp, targets, (e_ref, it_ref), cfv_ref, _, _ = datagen
    bs = _batch(sp, block_threads=-1)
    trials = bs.autotune_trials()
    cfg = bs.config()
    assert cfg["scheduler"] == "dataflow"
    if trials:  # a fresh choice (not from the per-device cache)
        assert all(t["spots_per_cta"] > 0 for t in trials)
        refine = [t for t in trials if t["stage"] == "refine"]
        best = min(refine or trials, key=lambda t: t["trial_ms"])
        assert (best["block_threads"], best["scan_buffers"], best["spots_per_cta"], best["node_parts"]) == \
            (cfg["block_threads"], cfg["scan_buffers"], cfg["spots_per_cta"], cfg["node_parts"])
    bs.solve(300, targets)
    assert np.array_equal(bs.results()[1], it_ref)
    assert np.array_equal(bs.root_cfvalues_all(), cfv_ref)
