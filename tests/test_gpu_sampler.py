"""Situations drawn on the device (ps_sample_situations) against the
oracle's restatement of the reference's sampler (cfvnet datagen/sampler.rs,
datagen/range_gen.rs) on the same SplitMix64 stream: boards, pots and stacks
exactly, ranges bit for bit; then a batch built from them solves."""

import numpy as np
import pytest

import poker_solver_rust_b200 as ps
from oracle import sampler as S
from poker_solver_rust_b200.sampler import SamplerConfig, sample_situations, to_spot_configs

pytestmark = pytest.mark.gpu

CASES = [
    (SamplerConfig(board_size=5, seed=11), 100, 6),
    (SamplerConfig(board_size=5, initial_stack=400, pot_intervals=[[4, 40], [40, 120], [120, 400]],
                   spr_intervals=[[0.0, 1.0], [1.0, 3.0], [3.0, 8.0]], seed=3), 0, 4),
    (SamplerConfig(board_size=4, seed=5), 7, 2),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_sampler_matches_restatement(case):
    cfg, first, n = CASES[case]
    got = sample_situations(cfg, first, n)
    b = got["boards"].cpu().numpy()
    pots = got["pots"].cpu().numpy()
    stacks = got["stacks"].cpu().numpy()
    rg = got["ranges"].cpu().numpy()
    for i in range(n):
        ref = S.sample_situation(cfg.board_size, cfg.initial_stack, cfg.pot_intervals, cfg.spr_intervals,
                                 cfg.seed, first + i)
        assert ref is not None
        board, pot, stack, ranges = ref
        assert list(b[i]) == board and pots[i] == pot and stacks[i] == stack
        assert np.array_equal(rg[i].view(np.uint32), ranges.view(np.uint32)), i
    # a chunk of the stream equals the same situations drawn in one call
    whole = sample_situations(cfg, first, n + 2)
    assert np.array_equal(whole["ranges"].cpu().numpy()[:n], rg)


def test_sampler_rejects_infeasible_intervals():
    cfg = SamplerConfig(board_size=5, initial_stack=10, spr_intervals=[[50.0, 60.0]], seed=1)
    with pytest.raises(ps.SolverError):
        sample_situations(cfg, 0, 3)
    with pytest.raises(ps.SolverError):
        sample_situations(SamplerConfig(board_size=3), 0, 1)


def test_sampled_spots_solve():
    cfg = SamplerConfig(board_size=5, seed=21)
    sit = sample_situations(cfg, 0, 16)
    sizes = ps.BetSizeOptions("50%, 100%, a", "100%")

    def tree(pot, stack):
        return ps.TreeConfig(initial_state=ps.BoardState.River, starting_pot=pot, effective_stack=stack,
                             river_bet_sizes=[sizes, sizes])

    cards, trees = to_spot_configs(sit, tree)
    bs = ps.BatchSolver(cards, trees)
    bs.solve(300, np.array([0.003 * t.starting_pot for t in trees], np.float32))
    e, it = bs.results()
    assert np.all(np.isfinite(e)) and (it > 0).all()
    recs = bs.records()
    assert len(recs) == 32 and np.allclose(recs["oop_range"][::2].sum(axis=1), 1.0, atol=1e-5)
