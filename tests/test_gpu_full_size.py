"""The bench workload at its full size: 4096 datagen river spots in one
persistent launch, checked through properties that hold at any size, plus a
sample of spots against the single-game path bit for bit.

- Stopping: every spot ends as the reference loop does (solver.rs:108-176):
  exploitability <= 0.3% of the pot at a check, or 300 iterations.
- Zero sum: the spots are unraked, so under one strategy profile the two
  players' root values cancel: sum w0 * cfv0 + sum w1 * cfv1 = 0.  Tolerance
  1e-4 of sum |w0 * cfv0| + sum |w1 * cfv1| (f32 sweeps).
- Root strategies are distributions over the actions, within 1e-5.
- Records: two per spot, game_value = sum(range * cfvs) in f32 order.
"""

import numpy as np
import pytest

import poker_solver_rust_b200 as ps
from tests import spots

pytestmark = pytest.mark.gpu

N_SPOTS = 4096


def test_full_datagen_batch_properties():
    sp = spots.datagen_spots(N_SPOTS, seed=7)
    tcs = [t for _, _, t in sp]
    bs = ps.BatchSolver([spots.card_config(r, b) for r, b, _ in sp], tcs)
    targets = np.array([0.003 * t.starting_pot for t in tcs], np.float32)
    bs.solve(300, targets)
    e, it = bs.results()
    assert ((e <= targets) | (it == 300)).all()
    stopped = (e <= targets) & (it < 300)
    assert (it[stopped] % 5 == 0).all()  # the target is met at a check
    cfv = bs.root_cfvalues_all().astype(np.float64)
    ranges = np.stack([np.stack(r) for r, _, _ in sp]).astype(np.float64)
    v = (ranges * cfv).sum(axis=2)
    scale = np.abs(ranges * cfv).sum(axis=(1, 2))
    assert (np.abs(v.sum(axis=1)) <= 1e-4 * np.maximum(scale, 1e-30)).all()
    for i in range(0, N_SPOTS, 97):
        H = int(np.count_nonzero(ranges[i, 0]))  # the root actor (OOP) holds every combo with weight
        s = bs.root_strategy(i)
        assert s.size % H == 0
        assert np.allclose(s.reshape(-1, H).sum(axis=0), 1.0, atol=1e-5)
    recs = bs.records()
    assert len(recs) == 2 * N_SPOTS
    gv = np.add.accumulate((recs["oop_range"] * recs["cfvs"]).astype(np.float32), axis=1, dtype=np.float32)
    assert np.array_equal(gv[0::2, -1], recs["game_value"][0::2])
    # sampled spots against the single-game path, bit for bit
    for i in (0, 1234, 4095):
        r, b, t = sp[i]
        g = spots.product_game(r, b, t)
        assert ps.solve(g, 300, float(targets[i])) == e[i] and g.last_iterations == it[i]
        for p in range(2):
            assert np.array_equal(bs.root_cfvalues(i, p), ps.root_cfvalues(g, p))
