"""Training records packed on the device (ps_batch_records) against the
oracle's restatement of the reference's GPU river datagen record assembly
(cfvnet datagen/domain/pipeline.rs:353-411), byte for byte, from the same
root cfvalues; and the file written by RecordWriter reads back the same."""

import numpy as np
import pytest

import poker_solver_rust_b200 as ps
from oracle.records import spot_records
from poker_solver_rust_b200 import records as R
from tests import spots

pytestmark = pytest.mark.gpu


def test_batch_records_match_restatement(tmp_path):
    sp = spots.datagen_spots(12, seed=61)
    bs = ps.BatchSolver([spots.card_config(r, b) for r, b, _ in sp], [t for _, _, t in sp])
    bs.solve(300, np.array([0.003 * t.starting_pot for _, _, t in sp], np.float32))
    recs = bs.records()
    assert recs.dtype == R.record_dtype(5) and len(recs) == 2 * len(sp)
    for i, (r, b, t) in enumerate(sp):
        g = spots.product_game(r, b, t)
        hands = [np.array([ps.card_pair_to_index(int(x), int(y)) for x, y in g.private_cards(p)])
                 for p in range(2)]
        cfv = [bs.root_cfvalues(i, p) for p in range(2)]
        ref = spot_records(cfv, hands, np.stack(r), b, t.starting_pot, t.effective_stack, g.num_combinations())
        assert recs[2 * i:2 * i + 2].tobytes() == ref.tobytes(), i
    with R.RecordWriter(str(tmp_path / "river.bin")) as w:
        w.write(recs)
    back = R.read_records(str(tmp_path / "river.bin"), 5)
    assert back.tobytes() == recs.tobytes()
