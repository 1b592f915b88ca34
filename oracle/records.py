"""ORACLE — test infrastructure only.

numpy restatement of the training records of the reference's GPU river
datagen (crates/cfvnet/src/datagen/domain/pipeline.rs:353-411) from each
player's root cfvalues, in the binary format of datagen/storage.rs:5-57.
Only ``tests/`` may import this module, as the checker of the device packer.
"""

from __future__ import annotations

import numpy as np

from poker_solver_rust_b200.records import record_dtype


def spot_records(root_cfv, hands, ranges, board, pot: float, stack: float, num_combinations: float):
    """Two records (player 0, player 1).  root_cfv[p]: [H_p] root cfvalues in
    per-combination units; hands[p]: [H_p] combo indices; ranges: [2, 1326]."""
    half = float(pot) / 2.0
    norm = half if half > 0.0 else 1.0
    comb = np.float32(num_combinations)
    cfvs = np.zeros((2, 1326), np.float32)
    mask = np.zeros(1326, np.uint8)  # one mask for both records: either player's hands
    for p in range(2):
        ev = (np.asarray(root_cfv[p], np.float32) * comb).astype(np.float32)  # f32 product
        cfvs[p, hands[p]] = ((ev.astype(np.float64) - half) / norm).astype(np.float32)
        mask[hands[p]] = 1
    recs = np.zeros(2, record_dtype(len(board)))
    for p in range(2):
        prod = (np.asarray(ranges[p], np.float32) * cfvs[p]).astype(np.float32)
        gv = np.add.accumulate(prod, dtype=np.float32)[-1]  # left fold in f32, combo order
        r = recs[p]
        r["board_size"] = len(board)
        r["board"] = board
        r["pot"] = np.float32(pot)
        r["effective_stack"] = np.float32(stack)
        r["player"] = p
        r["game_value"] = gv
        r["oop_range"] = ranges[0]
        r["ip_range"] = ranges[1]
        r["cfvs"] = cfvs[p]
        r["valid_mask"] = mask
    return recs
