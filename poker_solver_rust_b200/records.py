"""Training records of solved spots in the reference's binary format.

Format (cfvnet datagen/storage.rs:5-57, little endian, packed):
``[board_size u8][board u8 x board_size][pot f32][effective_stack f32]
[player u8][game_value f32][oop_range f32 x1326][ip_range f32 x1326]
[cfvs f32 x1326][valid_mask u8 x1326]``.

``BatchSolver.records()`` packs them on the device (``ps_batch_records``);
``RecordWriter`` appends them to files with the reference's per-file rotation
(datagen/domain/writer.rs:8-83); ``read_records`` loads a file as a numpy
structured array.
"""

from __future__ import annotations

import os

import numpy as np

NUM_COMBOS = 1326


def record_size(board_size: int) -> int:
    """storage.rs:9-21."""
    return 1 + board_size + 4 + 4 + 1 + 4 + 3 * NUM_COMBOS * 4 + NUM_COMBOS


def record_dtype(board_size: int) -> np.dtype:
    """Packed numpy dtype of one record (itemsize == record_size(board_size))."""
    return np.dtype([("board_size", "u1"), ("board", "u1", (board_size,)), ("pot", "<f4"),
                     ("effective_stack", "<f4"), ("player", "u1"), ("game_value", "<f4"),
                     ("oop_range", "<f4", (NUM_COMBOS,)), ("ip_range", "<f4", (NUM_COMBOS,)),
                     ("cfvs", "<f4", (NUM_COMBOS,)), ("valid_mask", "u1", (NUM_COMBOS,))])


def read_records(path: str, board_size: int) -> np.ndarray:
    """All records of a file with one board size (storage.rs:60-110, :114-118)."""
    data = np.fromfile(path, dtype=np.uint8)
    if data.size % record_size(board_size):
        raise ValueError(f"{path}: {data.size} bytes is not a whole number of {board_size}-card records")
    recs = data.view(record_dtype(board_size))
    if recs.size and (recs["board_size"] != board_size).any():
        raise ValueError(f"{path}: board size prefix differs from {board_size}")
    return recs


class RecordWriter:
    """Appends packed records to ``path``; with ``per_file`` set, starts a new
    file ``{stem}_{index:05}.bin`` beside it every ``per_file`` records
    (writer.rs:30-83)."""

    def __init__(self, path: str, per_file: int | None = None):
        self.base = path
        self.per_file = per_file
        self.file_index = 0
        self.records_in_file = 0
        self.total_count = 0
        self._f = open(self._path(0), "wb")

    def _path(self, index: int) -> str:
        if index == 0:
            return self.base
        stem = os.path.splitext(os.path.basename(self.base))[0]
        return os.path.join(os.path.dirname(self.base) or ".", f"{stem}_{index:05d}.bin")

    def write(self, records: np.ndarray) -> None:
        """records: a structured array of record_dtype."""
        recs = np.ascontiguousarray(records)
        k = 0
        while k < len(recs):
            if self.per_file is not None and self.records_in_file >= self.per_file:
                self._rotate()
            take = len(recs) - k if self.per_file is None else min(len(recs) - k,
                                                                    self.per_file - self.records_in_file)
            self._f.write(recs[k:k + take].tobytes())
            k += take
            self.records_in_file += take
            self.total_count += take

    def _rotate(self) -> None:
        self._f.close()
        self.file_index += 1
        self._f = open(self._path(self.file_index), "wb")
        self.records_in_file = 0

    def count(self) -> int:
        return self.total_count

    def flush(self) -> None:
        self._f.flush()

    def close(self) -> None:
        self._f.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
