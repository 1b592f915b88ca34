"""Generates tests/golden/reference_pins.json from the reference sources.

Run where a checkout of the reference is present, giving its root:
    python tests/golden/make_golden.py /path/to/poker_solver_rust

It reads crates/range-solver/src/hand_table.rs as text and stores only the
table's length, a SHA-256 digest of its little-endian int32 bytes and its
first/last entries, so the oracle's and the product's regenerated tables can
be pinned without copying the table.  The known answers of the reference's
own tests that the pins use are extracted by pattern from the test sources
(hand.rs, solver.rs, bet_size.rs, examples/basic.rs) and recorded with the
file they came from.
"""

from __future__ import annotations

import hashlib
import json
import os
import re
import struct
import sys

if len(sys.argv) != 2:
    sys.exit("usage: make_golden.py /path/to/poker_solver_rust (the reference checkout's root)")
REF = sys.argv[1]
SRC = os.path.join(REF, "crates", "range-solver", "src")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_pins.json")


def read(rel):
    with open(os.path.join(REF, rel)) as f:
        return f.read()


def main():
    pins = {}
    # ---- HAND_TABLE (hand_table.rs) ----
    txt = read("crates/range-solver/src/hand_table.rs")
    body = txt[txt.index("[", txt.index("=")) + 1: txt.rindex("]")]
    vals = [int(x) for x in re.findall(r"-?\d+", body)]
    raw = b"".join(struct.pack("<i", v) for v in vals)
    pins["hand_table"] = {
        "source": "crates/range-solver/src/hand_table.rs",
        "len": len(vals),
        "sha256_le_i32": hashlib.sha256(raw).hexdigest(),
        "first": vals[:5],
        "last": vals[-3:],
    }
    # ---- exhaustive category counts (hand.rs:440-448) ----
    h = read("crates/range-solver/src/hand.rs")
    counts = {int(k): int(v) for k, v in re.findall(r"assert_eq!\(counter\[(\d)\],\s*(\d+)\)", h)}
    pins["hand_category_counts"] = {"source": "crates/range-solver/src/hand.rs:440-448",
                                    "counts": [counts[i] for i in range(9)]}
    # ---- discount params (solver.rs:688-722) ----
    s = read("crates/range-solver/src/solver.rs")
    pins["discount_params"] = {
        "source": "crates/range-solver/src/solver.rs:688-722",
        "t0": {"alpha": 0.0, "beta": 0.5, "gamma": 0.0},
        "t1": {"alpha": 0.0, "beta": 0.5},
        "t4_gamma": 0.0,
        "t5_gamma": 0.125,
        "t100_alpha_gt": 0.9,
        "present_in_source": all(x in s for x in ("DiscountParams::new(4)", "DiscountParams::new(5)", "0.125")),
    }
    # ---- bet size parser table (bet_size.rs tests) ----
    b = read("crates/range-solver/src/bet_size.rs")
    ok = re.findall(r'\("([^"]*)",\s*(PotRelative|PrevBetRelative|Additive|Geometric|AllIn)(\(([^)]*)\))?\)', b)
    table = []
    for s_, kind, _, args in ok:
        args = [a.strip() for a in args.split(",")] if args else []
        table.append([s_, kind, args])
    err_block = b[b.index("let error_tests = ["): ]
    err_block = err_block[: err_block.index("];")]
    errs = re.findall(r'"([^"]*)"', err_block)
    pins["bet_size_from_str"] = {"source": "crates/range-solver/src/bet_size.rs:252-290", "ok": table,
                                 "errors": errs}
    # ---- examples/basic.rs ----
    e = read("crates/range-solver/examples/basic.rs")
    pins["basic_example"] = {
        "source": "crates/range-solver/examples/basic.rs",
        "oop_range": re.search(r'let oop_range = "([^"]+)"', e).group(1),
        "ip_range": re.search(r'let ip_range = "([^"]+)"', e).group(1),
        "flop": re.search(r'flop_from_str\("([^"]+)"\)', e).group(1),
        "turn": re.search(r'turn: card_from_str\("([^"]+)"\)', e).group(1),
        "bet_sizes": list(re.search(r'BetSizeOptions::try_from\(\("([^"]*)",\s*"([^"]*)"\)\)', e).groups()),
        "river_donk": re.search(r'river_donk_sizes: Some\(DonkSizeOptions::try_from\("([^"]*)"\)', e).group(1),
        "starting_pot": int(re.search(r"starting_pot: (\d+)", e).group(1)),
        "effective_stack": int(re.search(r"effective_stack: (\d+)", e).group(1)),
        "add_allin_threshold": float(re.search(r"add_allin_threshold: ([\d.]+)", e).group(1)),
        "force_allin_threshold": float(re.search(r"force_allin_threshold: ([\d.]+)", e).group(1)),
        "merging_threshold": float(re.search(r"merging_threshold: ([\d.]+)", e).group(1)),
        "oop_first10": re.findall(r'"(\w\w\w\w)"', e[e.index("&oop_cards_str[..10]"):e.index("// check memory")]),
        "root_actions": re.search(r'"(\[Check[^"]*\])"', e).group(1),
        "after_bet_actions": re.search(r'"(\[Fold[^"]*\])"', e).group(1),
        "ip_hands": int(re.search(r"assert_eq!\(ip_cards.len\(\), (\d+)\)", e).group(1)),
        "strategy_len": int(re.search(r"assert_eq!\(strategy.len\(\), (\d+)\)", e).group(1)),
        "max_iterations": int(re.search(r"let max_num_iterations = (\d+)", e).group(1)),
        "target_fraction_of_pot": 0.005,
    }
    with open(OUT, "w") as f:
        json.dump(pins, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
