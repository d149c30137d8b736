"""Generates the oracle's first-found rule sets at the configured parity sizes.

  c2_100k_oracle.json  the 100,000-target C2 subset (seed 0, drawn by index
                       from the 9,818,041 unpruned length-2 targets over the
                       8-bit instruction list), candidates of one
                       instruction, dead flags 0x00 and 0xFF
  c1_full_oracle.json  every unpruned length-2 target over the C1 pool
                       (53,951 targets), candidates of one instruction,
                       dead flags 0x00

Each rule is [target_index, source words, replacement words, bytes_saved,
cycles_saved, dead_flags]; `checked` is the reference's counter
(pkg/search/worker.go:134) summed over the targets.  Targets are enumerated
by the oracle itself (EnumerateSequences8 order + ShouldPrune) and a digest
of the target array is stored, so a test can confirm it runs the same
targets.  The oracle is a CPU restatement of pkg/search (worker.go:124-265);
this takes a few minutes on 8 cores:

    python tests/golden/make_parity_fixtures.py [--only c2|c1]
"""
import argparse
import hashlib
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import oracle_lib as O  # noqa: E402


def digest(arr):
    return hashlib.sha256(arr.astype("<u4").tobytes()).hexdigest()


def rules_json(rules):
    return [[r.target_index, list(r.src[:r.src_len]), list(r.rep[:r.rep_len]), r.bytes_saved,
             r.cycles_saved, r.dead_flags] for r in rules]


def run(targets, dead):
    t0 = time.perf_counter()
    rules, checked = O.search([list(map(int, row)) for row in targets], 1, dead=dead)
    secs = time.perf_counter() - t0
    print(f"  dead {dead:#04x}: {len(rules)} rules, checked {checked}, {secs:.1f} s", flush=True)
    return {"dead_flags": dead, "checked": checked, "rules": rules_json(rules)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=["c2", "c1"])
    a = ap.parse_args()
    if a.only in (None, "c2"):
        t = O.c2_subset(100000, seed=0)
        print(f"C2 subset: {len(t)} targets", flush=True)
        out = {"workload": "C2 subset: 100,000 of the 9,818,041 unpruned length-2 targets over the 8-bit "
                           "instruction list, drawn by index with numpy default_rng(0), in index order",
               "n_targets": int(len(t)), "targets_sha256": digest(t), "max_cand_len": 1,
               "passes": [run(t, 0x00), run(t, 0xFF)]}
        with open(os.path.join(HERE, "c2_100k_oracle.json"), "w") as f:
            json.dump(out, f, separators=(",", ":"))
    if a.only in (None, "c1"):
        t = O.c1_targets()
        print(f"C1: {len(t)} targets", flush=True)
        out = {"workload": "C1: every unpruned length-2 target over the small plain pool (imm8 set "
                           "{00,01,7F,80,FF} + 3 bytes of splitmix64(0))",
               "n_targets": int(len(t)), "targets_sha256": digest(t), "max_cand_len": 1,
               "passes": [run(t, 0x00)]}
        with open(os.path.join(HERE, "c1_full_oracle.json"), "w") as f:
            json.dump(out, f, separators=(",", ":"))


if __name__ == "__main__":
    main()
