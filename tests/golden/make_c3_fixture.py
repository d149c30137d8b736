"""Regenerates c3_oracle.json: first-found rules (pkg/search worker.go
semantics, candidates up to 2 instructions, per-target dead flags and the
dead-register extension) of the CPU oracle for a seeded C3 sample.

    python tests/golden/make_c3_fixture.py [n_targets] [workers]

The sample is workloads.c3_targets(n, seed=1); the fixture stores the targets
with their masks, the rules grouped by target index, and the reference's
'checked' counter, so the GPU tests compare without rerunning the oracle.
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "..", "z80-optimizer_b200"))

import oracle_lib  # noqa: E402
import workloads  # noqa: E402


def main():
    n = int(sys.argv[1]) if len(sys.argv) > 1 else 240
    workers = int(sys.argv[2]) if len(sys.argv) > 2 else os.cpu_count()
    arr, lens, dead, dregs = workloads.c3_targets(n, seed=1)
    targets = [list(map(int, arr[i, :lens[i]])) for i in range(n)]
    t0 = time.time()
    rules, checked = oracle_lib.search_ext(targets, 2, dead=list(map(int, dead)), dregs=list(map(int, dregs)),
                                           workers=workers)
    print(f"{len(rules)} rules, checked {checked}, {time.time() - t0:.1f} s", flush=True)
    doc = {"_about": "oracle first-found rules for workloads.c3_targets(n, seed=1), max_cand_len 2; "
                     "generated by make_c3_fixture.py",
           "n": n, "seed": 1, "max_cand_len": 2, "checked": checked,
           "targets": targets, "dead_flags": list(map(int, dead)), "dead_regs": list(map(int, dregs)),
           "rules": [[r.target_index, list(r.src[:r.src_len]), list(r.rep[:r.rep_len]), r.bytes_saved,
                      r.cycles_saved, r.dead_flags, r.dead_regs] for r in rules]}
    with open(os.path.join(HERE, "c3_oracle.json"), "w") as f:
        json.dump(doc, f)


if __name__ == "__main__":
    main()
