"""Small, fixed search case for profiler captures of the sweep kernel.

Runs the first-found search (pkg/search/worker.go:124-265 semantics) on a
seeded sample of the length-2 target set through the library's public API,
`--steps` times, and prints one line of statistics per step.  The case is
sized to keep a full-metric-set capture of one k_exhaustive launch short:

    python z80-optimizer_b200/profile_case.py --targets 30000 --seed 3 --steps 2

Options fix the sweep kernel's tuning (states per lane, chunk size) so the
captured launch is the configuration under study.
"""
import argparse
import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import numpy as np  # noqa: E402

import workloads  # noqa: E402
import z80b  # noqa: E402

OPT_LANE_STATES, OPT_CHUNK_BLOCKS = 1, 2


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--targets", type=int, default=30000)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--lane-states", type=int, default=4)
    ap.add_argument("--chunk-blocks", type=int, default=32)
    ap.add_argument("--dead-flags", default="none")
    a = ap.parse_args()
    arr = np.ascontiguousarray(workloads.c2_subset(a.targets, seed=a.seed))
    ctx = z80b.Context(0)
    ctx.set_option(OPT_LANE_STATES, a.lane_states)
    ctx.set_option(OPT_CHUNK_BLOCKS, a.chunk_blocks)
    job, keep = ctx.make_job(workloads.to_lists(arr), dead_flags=z80b.parse_dead_flags(a.dead_flags))
    for i in range(a.steps):
        t0 = time.perf_counter()
        rules, st = ctx.run_job(job)
        print(f"step {i}: {len(rules)} rules, {st.checks} checks, {st.exhaustive_pairs} exhaustive pairs, "
              f"{st.exhaustive_states:.4e} states, {st.launches} launches, device {st.device_ms:.2f} ms "
              f"(qc {st.qc_ms:.2f}, exhaustive {st.exh_ms:.2f}), wall {1e3 * (time.perf_counter() - t0):.1f} ms",
              flush=True)
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
