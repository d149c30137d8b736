"""Small, fixed cases for profiler captures, through the library's public API.

  --case c2      first-found search (pkg/search/worker.go:124-265) on a seeded
                 sample of the length-2 targets (the sweep kernel k_exhaustive)
  --case c3      the batched uneven workload: seeded C3 targets with dead
                 masks, candidates up to 2 instructions (k_pair_scan)
  --case mulopt  constant multiply, all K over one pool up to --max-len
                 (k_mul_length; one launch per length)

Each runs `--steps` times and prints one line of statistics per step; sizes
keep a full-metric-set capture of one launch short, e.g.

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
    ap.add_argument("--targets", type=int, default=30000, help="C2 targets (0 = all 9,818,041)")
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--lane-states", type=int, default=4)
    ap.add_argument("--chunk-blocks", type=int, default=32)
    ap.add_argument("--dead-flags", default="none")
    ap.add_argument("--qc-index", type=int, default=1, choices=[0, 1],
                    help="QuickCheck through the pool's bucket index (1) or over every candidate (0)")
    ap.add_argument("--xindep-bits", type=int, default=1, choices=[0, 1],
                    help="A-independent sweeps bit-sliced (1) or one state per lane slot (0)")
    ap.add_argument("--compact", type=int, default=1, choices=[0, 1],
                    help="A-dependent pairs naming at most two of B..L on the compact-state sweep kernel")
    ap.add_argument("--wide", type=int, default=1, choices=[0, 1],
                    help="other A-dependent pairs naming at most four of B..L on the wide compact-state kernel")
    ap.add_argument("--graph-rounds", type=int, default=1, choices=[0, 1],
                    help="first-found rounds driven on the device by one CUDA graph (1) or from the host (0; "
                         "ncu profiles no kernel inside a graph with conditional nodes)")
    ap.add_argument("--concurrent", type=int, default=1, choices=[0, 1],
                    help="device-driven rounds: sweep classes on parallel graph branches (1) or in sequence (0)")
    ap.add_argument("--case", default="c2", choices=["c2", "c3", "mulopt"])
    ap.add_argument("--pool", type=int, default=2, help="mulopt pool (Z80B_MULPOOL_*)")
    ap.add_argument("--max-len", type=int, default=9, help="mulopt: longest sequence")
    a = ap.parse_args()
    if a.case == "mulopt":
        ctx = z80b.Context(0)
        init = workloads.mul_init(2) if a.pool == 1 else (0, 0, 0)
        for i in range(a.steps):
            res, st = ctx.mul_search(a.pool, init, 1, a.max_len)
            print(f"step {i}: {sum(r['found'] for r in res)} constants found, {st.sequences:.4e} sequences, "
                  f"{st.launches} launches, device {st.device_ms:.2f} ms", flush=True)
        ctx.close()
        return 0
    if a.case == "c3":
        ctx = z80b.Context(0)
        ctx.set_option(OPT_LANE_STATES, a.lane_states)
        ctx.set_option(OPT_CHUNK_BLOCKS, a.chunk_blocks)
        ctx.set_option(z80b.OPT_QC_INDEX, a.qc_index)
        ctx.set_option(z80b.OPT_XINDEP_BITS, a.xindep_bits)
        ctx.set_option(z80b.OPT_COMPACT_SWEEP, a.compact)
        ctx.set_option(z80b.OPT_WIDE_SWEEP, a.wide)
        ctx.set_option(z80b.OPT_GRAPH_ROUNDS, a.graph_rounds)
        ctx.set_option(z80b.OPT_CONCURRENT_SWEEPS, a.concurrent)
        arr, lens, dead, dregs = workloads.c3_targets(a.targets, seed=1)
        targets = [list(map(int, arr[i, :lens[i]])) for i in range(a.targets)]
        job, keep = ctx.make_job(targets, per_target_dead=list(map(int, dead)), dead_regs=list(map(int, dregs)),
                                 max_cand_len=2)
        for i in range(a.steps):
            rules, st = ctx.run_job(job)
            print(f"step {i}: {len(rules)} rules, {st.checks} checks, {st.exhaustive_pairs} exhaustive pairs, "
                  f"{st.exhaustive_states:.4e} states ({st.exhaustive_evaluated:.4e} evaluated), "
                  f"{st.rounds} rounds, {st.launches} launches, device {st.device_ms:.2f} ms "
                  f"(qc {st.qc_ms:.2f}, exhaustive {st.exh_ms:.2f})", flush=True)
        ctx.close()
        return 0
    arr = np.ascontiguousarray(workloads.c2_subset(a.targets, seed=a.seed) if a.targets
                               else workloads.c2_targets())
    ctx = z80b.Context(0)
    ctx.set_option(OPT_LANE_STATES, a.lane_states)
    ctx.set_option(OPT_CHUNK_BLOCKS, a.chunk_blocks)
    ctx.set_option(z80b.OPT_QC_INDEX, a.qc_index)
    ctx.set_option(z80b.OPT_XINDEP_BITS, a.xindep_bits)
    ctx.set_option(z80b.OPT_COMPACT_SWEEP, a.compact)
    ctx.set_option(z80b.OPT_WIDE_SWEEP, a.wide)
    ctx.set_option(z80b.OPT_GRAPH_ROUNDS, a.graph_rounds)
    ctx.set_option(z80b.OPT_CONCURRENT_SWEEPS, a.concurrent)
    job, keep = ctx.make_job(workloads.to_lists(arr), dead_flags=z80b.parse_dead_flags(a.dead_flags))
    for i in range(a.steps):
        t0 = time.perf_counter()
        rules, st = ctx.run_job(job)
        print(f"step {i}: {len(rules)} rules, {st.checks} checks, {st.exhaustive_pairs} exhaustive pairs, "
              f"{st.exhaustive_states:.4e} states ({st.exhaustive_evaluated:.4e} evaluated), {st.rounds} rounds, "
              f"{st.launches} launches, device {st.device_ms:.2f} ms "
              f"(qc {st.qc_ms:.2f}, exhaustive {st.exh_ms:.2f}), wall {1e3 * (time.perf_counter() - t0):.1f} ms",
              flush=True)
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
