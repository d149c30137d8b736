"""Benchmark of the candidate-verification path on B200.

Workload (default): every unpruned length-2 target over the reference's
8-bit instruction list (9,818,041 targets, the C2 configuration),
candidates of length 1, the first-found semantics of pkg/search
(QuickCheck -> ExhaustiveCheck per target, shortest/first candidate wins).
One step = one pass of the whole pipeline over the targets.  `--targets N`
runs a seeded sample of N of them instead.

Metric: candidate checks/s = (target, candidate) pairs of the workload that
pass the byte-size and prune filters (the QuickCheck unit of work), per
second of the step.  `value` runs on targets already resident in HBM
(z80b_stage_job / z80b_run_staged, device time from CUDA events on the
library's stream); `e2e` calls z80b_search with pinned host buffers, so
every step includes the H2D copy of the targets and the D2H copy of the
rules.  Between steps L2 is flushed by writing a 512 MiB buffer.

CPU figures (the `cpu_baseline` leg and `--impl reference`) come from the
oracle, the C++ restatement of the reference's Go search (no Go toolchain
exists on the box), run on one fixed CPU sample of the workload: the
100,000 targets drawn by index with default_rng(0) (the C2 parity subset)
on all host threads.  Their time is the worker threads' CPU time divided by
the thread count (a balanced pool's wall time; one slow target does not
serialise a small sample), and a target whose sweeps need more than
CPU_TARGET_BUDGET_S of CPU is left out of checks and time alike (the sweep
tail; its count is reported).  `--impl reference` loads only the oracle:
the target set, the sample and the check count all come from it.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "z80-optimizer_b200")
sys.path.insert(0, PKG)

import numpy as np  # noqa: E402

METRIC = "Z80 candidate checks/s on 1 B200, batched vs plain GPU; p50/p99 query latency"
UNIT = "candidate checks/s"


T0 = time.perf_counter()


def progress(*a):
    print(f"[bench {time.perf_counter() - T0:8.2f}s]", *a, file=sys.stderr, flush=True)


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--targets", type=int, default=0,
                    help="seeded uniform sample of the C2 targets (0 = all 9,818,041)")
    ap.add_argument("--plain-sample", type=int, default=2000,
                    help="targets of the plain-vs-batched comparison (0 = skip)")
    ap.add_argument("--dead-flags", default="none")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample", type=int, default=100000,
                    help="targets in the CPU sample (drawn by index with default_rng(0))")
    ap.add_argument("--no-mulopt", action="store_true", help="skip the constant-multiply leg")
    ap.add_argument("--c3-targets", type=int, default=4000000,
                    help="C3 targets (the configuration's 4,000,000; 0 = skip the C3 leg)")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="served-query leg length (0 = skip)")
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="Poisson arrival rate of the served leg")
    ap.add_argument("--mulopt-max-len", type=int, default=9)
    return ap.parse_args(argv)


class ClockSampler:
    """nvidia-smi samples every 200 ms while running (median SM clock, reasons)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.stop = threading.Event()
        self.t = None

    def _run(self):
        while not self.stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"],
                                     capture_output=True, text=True, timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self.stop.wait(0.2)

    def __enter__(self):
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        self.t.join()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def make_job(z80b, arr, dead):
    n, L = arr.shape
    job = z80b.Job()
    job.targets = ctypes.cast(arr.ctypes.data, ctypes.POINTER(ctypes.c_uint32))
    job.n_targets = n
    job.target_len = L
    job.target_stride = L
    job.max_cand_len = 1
    job.global_dead_flags = dead
    job.mode = z80b.MODE_FIRST
    job.path = z80b.PATH_BATCHED
    return job


def cpu_sample(allt, n, seed=0):
    """The CPU sample: n targets of the workload drawn by index with
    default_rng(seed), in index order (for all C2 targets and n = 100,000,
    the C2 parity subset)."""
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(len(allt), size=min(n, len(allt)), replace=False))
    return allt[idx]


# CPU seconds one target may spend in its ExhaustiveCheck sweeps in the timed
# CPU sample: the sweep tail (true equivalences swept over up to 2^34
# states, about 10 minutes each on one core) would otherwise hold a pass for
# many minutes.  Targets that run past it are left out of the checks and the
# time alike, so the CPU rate shown is the rate without that tail (an upper
# bound on the CPU's rate over the whole workload).
CPU_TARGET_BUDGET_S = 2.0


def cpu_pass(sample, dead, workers):
    """The oracle (CPU restatement of pkg/search worker.go:124-265, one task
    per target on `workers` threads) over `sample`.  Returns (balanced
    seconds, wall seconds, per-target seconds (-1: abandoned), candidate
    checks of the finished targets, rules): balanced seconds = the threads'
    CPU time on the finished targets / workers, the wall time of a busy pool,
    which the whole workload approaches; a small sample's wall time is
    bounded below by its slowest target instead."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    t0 = time.perf_counter()
    rules, _, secs = oracle_lib.search_timed([list(map(int, r)) for r in sample], 1, dead=dead, workers=workers,
                                             target_budget=CPU_TARGET_BUDGET_S)
    wall = time.perf_counter() - t0
    done = np.array([x >= 0 for x in secs], dtype=bool)
    checks = oracle_lib.eligible_checks(sample[done]) if done.any() else 0
    return sum(x for x in secs if x >= 0) / workers, wall, secs, checks, len(rules)


def tail_note(secs):
    """The sweep-size tail of a sample: the targets abandoned at the budget,
    and how much of the finished targets' CPU time the slowest ones take."""
    fin = sorted((x for x in secs if x >= 0), reverse=True)
    tot = sum(fin) or 1.0
    return (f"{sum(1 for x in secs if x < 0)} targets abandoned after {CPU_TARGET_BUDGET_S:.0f} CPU s of sweeps "
            f"and left out (sweep tail); of the finished ones the slowest took {fin[0] if fin else 0:.2f} s, the "
            f"10 slowest {100 * sum(fin[:10]) / tot:.1f}% of the CPU time")


def cpu_baseline(allt, dead, n_sample):
    workers = os.cpu_count() or 1
    sample = cpu_sample(allt, n_sample)
    bal, wall, secs, checks, _ = cpu_pass(sample, dead, workers)
    return {"value": checks / bal, "unit": UNIT, "cores": workers, "kind": "port",
            "sample": f"{len(sample)} targets drawn by index (default_rng(0)) from the workload, one pass on "
                      f"{workers} threads: {checks} candidate checks, {bal:.2f} s balanced ({wall:.2f} s wall); "
                      + tail_note(secs)}


def mulopt_leg(ctx, z80b, workloads, args, with_cpu):
    """Constant-multiply workload: every K = 2..255 over the 21-op pool with
    B, C, F from seed 2, lengths 1..max_len, one z80b_mul_search per step
    (device time of its kernels); the CPU oracle's findOptimal on a bounded
    set of constants beside it."""
    import torch
    init = workloads.mul_init(2)
    ml = args.mulopt_max_len
    for _ in range(args.warmup):
        ctx.mul_search(z80b.MULPOOL_WIDE21, init, 1, ml)
    ms, res, st = [], None, None
    for _ in range(args.steps):
        torch.cuda.synchronize()
        res, st = ctx.mul_search(z80b.MULPOOL_WIDE21, init, 1, ml)
        ms.append(st.device_ms)
    t = statistics.median(ms)
    hist = {}
    for r in res:
        if r["found"]:
            hist[r["length"]] = hist.get(r["length"], 0) + 1
    out = {"workload": f"K=2..255, 21-op pool, B,C,F=({init[0]:#04x},{init[1]:#04x},{init[2]:#04x}) from seed 2, "
                       f"lengths 1..{ml}",
           "device_ms_per_step": t, "launches_per_step": st.launches,
           "sequences_per_step": st.sequences, "sequences_per_s": st.sequences / (t / 1e3),
           "per_k_sequences_per_step": st.per_k_sequences,
           "per_k_sequences_per_s": st.per_k_sequences / (t / 1e3),
           "unit_note": "a sequence is one odometer entry walked once for all K; per-K sequences are what one "
                        "odometer per constant (cmd/mulopt findOptimal) tests",
           "found": sum(hist.values()), "not_found": 254 - sum(hist.values()),
           "lengths": {str(k): hist[k] for k in sorted(hist)},
           "full_checks": st.full_checks, "full_pass": st.full_pass}
    if with_cpu:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_lib
        from concurrent.futures import ThreadPoolExecutor
        ks = list(range(2, 19))   # constants whose optimum has <= 6 instructions
        seqs = 0
        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
            cres = list(ex.map(lambda k: oracle_lib.mul_find_pool(1, k, 1, 6, *init), ks))
        secs = time.perf_counter() - t0
        for r in cres:
            seqs += sum(21 ** L for L in range(1, (r[0] if r else 6) + 1))
        gpu_by_k = {r["k"]: r for r in res}
        agree = all(c is not None and (c[0], c[1], c[2]) == (gpu_by_k[k]["length"], gpu_by_k[k]["tstates"],
                                                            gpu_by_k[k]["ops"]) for k, c in zip(ks, cres))
        out["cpu_baseline"] = {"value": seqs / secs, "unit": "per-K sequences/s", "cores": os.cpu_count() or 1,
                               "kind": "port", "sample": f"findOptimal for K=2..18 (lengths 1..6) in {secs:.2f} s, "
                                                         f"{seqs} per-K sequences, one thread per K",
                               "agrees_with_device": agree}
    return out


def tune_record(tr, sample):
    """The autotuner's choice and its trial grid, each trial with the sweep
    kernels it launched."""
    trials = tr.trial_list()
    best = min(trials, key=lambda t: t["ms"])
    return {"chosen": {"xindep_bits": tr.xindep_bits, "lane_states": tr.lane_states,
                       "chunk_blocks": tr.chunk_blocks, "compact": tr.compact, "kernels": best["kernels"]},
            "grid": "A-independent kernel (bit-sliced; scalar at 1, 2, 4, 8 states per lane) x units per chunk "
                    "(8, 32, 128, 512) x compact kernel (off, on)",
            "sample": sample,
            "trials": [[t["xindep_bits"], t["lane_states"], t["chunk_blocks"], t["compact"], round(t["ms"], 3),
                        t["kernels"]] for t in trials],
            "trial_fields": ["xindep_bits", "lane_states", "chunk_blocks", "compact", "device_ms", "kernels"]}


def c3_leg(ctx, z80b, workloads, args):
    """Batched uneven workload: seeded C3 targets (60% length 2, 40% length
    3, per-target dead-register and dead-flag masks), candidates up to 2
    instructions, first-found semantics.  The sweep configuration is tuned
    on the first 20,000 targets (whose first search also builds the length-2
    pair pool and its bucket indexes), then one timed search covers every target
    (device time of the pipeline).  Beside it, the first 1,000 targets
    through the one-target-per-launch path and the batched path."""
    import torch
    n = args.c3_targets
    arr, lens, dead, dregs = workloads.c3_targets(n, seed=1)
    arr = np.ascontiguousarray(arr)

    def job_for(lo, hi, path):
        j = z80b.Job()
        a = np.ascontiguousarray(arr[lo:hi])
        ln, d, r = (np.ascontiguousarray(x[lo:hi]) for x in (lens, dead, dregs))
        j.targets = a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
        j.target_lens = ln.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
        j.dead_flags = d.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
        j.dead_regs = r.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
        j.n_targets = hi - lo
        j.target_stride = 4
        j.max_cand_len = 2
        j.mode = z80b.MODE_FIRST
        j.path = path
        return j, (a, ln, d, r)

    # tune the sweep kernel for this workload on its first 20,000 targets
    # (longer sequences than C2's, so another setting may win; the first
    # trial also builds the pair pool and its bucket indexes); the C2
    # setting is restored after the leg
    tuned = [z80b.OPT_EXH_LANE_STATES, z80b.OPT_EXH_CHUNK_BLOCKS, z80b.OPT_XINDEP_BITS, z80b.OPT_COMPACT_SWEEP,
             z80b.OPT_WIDE_SWEEP]
    saved = [ctx.get_option(o) for o in tuned]
    tj, tkeep = job_for(0, min(20000, n), z80b.PATH_BATCHED)
    tr = ctx.autotune(tj)
    job, keep = job_for(0, n, z80b.PATH_BATCHED)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    rules, st = ctx.run_job(job)
    wall = time.perf_counter() - t1
    nrules = len(rules)
    t = st.device_ms
    out = {"workload": f"C3: {n} targets from seed 1 (60% length 2 / 40% length 3, dead-register and dead-flag "
                       f"mask per target), candidates up to 2 instructions",
           "value": st.checks / (t / 1e3), "unit": UNIT, "device_ms_per_step": t, "rules": nrules,
           "qc_survivors": st.qc_survivors, "exhaustive_pairs": st.exhaustive_pairs,
           "exhaustive_states": st.exhaustive_states, "rounds": st.rounds, "launches": st.launches,
           "exhaustive_ms": st.exh_ms, "checks": st.checks, "wall_s": wall,
           "steps": 1, "timing": "one search over every target after the tuning searches of the first 20,000",
           "autotune": tune_record(tr, "first 20,000 targets of the leg")}
    if args.plain_sample:
        m = min(1000, n)
        pj, keep2 = job_for(0, m, z80b.PATH_PLAIN)
        bj, keep3 = job_for(0, m, z80b.PATH_BATCHED)
        t1 = time.perf_counter()
        _, stp = ctx.run_job(pj)
        tp = time.perf_counter() - t1
        t1 = time.perf_counter()
        _, stb = ctx.run_job(bj)
        tb = time.perf_counter() - t1
        out["plain_vs_batched"] = {"targets": m, "plain_checks_per_s": stp.checks / tp,
                                   "batched_checks_per_s": stb.checks / tb, "batched_over_plain": tp / tb,
                                   "timing": "host wall clock around z80b_search (both synchronous)"}
    for o, v in zip(tuned, saved):
        ctx.set_option(o, v)
    return out


C2_TARGETS = 9818041  # unpruned length-2 targets over the 8-bit list (checked by the tests)


def workload_config(args, world):
    """The `config` object of both arms' JSON lines."""
    nsel = min(args.targets, C2_TARGETS) if args.targets else C2_TARGETS
    return {"workload": "length-2 targets (C2)" + (f", seeded sample of {nsel} / {C2_TARGETS}"
                                                 if args.targets else ", all"),
            "targets": nsel, "target_len": 2,
            "max_cand_len": 1, "candidates": 4531, "semantics": "pkg/search first-found",
            "dead_flags": args.dead_flags, "vectors": "reference QuickCheck 8 (verifier.go:19-28)",
            "l2": "flushed between steps (512 MiB write)", "path": "batched",
            "parallelism": f"targets sharded over {world} GPU(s)"}


def reference_arm(args, rank, workload):
    """The reference's CPU path (the oracle: the Go toolchain is absent) on
    the workload's CPU sample, loading only the oracle.  Warm-up steps run
    200 other targets; the timed steps split the CPU sample into `steps`
    consecutive parts, so all timed steps together make one pass over it
    (the same sample and the same time measure as the `cpu_baseline` leg of
    the GPU arm).  Under torchrun only rank 0 runs."""
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    dead = oracle_lib.parse_dead_flags(args.dead_flags)
    if dead is None:
        raise SystemExit(f"bad --dead-flags value {args.dead_flags!r}")
    full = oracle_lib.c2_targets()
    assert len(full) == C2_TARGETS
    allt = oracle_lib.c2_subset(args.targets, seed=0) if args.targets else full
    workers = os.cpu_count() or 1
    sample = cpu_sample(allt, args.cpu_sample)
    warm = cpu_sample(allt, 200, seed=99)
    for i in range(args.warmup):
        cpu_pass(warm, dead, workers)
        progress(f"reference warmup {i}")
    bal, wall, checks, secs = 0.0, 0.0, 0, []
    for part in np.array_split(sample, args.steps):
        b, w, s, c, _ = cpu_pass(part, dead, workers)
        bal, wall, checks, secs = bal + b, wall + w, checks + c, secs + s
        progress(f"reference step: {len(part)} targets, {b:.2f} s balanced, {w:.2f} s wall")
    value = checks / bal
    note = (f"{len(sample)} targets drawn by index (default_rng(0)) from the workload, split into {args.steps} "
            f"steps of ~{len(sample) // args.steps} on {workers} threads: {checks} candidate checks, {bal:.2f} s "
            f"balanced ({wall:.2f} s wall); " + tail_note(secs))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * bal / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic", "config": workload,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": "port", "sample": note},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    # The workload description is built before either arm loads anything, so
    # both arms print the same config.
    workload = workload_config(args, world)
    ntot = C2_TARGETS

    if args.impl == "reference":
        return reference_arm(args, rank, workload)

    import z80b
    import workloads
    dead = z80b.parse_dead_flags(args.dead_flags)
    full = workloads.c2_targets()
    assert len(full) == ntot
    allt = workloads.c2_subset(args.targets, seed=0) if args.targets else full

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    # strong scaling: the fixed target set is split into contiguous shards
    lo, hi = workloads.shard_bounds(len(allt), rank, world)
    mine = np.ascontiguousarray(allt[lo:hi])
    ctx = z80b.Context(local if world > 1 else 0)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    progress(f"rank {rank}: {len(mine)} targets staged")

    # ---- autotune (sweep kernel configuration) on a 200k-target sample
    # tuned on the workload itself: small samples favour small chunks (few
    # chunks to balance), which lose at the full size
    tr = ctx.autotune(make_job(z80b, mine, dead))
    tuning = tune_record(tr, f"the workload itself ({len(mine):,} targets)")
    progress(f"autotune: {tuning['chosen']}")

    # ---- value: targets resident in HBM
    job = make_job(z80b, mine, dead)
    ctx.stage(job)
    for i in range(args.warmup):
        flush.fill_(1)
        torch.cuda.synchronize()
        _, wst = ctx.run_staged()
        progress(f"warmup {i}: {wst.device_ms:.1f} ms, {wst.exhaustive_states:.3e} states, {wst.rounds} rounds")
    dev_ms, exh_ms, qc_ms, launches, checks, states, evaluated, rules = 0.0, 0.0, 0.0, 0, 0, 0, 0, 0
    stats_last = None
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            n, st = ctx.run_staged()
            dev_ms += st.device_ms
            exh_ms += st.exh_ms
            qc_ms += st.qc_ms
            launches += st.launches
            checks += st.checks
            states += st.exhaustive_states
            evaluated += st.exhaustive_evaluated
            rules = n
            stats_last = st
            progress(f"step: {st.device_ms:.1f} ms (qc {st.qc_ms:.1f}, exhaustive {st.exh_ms:.1f})")
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    t_step = dev_ms / args.steps
    if dist:
        t = torch.tensor([t_step], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_step = float(t.item())
        c = torch.tensor([checks], device="cuda", dtype=torch.float64)
        dist.all_reduce(c)
        checks_all = float(c.item())
    else:
        checks_all = float(checks)
    value = checks_all / args.steps / (t_step / 1e3)
    # algorithmic emulated instructions of the steps (length-2 targets, length-1 candidates)
    emulated = 8.0 * checks + 16.0 * len(mine) * args.steps + 3.0 * evaluated

    # ---- e2e: public API with pinned host buffers
    pinned = torch.from_numpy(mine).pin_memory()
    pj = make_job(z80b, mine, dead)
    pj.targets = ctypes.cast(pinned.data_ptr(), ctypes.POINTER(ctypes.c_uint32))
    cap = max(1024, 2 * rules + 1024)
    out = (z80b.Rule * cap)()
    nr = ctypes.c_uint64()
    st2 = z80b.Stats()
    L = z80b.lib()
    for _ in range(max(1, args.warmup)):
        flush.fill_(1)
        torch.cuda.synchronize()
        ctx._check(L.z80b_search(ctx._h, ctypes.byref(pj), out, cap, ctypes.byref(nr), ctypes.byref(st2)))
    e2e_t = 0.0
    e2e_checks = 0
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t1 = time.perf_counter()
        ctx._check(L.z80b_search(ctx._h, ctypes.byref(pj), out, cap, ctypes.byref(nr), ctypes.byref(st2)))
        e2e_t += time.perf_counter() - t1
        e2e_checks += st2.checks
    e2e_step = e2e_t / args.steps
    progress(f"e2e: {1e3 * e2e_step:.1f} ms per step")
    if dist:
        t = torch.tensor([e2e_step], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_step = float(t.item())
        c = torch.tensor([e2e_checks], device="cuda", dtype=torch.float64)
        dist.all_reduce(c)
        e2e_checks = float(c.item())
    e2e_value = e2e_checks / args.steps / e2e_step
    h2d = int(mine.nbytes)
    d2h = int(nr.value) * 12 + 64

    # ---- roofline of the dominant kernels (the ExhaustiveCheck sweep classes)
    # Integer issue-bound work (no contraction, nothing per state from
    # DRAM): peak = SMs x 4 warp-instruction issue slots per clock x the max
    # SM clock.  The unit is one evaluated sweep state; its cost in warp
    # instructions is fixed by an ncu capture of every sweep launch of one
    # step of a C2 sample (roofline.json "sweep_capture": the capture's
    # smsp__inst_executed.sum over its evaluated states), and this run's
    # sweep time turns it into an issue rate, so frac reads as the issue-slot
    # utilisation of the whole sweep phase at this run's speed (gaps between
    # rounds and tails of launches included).
    rl = json.load(open(os.path.join(PKG, "roofline.json")))
    cap = rl["sweep_capture"]
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    sm_mhz = peaks.get("sm_max_mhz", 1965.0)
    exh_s = exh_ms / args.steps / 1e3
    evaluated_step = evaluated / args.steps
    issue_peak = rl["sms"] * rl["issue_slots_per_sm_per_clock"] * sm_mhz * 1e6
    issued = evaluated_step * cap["warp_instructions_per_evaluated_state"]
    achieved = issued / exh_s if exh_s else 0.0
    # the scalar cost model (INT32 lane-ops a one-state-per-lane step of the
    # reference would need per evaluated state): an algorithmic work rate,
    # above 1 of the lane peak because the bit-sliced kernels step 32
    # states per lane instruction
    per_state = 3 * rl["ops_per_emulated_insn"] + rl["ops_per_state"]  # 2-insn target + 1-insn candidate
    scalar_rate = evaluated_step * per_state / exh_s if exh_s else 0.0
    scalar_peak = rl["sms"] * rl["int32_lanes_per_sm"] * sm_mhz * 1e6
    rounds = max(1, stats_last.rounds) if stats_last is not None else 1
    pairs_step = stats_last.exhaustive_pairs if stats_last is not None else 0
    roofline = {"bound": "issue", "kernel": "k_exhaustive (the sweep classes of a round)",
                "achieved": achieved / 1e12, "peak": issue_peak / 1e12,
                "unit": "T warp-instructions/s (issue slots)",
                "frac": achieved / issue_peak if issue_peak else None,
                # DRAM bytes of one round's sweep launches: the capture's
                # bytes per swept pair (pair records, programs, chunk
                # prefixes; nothing per state) x this run's pairs per round
                "traffic": cap["dram_bytes_per_pair"] * pairs_step / rounds,
                "traffic_unit": "DRAM bytes per sweep round (its sweep launches)",
                "peak_source": f"{rl['sms']} SMs x {rl['issue_slots_per_sm_per_clock']} issue slots x "
                               f"{sm_mhz:.0f} MHz ({'MEASURED_PEAKS.json' if 'sm_max_mhz' in peaks else 'nominal max SM clock'})",
                "work_unit": f"evaluated sweep state, {cap['warp_instructions_per_evaluated_state']:.4g} warp "
                             f"instructions each ({cap['source']})",
                "ncu_issue_active_pct": cap["issue_active_pct"],
                "scalar_equivalent": {"achieved": scalar_rate / 1e12, "peak": scalar_peak / 1e12,
                                      "unit": "T INT32 lane-ops/s", "frac": scalar_rate / scalar_peak,
                                      "ops_per_state": per_state},
                "exhaustive_ms_per_step": exh_ms / args.steps, "qc_ms_per_step": qc_ms / args.steps,
                "evaluated_states_per_step": evaluated_step}

    # ---- plain (one target per launch) vs batched on the same sample
    plain = None
    if args.plain_sample and rank == 0:
        ps = np.ascontiguousarray(workloads.c2_subset(args.plain_sample, seed=7))
        pjob = make_job(z80b, ps, dead)
        pjob.path = z80b.PATH_PLAIN
        _, stp = ctx.run_job(pjob)
        t1 = time.perf_counter()
        _, stp = ctx.run_job(pjob)
        tp = time.perf_counter() - t1
        bjob = make_job(z80b, ps, dead)
        _, stb = ctx.run_job(bjob)
        t1 = time.perf_counter()
        _, stb = ctx.run_job(bjob)
        tb = time.perf_counter() - t1
        progress(f"plain {tp:.2f} s vs batched {tb:.2f} s on {len(ps)} targets")
        plain = {"targets": int(len(ps)), "plain_checks_per_s": stp.checks / tp,
                 "batched_checks_per_s": stb.checks / tb, "batched_over_plain": tp / tb,
                 "plain_launches": stp.launches, "batched_launches": stb.launches,
                 "timing": "host wall clock around z80b_search (both synchronous)"}

    c3 = None
    if rank == 0 and args.c3_targets:
        c3 = c3_leg(ctx, z80b, workloads, args)
        progress(f"c3: {c3['device_ms_per_step']:.1f} ms per step, {c3['rules']} rules")

    serve = None
    if rank == 0 and args.serve_seconds > 0:
        import serve_load
        serve, _ = serve_load.run(rate=args.serve_rate, seconds=args.serve_seconds, seed=3, verify=True)
        progress(f"serve: p50 {serve['p50_ms']:.2f} ms, p99 {serve['p99_ms']:.2f} ms, {serve['qps']:.0f} q/s")

    mulopt = None
    if rank == 0 and not args.no_mulopt:
        mulopt = mulopt_leg(ctx, z80b, workloads, args, world == 1 and not args.no_cpu_baseline)
        progress(f"mulopt: {mulopt['device_ms_per_step']:.1f} ms per step, {mulopt['found']} constants found")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(allt, dead, args.cpu_sample)
        progress(f"cpu baseline: {cpu['sample']}")

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_step, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": workload,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": 1e3 * e2e_step},
            "roofline": roofline, "cpu_baseline": cpu, "clocks": clk.summary(),
            "gpu_launches": launches, "plain_vs_batched": plain, "autotune": tuning,
            "emulated_instructions": {"value": emulated / args.steps / (t_step / 1e3), "unit": "emulated Z80 instructions/s",
                                      "model": "8 per length-1 check + 8 per target instruction + (target + "
                                               "candidate instructions) per swept state"},
            "c3": c3, "mulopt": mulopt, "serve": serve,
            "detail": {"rules": rules, "checked_ref": stats_last.checked_ref if stats_last else None,
                       "qc_survivors": stats_last.qc_survivors if stats_last else None,
                       "exhaustive_pairs": stats_last.exhaustive_pairs if stats_last else None,
                       "exhaustive_states_per_step": states / args.steps,
                       "exhaustive_evaluated_per_step": evaluated / args.steps,
                       "rounds": stats_last.rounds if stats_last else None,
                       "wall_s_timed": wall}}
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
