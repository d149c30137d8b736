"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Every comparison is bit-exact: states, fingerprints, verifier verdicts,
FlagDiff masks, rule lists and the reference's 'checked' counter.
"""
import hashlib
import json
import os
import random

import numpy as np
import pytest

import workloads
import z80b

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def digest(arr):
    return hashlib.sha256(np.ascontiguousarray(arr, dtype="<u4").tobytes()).hexdigest()


def fixture_keys(rules):
    return [(r[0], tuple(r[1]), tuple(r[2]), r[3], r[4], r[5]) for r in rules]


_C2FX = None


def c2_fixture_slice(lo, hi, dead):
    """Targets lo..hi of the C2 parity subset and the oracle's rules for them
    under dead flags 0x00 or 0xFF (from c2_100k_oracle.json, re-indexed)."""
    global _C2FX
    if _C2FX is None:
        _C2FX = golden("c2_100k_oracle.json")
    p = next(x for x in _C2FX["passes"] if x["dead_flags"] == dead)
    targets = workloads.to_lists(workloads.c2_subset(100000, seed=0)[lo:hi])
    want = [(r[0] - lo, tuple(r[1]), tuple(r[2]), r[3], r[4], r[5]) for r in p["rules"] if lo <= r[0] < hi]
    return targets, want


def rule_keys(rules):
    return [(r.target_index, tuple(r.src[:r.src_len]), tuple(r.rep[:r.rep_len]),
             r.bytes_saved, r.cycles_saved, r.dead_flags) for r in rules]


def test_exec_all_opcodes(ctx, O):
    rng = random.Random(11)
    states, seqs, exp = [], [], []
    for op in range(455):
        for _ in range(64):
            vals = {k: rng.randrange(256) for k in "AFBCDEHL"}
            vals["SP"] = rng.randrange(65536)
            vals["M"] = rng.randrange(256)
            imm = rng.randrange(65536)
            st = O.state(**vals)
            seq = [O.pack(op, imm)]
            exp.append(O.exec_seq(st, seq).tup())
            s = z80b.State(vals["A"], vals["F"], vals["B"], vals["C"], vals["D"], vals["E"],
                           vals["H"], vals["L"], vals["SP"], vals["M"], 0)
            states.append(s)
            seqs.append(seq)
    got = ctx.exec(states, seqs)
    for i, (g, e) in enumerate(zip(got, exp)):
        assert g.tup() == e, (i // 64, O.op_name(i // 64))


def test_fingerprints(ctx, O):
    pool = z80b.pool8()
    fps = ctx.fingerprints([[w] for w in pool], 1)
    for w, fp in zip(pool, fps):
        assert fp == O.fingerprint([w]), O.disasm([w])
    rng = random.Random(5)
    seqs = [[rng.choice(pool), rng.choice(pool)] for _ in range(3000)]
    fps = ctx.fingerprints(seqs, 2)
    for s, fp in zip(seqs, fps):
        assert fp == O.fingerprint(s)


def test_quickcheck_gpu_reference_cases(ctx, O):
    # pkg/gpu/cuda_test.go:18-157
    o = O.ops()
    cands = [O.pack(o[n], v) for n, v in [("XOR_A", 0), ("LD_A_N", 0), ("AND_A", 0), ("OR_A", 0),
                                            ("ADD_A_B", 0), ("SUB_B", 0), ("NOP", 0), ("LD_A_N", 0x42)]]
    ctx.load_candidates(cands, 1)
    for i, c in enumerate(cands):
        hits = ctx.quickcheck_gpu(O.fingerprint([c]), 0)
        assert i in hits
    # every loaded candidate against the oracle's fingerprint matching
    for dead in (0, 0x28, 0xFF):
        for c in cands:
            fp = O.fingerprint([c])
            exp = []
            for j, d in enumerate(cands):
                a, b = bytearray(O.fingerprint([d])), bytearray(fp)
                for k in range(1, 80, 10):
                    a[k] &= ~dead & 0xFF
                    b[k] &= ~dead & 0xFF
                if a == b:
                    exp.append(j)
            assert ctx.quickcheck_gpu(fp, dead) == exp


def test_quickcheck_gpu_full_first_op(ctx, O):
    # the 266,675 candidates SearchGPU uploads (enumerator.go:358-374)
    pool = z80b.pool8()
    first = pool + [z80b.pack(op, v) for op in (382, 383, 384, 385) for v in range(65536)]
    ctx.load_candidates(first, 1)
    rng = random.Random(9)
    fps_all = None
    for trial in range(6):
        t = [rng.choice(pool), rng.choice(pool)]
        fp = O.fingerprint(t)
        hits = ctx.quickcheck_gpu(fp, 0)
        for h in hits:
            assert O.fingerprint([first[h]]) == fp
    # a target equal to a 16-bit load: its own instruction must be among the hits
    t = [z80b.pack(384, 0x1234)]
    hits = ctx.quickcheck_gpu(O.fingerprint(t), 0)
    assert first.index(t[0]) in hits


def test_verify_pairs(ctx, O):
    rng = random.Random(21)
    pool = z80b.pool8()
    o = O.ops()
    pairs = []
    # equivalences and near misses (reference tests + peephole data)
    pairs.append(([O.pack(o["AND_N"], 0xFF)], [O.pack(o["AND_A"])]))
    pairs.append(([O.pack(o["LD_A_N"], 0)], [O.pack(o["XOR_A"])]))
    pairs.append(([O.pack(o["ADD_A_N"], 1)], [O.pack(o["INC_A"])]))
    pairs.append(([O.pack(o["SUB_A"]), O.pack(o["LD_A_N"], 0)], [O.pack(o["SUB_A"])]))
    # pairs that pass QuickCheck (so the sweeps run past the first states);
    # oracle sweeps are bounded to 2^25 states to keep the checker fast
    targets = workloads.to_lists(workloads.c2_subset(3000, seed=4))
    big = 0
    for t in targets:
        for ci in O.qc_survivors(t)[:2]:
            c = [pool[ci]]
            n = O.exhaustive_states(t, c)
            if n > (1 << 25) or (n > (1 << 17) and big >= 4):
                continue
            big += n > (1 << 17)
            pairs.append((t, c))
        if len(pairs) > 40:
            break
    for _ in range(400):
        pairs.append(([rng.choice(pool), rng.choice(pool)], [rng.choice(pool)]))
    for dead in (0, 0x28, 0xFF):
        deads = [dead] * len(pairs)
        got = ctx.verify_pairs(pairs, dead=deads)
        for (t, c), (bits, fd) in zip(pairs, got):
            exp = (int(O.quickcheck(t, c, dead)) | (int(O.midcheck(t, c, dead)) << 1) |
                   (int(O.exhaustive(t, c, dead)) << 2))
            assert bits == exp, (O.disasm(t), O.disasm(c), dead, bits, exp)
            assert fd == O.flagdiff(t, c)


def _search_both(ctx, O, targets, dead=0, path=z80b.PATH_BATCHED, per_target_dead=None):
    rules, st = ctx.search(targets, dead_flags=dead, path=path, per_target_dead=per_target_dead)
    if per_target_dead is None:
        exp, checked = O.search(targets, 1, dead=dead)
        return rules, st, exp, checked
    exp, checked = [], 0
    groups = {}
    for i, d in enumerate(per_target_dead):
        groups.setdefault(d, []).append(i)
    for d, idx in groups.items():
        r, ch = O.search([targets[i] for i in idx], 1, dead=d)
        for x in r:
            x.target_index = idx[x.target_index]
        exp += r
        checked += ch
    exp.sort(key=lambda r: (r.target_index, r.dead_flags != 0))
    return rules, st, exp, checked


@pytest.mark.parametrize("pas", [0, 1], ids=["dead00", "deadFF"])
def test_search_first_c2_100k(ctx, pas):
    """The C2 parity subset at its configured size: 100,000 targets (seed 0),
    against the oracle's rules and 'checked' counter for dead flags 0x00 and
    0xFF (tests/golden/c2_100k_oracle.json, make_parity_fixtures.py)."""
    fx = golden("c2_100k_oracle.json")
    arr = workloads.c2_subset(100000, seed=0)
    assert digest(arr) == fx["targets_sha256"]
    p = fx["passes"][pas]
    rules, st = ctx.search(workloads.to_lists(arr), dead_flags=p["dead_flags"])
    assert rule_keys(rules) == fixture_keys(p["rules"])
    assert st.checked_ref == p["checked"]
    assert st.targets == 100000


def test_search_first_c1_all(ctx):
    """Every C1 target (53,951) against the oracle's rules and counter
    (tests/golden/c1_full_oracle.json)."""
    fx = golden("c1_full_oracle.json")
    arr = workloads.c1_targets()
    assert digest(arr) == fx["targets_sha256"] and len(arr) == fx["n_targets"]
    p = fx["passes"][0]
    rules, st = ctx.search(workloads.to_lists(arr), dead_flags=p["dead_flags"])
    assert rule_keys(rules) == fixture_keys(p["rules"])
    assert st.checked_ref == p["checked"]


def test_search_first_c2_subset_dead28(ctx, O):
    """A third dead-flag mask (the undocumented bits 3 and 5) on 6,000 C2
    targets, the oracle run live."""
    targets = workloads.to_lists(workloads.c2_subset(6000, seed=0))
    rules, st, exp, checked = _search_both(ctx, O, targets, 0x28)
    assert rule_keys(rules) == rule_keys(exp)
    assert st.checked_ref == checked


def test_search_per_target_dead(ctx, O):
    targets = workloads.to_lists(workloads.c2_subset(3000, seed=8))
    g = workloads.splitmix64(1)
    dead = [next(g) & 0xFF for _ in targets]
    rules, st, exp, checked = _search_both(ctx, O, targets, per_target_dead=dead)
    assert rule_keys(rules) == rule_keys(exp)
    assert st.checked_ref == checked


def test_plain_path_equals_batched(ctx, O):
    targets = workloads.to_lists(workloads.c2_subset(300, seed=3))
    a, sa = ctx.search(targets, dead_flags=0xFF, path=z80b.PATH_BATCHED)
    b, sb = ctx.search(targets, dead_flags=0xFF, path=z80b.PATH_PLAIN)
    assert rule_keys(a) == rule_keys(b)
    assert sa.checked_ref == sb.checked_ref and sa.checks == sb.checks
    exp, _ = O.search(targets, 1, dead=0xFF)
    assert rule_keys(a) == rule_keys(exp)


def test_search_all_hits(ctx, O):
    # gpu.SearchGPU semantics: every candidate of EnumerateFirstOp that passes
    pool = z80b.pool8()
    first = pool + [z80b.pack(op, v) for op in (382, 383, 384, 385) for v in range(65536)]
    ctx.load_candidates(first, 1)
    targets = workloads.to_lists(workloads.c2_subset(150, seed=5))
    o = O.ops()
    targets += [[O.pack(o["SUB_A"]), O.pack(o["LD_A_N"], 0)], [O.pack(o["LD_A_N"], 0), O.pack(o["NEG"])],
                [O.pack(o["LD_H_N"], 0x12), O.pack(o["LD_L_N"], 0x34)]]
    for dead in (0, 0xFF):
        rules, st = ctx.search(targets, dead_flags=dead, mode=z80b.MODE_ALL)
        exp = O.search_gpu_semantics(targets, first, dead)
        assert rule_keys(rules) == rule_keys(exp), dead
    assert any(r.rep[0] & 0xFFFF >= 382 for r in rules)  # a 16-bit load replacement was found


def test_target_lengths_and_edges(ctx, O):
    pool = z80b.pool8()
    rng = random.Random(13)
    targets = [[rng.choice(pool)] for _ in range(300)]
    targets += [[rng.choice(pool) for _ in range(3)] for _ in range(150)]
    targets += [[rng.choice(pool) for _ in range(4)] for _ in range(60)]
    o = O.ops()
    targets += [[O.pack(o["AND_N"], 0xFF)], [O.pack(o["OR_N"], 0)], [O.pack(o["LD_A_N"], 0)]]
    rules, st = ctx.search(targets, dead_flags=0xFF)
    exp, checked = O.search(targets, 1, dead=0xFF)
    assert rule_keys(rules) == rule_keys(exp)
    assert st.checked_ref == checked
    # empty job
    rules, st = ctx.search([])
    assert rules == [] and st.targets == 0


def test_invalid_inputs(ctx):
    with pytest.raises(z80b.Z80BError) as e:
        ctx.search([[455]])
    assert e.value.status == z80b.EINVAL
    with pytest.raises(z80b.Z80BError) as e:
        ctx.search([[1, 2, 3, 4, 5]])
    assert e.value.status == z80b.EINVAL
    with pytest.raises(z80b.Z80BError):
        ctx.search([[1]], max_cand_len=0)


def test_staged_equals_search(ctx):
    targets = workloads.to_lists(workloads.c2_subset(2000, seed=6))
    job, keep = ctx.make_job(targets, dead_flags=0xFF)
    ctx.stage(job)
    n, st = ctx.run_staged()
    staged = ctx.fetch_rules(n)
    rules, _ = ctx.search(targets, dead_flags=0xFF)
    assert rule_keys(staged) == rule_keys(rules)


@pytest.mark.parametrize("all_hits", [False, True])
def test_qc_index_equals_full_scan(ctx, O, all_hits):
    """QuickCheck through the pool's bucket index, in one pass (the count
    pass keeps the survivors of targets with few) and in two, gives the
    rules, survivor counts and QuickCheck unit counts of the scan over every
    candidate, under per-target dead flags and dead registers (and, in
    all-hits mode, the 80-byte fingerprint compare over a loaded pool)."""
    targets = workloads.to_lists(workloads.c2_subset(4000, seed=21))
    g = workloads.splitmix64(5)
    dead = [next(g) & 0xFF for _ in targets]
    dregs = [next(g) & 0x3F if i % 3 else 0 for i in range(len(targets))]
    kw = dict(per_target_dead=dead, dead_regs=dregs)
    if all_hits:
        ctx.load_candidates(z80b.pool8(), 1)
        kw = dict(dead_flags=0xFF, mode=z80b.MODE_ALL)
    out = []
    try:
        for on, single in ((0, 1), (1, 0), (1, 1)):
            ctx.set_option(z80b.OPT_QC_INDEX, on)
            ctx.set_option(z80b.OPT_QC_SINGLE_PASS, single)
            rules, st = ctx.search(targets, **kw)
            out.append((rule_keys(rules), st.checks, st.checked_ref, st.qc_survivors, st.exhaustive_pairs))
    finally:
        ctx.set_option(z80b.OPT_QC_INDEX, 1)
        ctx.set_option(z80b.OPT_QC_SINGLE_PASS, 1)
    assert out[0] == out[1] == out[2]
    assert len(out[1][0]) > 100
    if not all_hits:
        exp, checked = O.search_ext(targets, 1, dead=dead, dregs=dregs)
        assert out[1][0] == rule_keys(exp)
        assert out[1][2] == checked


def test_qc_index_follows_reloaded_pool(ctx):
    """Loading another candidate pool replaces the QuickCheck index built for
    the previous one: the bucket index and the full scan agree on each pool."""
    targets = workloads.to_lists(workloads.c2_subset(1500, seed=23))
    pool = z80b.pool8()
    out = []
    try:
        for cands in (pool[:2000], pool[1000:]):
            ctx.load_candidates(cands, 1)
            got = []
            for on in (1, 0):
                ctx.set_option(z80b.OPT_QC_INDEX, on)
                rules, st = ctx.search(targets, dead_flags=0xFF, mode=z80b.MODE_ALL)
                got.append((rule_keys(rules), st.checks, st.qc_survivors))
            assert got[0] == got[1]
            out.append(got[0])
    finally:
        ctx.set_option(z80b.OPT_QC_INDEX, 1)
    assert out[0] != out[1]


@pytest.mark.parametrize("lane_states,chunk", [(1, 8), (2, 32), (4, 128), (8, 512), (4, 1)])
def test_tuning_options_keep_parity(ctx, lane_states, chunk):
    """Every setting of states per lane (scalar A-independent kernel) and
    units per chunk gives the oracle's rules on 10,000 targets of the C2
    parity subset (dead flags 0xFF)."""
    lo = 10000 * (lane_states % 5)
    targets, want = c2_fixture_slice(lo, lo + 10000, 0xFF)
    opts = [z80b.OPT_EXH_LANE_STATES, z80b.OPT_EXH_CHUNK_BLOCKS, z80b.OPT_XINDEP_BITS]
    old = [ctx.get_option(o) for o in opts]
    ctx.set_option(z80b.OPT_EXH_LANE_STATES, lane_states)
    ctx.set_option(z80b.OPT_EXH_CHUNK_BLOCKS, chunk)
    ctx.set_option(z80b.OPT_XINDEP_BITS, 0 if lane_states != 4 else 1)
    try:
        rules, st = ctx.search(targets, dead_flags=0xFF)
    finally:
        for o, v in zip(opts, old):
            ctx.set_option(o, v)
    assert rule_keys(rules) == want


def test_autotune_picks_a_valid_setting(ctx):
    targets, want = c2_fixture_slice(50000, 52000, 0xFF)
    job, keep = ctx.make_job(targets)
    opts = [z80b.OPT_EXH_LANE_STATES, z80b.OPT_EXH_CHUNK_BLOCKS, z80b.OPT_XINDEP_BITS, z80b.OPT_COMPACT_SWEEP,
            z80b.OPT_WIDE_SWEEP]
    saved = [ctx.get_option(o) for o in opts]
    try:
        r = ctx.autotune(job)
        assert r.lane_states in (1, 2, 4, 8) and r.chunk_blocks in (8, 32, 128, 512)
        assert [ctx.get_option(o) for o in opts] == [r.lane_states, r.chunk_blocks, r.xindep_bits, r.compact,
                                                      r.compact]
        trials = r.trial_list()
        assert len(trials) == 40 and all(t["ms"] > 0 for t in trials)
        # every cell is a distinct kernel configuration, and names what it ran
        cells = {(t["xindep_bits"], t["lane_states"], t["chunk_blocks"], t["compact"]) for t in trials}
        assert len(cells) == 40
        scalar = ("k_exhaustive<1,1>", "k_exhaustive<2,1>", "k_exhaustive<4,1>", "k_exhaustive<8,1>")
        for t in trials:
            if t["xindep_bits"]:
                assert not any(k in t["kernels"] for k in scalar), t
            else:
                assert "k_exhaustive<1,2>" not in t["kernels"], t
                assert all(k not in t["kernels"] for k in scalar if k != f"k_exhaustive<{t['lane_states']},1>"), t
            if t["compact"] == 0:
                assert "k_exhaustive<1,3>" not in t["kernels"] and "k_exhaustive<1,4>" not in t["kernels"], t
        assert any("k_exhaustive<1,3>" in t["kernels"] for t in trials if t["compact"])
        # the chosen setting keeps parity
        rules, st = ctx.search(targets, dead_flags=0xFF)
        assert rule_keys(rules) == want
    finally:
        for o, v in zip(opts, saved):
            ctx.set_option(o, v)
