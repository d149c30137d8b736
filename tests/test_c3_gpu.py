"""Length-2 candidates with per-target dead flags and dead registers (the
batched uneven workload) on the device against the CPU oracle.

Rules are compared bit for bit (target, source, replacement, byte and cycle
savings, dead flags, dead registers) together with the reference's
'checked' counter."""
import json
import os

import pytest

import z80b
from conftest import ROOT

pytestmark = pytest.mark.gpu


def fixture():
    return json.load(open(os.path.join(ROOT, "tests", "golden", "c3_oracle.json")))


def dev_keys(rules):
    return [(r.target_index, list(r.src[:r.src_len]), list(r.rep[:r.rep_len]), r.bytes_saved, r.cycles_saved,
             r.dead_flags, r.dead_regs) for r in rules]


def run(ctx, fx, idx=None, path=z80b.PATH_BATCHED):
    idx = range(fx["n"]) if idx is None else idx
    targets = [fx["targets"][i] for i in idx]
    return ctx.search(targets, per_target_dead=[fx["dead_flags"][i] for i in idx],
                      dead_regs=[fx["dead_regs"][i] for i in idx], max_cand_len=2, path=path)


def test_c3_sample_rules_and_checked(ctx):
    fx = fixture()
    rules, st = run(ctx, fx)
    got = [tuple([k[0], tuple(k[1]), tuple(k[2])] + list(k[3:])) for k in dev_keys(rules)]
    want = [tuple([r[0], tuple(r[1]), tuple(r[2])] + list(r[3:])) for r in fx["rules"]]
    assert got == want
    assert st.checked_ref == fx["checked"]
    assert any(len(r.rep[:r.rep_len]) == 2 for r in rules)


def test_c3_plain_equals_batched(ctx):
    fx = fixture()
    idx = list(range(0, fx["n"], 8))
    a, _ = run(ctx, fx, idx)
    b, _ = run(ctx, fx, idx, path=z80b.PATH_PLAIN)
    assert dev_keys(a) == dev_keys(b)


def test_length2_needs_first_mode(ctx):
    with pytest.raises(z80b.Z80BError) as e:
        ctx.search([[z80b.pack(0), z80b.pack(1)]], mode=z80b.MODE_ALL, max_cand_len=2)
    assert e.value.status == z80b.EINVAL


def test_streaming_answers_equal_final_rules(ctx):
    """z80b_search_cb hands every target's rules to the callback exactly
    once, and they are the rules z80b_search returns for it."""
    fx = fixture()
    idx = list(range(0, fx["n"], 2))
    targets = [fx["targets"][i] for i in idx]
    rules, st, events = ctx.search_streaming(targets, per_target_dead=[fx["dead_flags"][i] for i in idx],
                                             dead_regs=[fx["dead_regs"][i] for i in idx], max_cand_len=2)
    assert sorted(t for t, _ in events) == list(range(len(targets)))
    by_t = {}
    for r in rules:
        by_t.setdefault(r.target_index, []).append(r.key())
    for t, keys in events:
        assert keys == by_t.get(t, []), t


@pytest.mark.parametrize("xbits", [1, 0])
def test_a_independent_sweep_kernels_keep_parity(ctx, O, xbits):
    """Both A-independent sweep kernels (Z80B_OPT_XINDEP_BITS = 1: bit-sliced,
    32 blocks per lane word, the default; 0: one state per lane slot): the C3
    sample's rules and 'checked' counter, and a C2 sample against the
    oracle."""
    import workloads
    fx = fixture()
    old = ctx.get_option(z80b.OPT_XINDEP_BITS)
    ctx.set_option(z80b.OPT_XINDEP_BITS, xbits)
    try:
        rules, st = run(ctx, fx)
        targets = workloads.to_lists(workloads.c2_subset(3000, seed=12))
        r2, st2 = ctx.search(targets, dead_flags=0xFF)
    finally:
        ctx.set_option(z80b.OPT_XINDEP_BITS, old)
    got = [tuple([k[0], tuple(k[1]), tuple(k[2])] + list(k[3:])) for k in dev_keys(rules)]
    want = [tuple([r[0], tuple(r[1]), tuple(r[2])] + list(r[3:])) for r in fx["rules"]]
    assert got == want
    assert st.checked_ref == fx["checked"]
    exp, checked = O.search(targets, 1, dead=0xFF)
    key = lambda r: (r.target_index, tuple(r.src[:r.src_len]), tuple(r.rep[:r.rep_len]), r.bytes_saved,
                     r.cycles_saved, r.dead_flags)
    assert [key(r) for r in r2] == [key(r) for r in exp]
    assert st2.checked_ref == checked


@pytest.mark.parametrize("compact,wide", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_compact_sweep_keeps_parity(ctx, O, compact, wide):
    """Z80B_OPT_COMPACT_SWEEP and Z80B_OPT_WIDE_SWEEP off and on: the C3
    sample's rules and 'checked' counter, and a C2 sample against the
    oracle, are unchanged (compact: pairs naming at most two of B..L,
    A-dependent and A-independent, on the A/F/B/C-state kernel; wide: the
    other A-dependent pairs naming at most four of B..L and not SP, on the
    A/F/B/C/H/L/M-state kernel)."""
    import workloads
    fx = fixture()
    opts = [z80b.OPT_COMPACT_SWEEP, z80b.OPT_WIDE_SWEEP]
    old = [ctx.get_option(o) for o in opts]
    ctx.set_option(z80b.OPT_COMPACT_SWEEP, compact)
    ctx.set_option(z80b.OPT_WIDE_SWEEP, wide)
    try:
        rules, st = run(ctx, fx)
        targets = workloads.to_lists(workloads.c2_subset(3000, seed=12))
        r2, st2 = ctx.search(targets, dead_flags=0xFF)
    finally:
        for o, v in zip(opts, old):
            ctx.set_option(o, v)
    got = [tuple([k[0], tuple(k[1]), tuple(k[2])] + list(k[3:])) for k in dev_keys(rules)]
    want = [tuple([r[0], tuple(r[1]), tuple(r[2])] + list(r[3:])) for r in fx["rules"]]
    assert got == want
    assert st.checked_ref == fx["checked"]
    exp, checked = O.search(targets, 1, dead=0xFF)
    key = lambda r: (r.target_index, tuple(r.src[:r.src_len]), tuple(r.rep[:r.rep_len]), r.bytes_saved,
                     r.cycles_saved, r.dead_flags)
    assert [key(r) for r in r2] == [key(r) for r in exp]
    assert st2.checked_ref == checked


@pytest.mark.parametrize("case", ["c3", "c2"])
def test_device_rounds_equal_host_rounds(ctx, case):
    """The first-found rounds driven on the device (one CUDA graph, a WHILE
    node over build / scan / sweep / resolve), with the sweep classes on
    parallel branches of the graph or one after another, and driven from the
    host give the same rules, counters, rounds and swept pairs.  (The count
    of swept states is not compared: how far other warps get into a pair's
    sweep before they see it rejected is a matter of timing in every mode.)"""
    import workloads
    opts = [z80b.OPT_GRAPH_ROUNDS, z80b.OPT_CONCURRENT_SWEEPS]
    saved = [ctx.get_option(o) for o in opts]
    try:
        res = []
        for g, conc in ((1, 1), (1, 0), (0, 1)):
            ctx.set_option(z80b.OPT_GRAPH_ROUNDS, g)
            ctx.set_option(z80b.OPT_CONCURRENT_SWEEPS, conc)
            if case == "c3":
                rules, st = run(ctx, fixture())
            else:
                rules, st = ctx.search(workloads.to_lists(workloads.c2_subset(6000, seed=4)), dead_flags=0xFF)
            res.append((dev_keys(rules), st.checked_ref, st.checks, st.rounds, st.exhaustive_pairs))
        assert res[0] == res[1] == res[2]
        assert res[0][3] > 1  # several rounds
    finally:
        for o, v in zip(opts, saved):
            ctx.set_option(o, v)
