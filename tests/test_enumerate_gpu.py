"""Sharded and streamed enumeration on the device: `z80opt enumerate` over a
first-instruction range with length-3 targets, rules streamed as JSON lines,
and the all-hits mode without the ExhaustiveCheck tier (--no-exhaust)."""
import json
import os
import subprocess

import pytest

import workloads
import z80b
from conftest import ROOT

EXE = os.path.join(ROOT, "z80-optimizer_b200", "_build", "z80opt")


def run(*args):
    return subprocess.run([EXE, *args], capture_output=True, text=True, timeout=900)


def rule_keys(rules):
    return [(r.target_index, tuple(r.src[:r.src_len]), tuple(r.rep[:r.rep_len]), r.bytes_saved, r.cycles_saved,
             r.dead_flags) for r in rules]


@pytest.mark.gpu
def test_enumerate_range_length3_jsonl(tmp_path, O):
    """Length-2 and length-3 targets whose first instruction is in [1200,
    1210), sampled: the JSON lines equal the table output of the same
    command, every source starts inside the range, and every rule passes the
    oracle's ExhaustiveCheck."""
    args = ["enumerate", "--max-target", "3", "--first-op-start", "1200", "--first-op-end", "1210",
            "--sample", "1500", "--seed", "11"]
    jl = tmp_path / "r.jsonl"
    r = run(*args, "--jsonl", str(jl))
    assert r.returncode == 0, r.stderr
    lines = [json.loads(x) for x in open(jl)]
    out = tmp_path / "r.json"
    r = run(*args, "--output", str(out))
    assert r.returncode == 0, r.stderr
    table = json.load(open(out))
    key = lambda x: (x["source_asm"], x["replacement_asm"], x["bytes_saved"], x["cycles_saved"])
    assert sorted(map(key, lines)) == sorted(map(key, table))
    assert len(lines) > 20
    pool = z80b.pool8()
    first = set(pool[1200:1210])
    n3 = 0
    for x in lines:
        src, rep = O.parse_assembly(x["source_asm"]), O.parse_assembly(x["replacement_asm"])
        assert src[0] in first
        # candidates up to MaxTargetLen - 1 = 2 instructions for every target
        # length (pkg/search/search.go:27-29,66-73), fewer bytes
        assert len(rep) <= 2 and x["bytes_saved"] > 0
        assert O.exhaustive(src, rep, 0), x
        n3 += len(src) == 3
    assert n3 > 0


@pytest.mark.gpu
def test_all_hits_without_exhaustive_tier(ctx, O):
    """Z80B_JOB_NO_EXHAUSTIVE: the rules are every QuickCheck + MidCheck
    survivor, a superset of the verified rules; the extra ones fail the
    oracle's ExhaustiveCheck."""
    ctx.load_candidates(z80b.pool8(), 1)
    targets = workloads.to_lists(workloads.c2_subset(400, seed=31))
    full, _ = ctx.search(targets, dead_flags=0x28, mode=z80b.MODE_ALL)
    raw, _ = ctx.search(targets, dead_flags=0x28, mode=z80b.MODE_ALL, no_exhaustive=True)
    fk, rk = set(rule_keys(full)), set(rule_keys(raw))
    assert fk <= rk and len(rk) > len(fk)
    for r in raw:
        t, c = list(r.src[:r.src_len]), list(r.rep[:r.rep_len])
        assert O.quickcheck(t, c, 0x28) and O.midcheck(t, c, 0x28)
        k = rule_keys([r])[0]
        assert O.exhaustive(t, c, 0x28) == (k in fk)
    with pytest.raises(z80b.Z80BError):
        ctx.search(targets[:5], no_exhaustive=True)  # needs the all-hits mode
