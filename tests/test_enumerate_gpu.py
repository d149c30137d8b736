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
def test_enumerate_range_length3_equals_oracle(tmp_path, O):
    """A sampled length-2/3 enumeration over the first-instruction range
    [1200, 1210): the searched targets (--targets-out) run through the
    oracle's first-found search (worker.go:124-265, candidates up to
    MaxTargetLen - 1 = 2 instructions) give exactly the rule set the CLI
    reports."""
    tl, out = tmp_path / "t.jsonl", tmp_path / "r.json"
    r = run("enumerate", "--max-target", "3", "--first-op-start", "1200", "--first-op-end", "1210",
            "--sample", "300", "--seed", "5", "--targets-out", str(tl), "--output", str(out))
    assert r.returncode == 0, r.stderr
    targets = [json.loads(x) for x in open(tl)]
    assert len(targets) == 600  # 300 per target length
    assert {len(t) for t in targets} == {2, 3}
    pool = z80b.pool8()
    first = set(pool[1200:1210])
    assert all(t[0] in first for t in targets)
    got = sorted((x["source_asm"], x["replacement_asm"], x["bytes_saved"], x["cycles_saved"])
                 for x in json.load(open(out)))
    rules, _ = O.search(targets, 2)
    want = sorted((O.disasm(list(x.src[:x.src_len])), O.disasm(list(x.rep[:x.rep_len])), x.bytes_saved,
                   x.cycles_saved) for x in rules)
    assert got == want
    assert any(len(O.parse_assembly(g[0])) == 3 for g in got)


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


@pytest.mark.gpu
def test_stoke_verifier_calls_host_api(tmp_path, O):
    """ExhaustiveCheck[Masked] and FlagDiff through the C++ host API, the
    calls pkg/stoke/search.go:108-117 makes, against the oracle."""
    build = os.path.join(ROOT, "z80-optimizer_b200", "_build")
    exe = tmp_path / "stoke_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe), os.path.join(ROOT, "tests", "native", "stoke_check.cpp"),
                    os.path.join(ROOT, "z80-optimizer_b200", "csrc", "host", "search_api.cpp"),
                    "-I" + os.path.join(ROOT, "z80-optimizer_b200", "csrc", "host"),
                    "-I" + os.path.join(ROOT, "include"), "-L" + build, "-lz80b200", "-Wl,-rpath," + build,
                    "-lpthread"], check=True)
    pool = z80b.pool8()
    rng = __import__("random").Random(17)
    o = O.ops()
    pairs = [([O.pack(o["SUB_A"]), O.pack(o["LD_A_N"], 0)], [O.pack(o["SUB_A"])], 0),
             ([O.pack(o["LD_A_N"], 0), O.pack(o["NEG"])], [O.pack(o["SUB_A"])], 0xFF),
             ([O.pack(o["AND_N"], 0xFF)], [O.pack(o["OR_N"], 0)], 0x10)]
    for _ in range(60):
        t = [rng.choice(pool) for _ in range(rng.choice((1, 2)))]
        pairs.append((t, [rng.choice(pool)], rng.choice((0, 0xFF, 0x28))))
    f = tmp_path / "pairs.txt"
    f.write_text("".join(f"{d:x} " + " ".join(f"{w:x}" for w in t) + " ; " + " ".join(f"{w:x}" for w in c) + "\n"
                         for t, c, d in pairs))
    r = subprocess.run([str(exe), str(f)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    got = [tuple(map(int, x.split())) for x in r.stdout.splitlines()]
    assert got == [(int(O.exhaustive(t, c, d)), O.flagdiff(t, c)) for t, c, d in pairs]
    assert any(g[0] for g in got)
