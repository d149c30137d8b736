"""Constant-multiply search (cmd/mulopt) on the host side: the instruction
model of the search kernels against the oracle, the oracle against the
reference's published table, and the pool descriptions of the C ABI."""
import json
import os
import subprocess

import pytest

import z80b
from conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden")


def test_mul_model_matches_oracle(tmp_path):
    """z80b_mul_ops.cuh (4 inputs per word) = oracle MulRunPool, all pools."""
    exe = tmp_path / "mul_check"
    srcs = [os.path.join(ROOT, "tests", "native", "mul_check.cpp")] + [
        os.path.join(ROOT, "oracle", f) for f in
        ("z80_oracle_isa_cpu.cpp", "z80_oracle_search.cpp", "z80_oracle_mulopt.cpp")]
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe)] + srcs + ["-lpthread"], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("OK")


def published():
    return json.load(open(os.path.join(GOLDEN, "mulopt8_published.json")))["results"]


def test_published_sequences_verify_under_oracle(O):
    """Every sequence of data/mulopt8_clobber.json computes x*K for all x
    under the oracle's model of cuda/z80_mulopt_fast.cu, with its T-states."""
    names = [O.mul_op_name(O.MUL_POOL_FAST, i) for i in range(O.mul_pool_size(2))]
    rows = published()
    assert len(rows) == 254 and [r["k"] for r in rows] == list(range(2, 256))
    for r in rows:
        seq = [names.index(n) for n in r["ops"]]
        assert len(seq) == r["length"]
        assert sum(O.mul_tstates_pool(2, i) for i in seq) == r["tstates"]
        assert all(O.mul_run_pool(2, seq, x) == (x * r["k"]) & 0xFF for x in range(256)), r


def test_oracle_optimum_matches_published_short(O):
    """findOptimal of the oracle reproduces the published length and T-states
    where the table's sequences are short (the longer ones are CPU-hours)."""
    for r in published():
        if r["length"] > 5:
            continue
        got = O.mul_find_pool(2, r["k"], 1, r["length"])
        assert got is not None and (got[0], got[1]) == (r["length"], r["tstates"]), (r, got)


@pytest.mark.parametrize("pool", [0, 1, 2, 3])
def test_pool_description_matches_oracle(O, pool):
    names, ts, max_len = z80b.mul_pool(pool)
    assert len(names) == O.mul_pool_size(pool)
    assert names == [O.mul_op_name(pool, i) for i in range(len(names))]
    assert ts == [O.mul_tstates_pool(pool, i) for i in range(len(names))]
    assert len(names) ** max_len < 1 << 48 <= len(names) ** (max_len + 1)


def test_oracle_fixture_rederives(O):
    """The committed oracle fixture agrees with a fresh oracle run on its
    cheap entries (length <= 5)."""
    path = os.path.join(GOLDEN, "mulopt_oracle.json")
    if not os.path.exists(path):
        pytest.skip("mulopt_oracle.json not generated")
    doc = json.load(open(path))
    n = 0
    for name, p in doc["pools"].items():
        i = p["init"]
        for r in p["results"]:
            if 0 < r["length"] <= 5:
                got = O.mul_find_pool(p["pool"], r["k"], 1, 5, i["b"], i["c"], i["f"])
                assert got == (r["length"], r["tstates"], r["ops"]), (name, r, got)
                n += 1
    assert n > 20


def test_json_format():
    res = [{"k": 3, "found": True, "length": 3, "tstates": 12, "ops": [3, 0, 1], "index": 0},
           {"k": 4, "found": False, "length": 0, "tstates": 0, "ops": [], "index": 0}]
    text = z80b.mul_results_json(res, z80b.MULPOOL_MULOPT)
    assert json.loads(text) == [{"k": 3, "ops": ["LD B,A", "ADD A,A", "ADD A,B"], "length": 3, "tstates": 12}]
    assert text.startswith("[\n  {\n    \"k\": 3,")
