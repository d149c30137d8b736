"""Constant-multiply search on the device (z80b_mul_search) against the CPU
oracle's findOptimal and the reference's published table.

Bit-exact: per K the found flag, length, T-states and the sequence itself
(shortest, then fewest T-states, then first in odometer order)."""
import json
import os

import pytest

import z80b
from conftest import ROOT

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(ROOT, "tests", "golden")
POOL_IDS = {"mulopt14": 0, "wide21": 1, "fast14": 2, "cuda21": 3}


def oracle_fixture():
    return json.load(open(os.path.join(GOLDEN, "mulopt_oracle.json")))["pools"]


@pytest.mark.parametrize("name", ["mulopt14", "wide21", "fast14", "cuda21"])
def test_matches_oracle_k2_32(ctx, name):
    p = oracle_fixture()[name]
    i = p["init"]
    res, st = ctx.mul_search(POOL_IDS[name], (i["b"], i["c"], i["f"]), 1, p["max_len"], ks=range(2, 33))
    got = [(r["k"], r["length"] if r["found"] else 0, r["tstates"] if r["found"] else 0, r["ops"])
           for r in res]
    want = [(r["k"], r["length"], r["tstates"], r["ops"]) for r in p["results"]]
    assert got == want
    assert st.full_pass >= sum(1 for r in p["results"] if r["length"])


def test_fast14_all_constants_match_published(ctx, O):
    """All 254 constants of data/mulopt8_clobber.json (lengths up to 11) in
    one search; the length and T-states are the reference's, and every
    returned sequence computes x*K under the oracle."""
    rows = json.load(open(os.path.join(GOLDEN, "mulopt8_published.json")))["results"]
    res, st = ctx.mul_search(z80b.MULPOOL_FAST14, (0, 0, 0), 1, 11)
    assert [r["k"] for r in res] == list(range(2, 256))
    for r, want in zip(res, rows):
        assert r["found"], r
        assert (r["length"], r["tstates"]) == (want["length"], want["tstates"]), (r, want)
        assert sum(O.mul_tstates_pool(2, i) for i in r["ops"]) == r["tstates"]
        assert all(O.mul_run_pool(2, r["ops"], x) == (x * r["k"]) & 0xFF for x in range(256)), r
    assert st.lengths == 11


def test_alone_equals_in_the_mix(ctx):
    """A constant searched alone gets the same answer as in the full batch."""
    init = (0xCE, 0x42, 0x2F)
    mix, _ = ctx.mul_search(z80b.MULPOOL_WIDE21, init, 1, 6)
    by_k = {r["k"]: r for r in mix}
    for k in (3, 7, 11, 16, 37, 200, 255):
        alone, _ = ctx.mul_search(z80b.MULPOOL_WIDE21, init, 1, 6, ks=[k])
        assert alone[0] == by_k[k]


def test_min_len_skips_shorter(ctx):
    full, _ = ctx.mul_search(z80b.MULPOOL_MULOPT, (0, 0, 0), 1, 6)
    part, _ = ctx.mul_search(z80b.MULPOOL_MULOPT, (0, 0, 0), 4, 6)
    for a, b in zip(full, part):
        if a["found"] and a["length"] >= 4:
            assert a == b
        if b["found"]:
            assert b["length"] >= 4


def test_rejects_bad_arguments(ctx):
    for kw in ({"ks": [1]}, {"ks": [256]}, {"max_len": 13}, {"min_len": 0}):
        args = dict(pool=z80b.MULPOOL_FAST14, min_len=1, max_len=4)
        args.update(kw)
        with pytest.raises(z80b.Z80BError) as e:
            ctx.mul_search(**args)
        assert e.value.status == z80b.EINVAL
    with pytest.raises(z80b.Z80BError):
        ctx.mul_search(7, max_len=3)
