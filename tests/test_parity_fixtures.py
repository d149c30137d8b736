"""The oracle fixtures that pin the GPU parity tests at the configured sizes.

c2_100k_oracle.json and c1_full_oracle.json (make_parity_fixtures.py) hold
the oracle's first-found rules for the C2 parity subset (100,000 targets)
and for every C1 target.  Here, without a GPU: the target sets that the
oracle enumerated equal the library's enumeration (same digest), and the
oracle as built now reproduces the stored rules on a slice of each set.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import workloads

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def digest(arr):
    return hashlib.sha256(np.ascontiguousarray(arr, dtype="<u4").tobytes()).hexdigest()


def load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def keys_of(rules, lo, hi):
    return [(r[0] - lo, tuple(r[1]), tuple(r[2]), r[3], r[4], r[5]) for r in rules if lo <= r[0] < hi]


@pytest.mark.parametrize("name,make_o,make_w", [
    ("c2_100k_oracle.json", lambda O: O.c2_subset(100000, seed=0), lambda: workloads.c2_subset(100000, seed=0)),
    ("c1_full_oracle.json", lambda O: O.c1_targets(), lambda: workloads.c1_targets()),
])
def test_fixture_targets_and_slice(O, name, make_o, make_w):
    fx = load(name)
    arr = make_o(O)
    assert len(arr) == fx["n_targets"]
    assert digest(arr) == fx["targets_sha256"]
    assert digest(make_w()) == fx["targets_sha256"]
    lo, hi = 0, 400
    for p in fx["passes"]:
        rules, _ = O.search([list(map(int, r)) for r in arr[lo:hi]], 1, dead=p["dead_flags"])
        got = [(r.target_index, tuple(r.src[:r.src_len]), tuple(r.rep[:r.rep_len]), r.bytes_saved,
                r.cycles_saved, r.dead_flags) for r in rules]
        assert got == keys_of(p["rules"], lo, hi), p["dead_flags"]
