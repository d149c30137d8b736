"""The allocation-free ExhaustiveCheck entry point against z80b_verify_pairs.

z80b_exhaustive_noalloc exists for callers that cannot allocate device
memory (their GPU memory is budgeted elsewhere, or an allocation's implicit
synchronization is not acceptable on their path).  It keeps its scratch in a
fixed array inside the library, so these checks call it twice in a row (the
second call must not see the first call's leftovers) and compare both
results, bit for bit, with the regular context-based entry point and with
the CPU oracle's ExhaustiveCheck.  This
file is collected last so that a failure here stops a -x run only after
every other test has run.
"""
import ctypes
import random

import pytest

import workloads
import z80b

pytestmark = pytest.mark.gpu


def _noalloc(pairs, dead, stride=4):
    L = z80b.lib()
    f = L.z80b_exhaustive_noalloc
    u32p, u8p = ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint8)
    f.argtypes = [ctypes.c_int, u32p, u8p, u32p, u8p, ctypes.c_uint32, ctypes.c_uint32, u8p, u8p,
                  ctypes.c_void_p]
    n = len(pairs)
    t = (ctypes.c_uint32 * max(1, n * stride))()
    c = (ctypes.c_uint32 * max(1, n * stride))()
    tl = (ctypes.c_uint8 * max(1, n))()
    cl = (ctypes.c_uint8 * max(1, n))()
    for i, (a, b) in enumerate(pairs):
        tl[i], cl[i] = len(a), len(b)
        for j, w in enumerate(a):
            t[i * stride + j] = w
        for j, w in enumerate(b):
            c[i * stride + j] = w
    d = (ctypes.c_uint8 * max(1, n))(*dead)
    out = (ctypes.c_uint8 * max(1, n))()
    st = f(0, t, tl, c, cl, stride, n, d, out, None)
    return st, list(out[:n])


def _pairs(seed, n_random):
    rng = random.Random(seed)
    pool = z80b.pool8()
    o = workloads.ops()
    P = z80b.pack
    pairs = [([P(o["AND_N"], 0xFF)], [P(o["AND_A"])]),
             ([P(o["LD_A_N"], 0)], [P(o["XOR_A"])]),
             ([P(o["SUB_A"]), P(o["LD_A_N"], 0)], [P(o["SUB_A"])]),
             ([P(o["LD_B_A"]), P(o["LD_A_B"])], [P(o["LD_B_A"])]),
             ([P(o["ADD_A_B"])], [P(o["SUB_B"])])]
    pairs += [([rng.choice(pool), rng.choice(pool)], [rng.choice(pool)]) for _ in range(n_random)]
    deads = [rng.choice([0x00, 0x28, 0xFF]) for _ in pairs]
    return pairs, deads


def test_noalloc_matches_verify_pairs_twice(ctx, O):
    for call, seed in enumerate((1, 2)):
        pairs, deads = _pairs(seed, 300)
        st, got = _noalloc(pairs, deads)
        assert st == z80b.OK, st
        want = [(bits >> 2) & 1 for bits, _ in ctx.verify_pairs(pairs, dead=deads, tiers=z80b.TIER_EXH)]
        assert got == want, f"call {call}"
        # and against the oracle's ExhaustiveCheckMasked (verifier.go:642-654) directly
        assert got == [int(O.exhaustive(t, c, d)) for (t, c), d in zip(pairs, deads)], f"call {call}"
        assert any(got) and not all(got)


def test_noalloc_keeps_the_callers_current_device(ctx):
    import torch
    before = torch.cuda.current_device()
    pairs, deads = _pairs(4, 20)
    st, _ = _noalloc(pairs, deads)
    assert st == z80b.OK
    assert torch.cuda.current_device() == before


def test_noalloc_rejects_oversize(ctx):
    pairs, deads = _pairs(3, 0)
    n = 4097
    big = (pairs * (n // len(pairs) + 1))[:n]
    st, _ = _noalloc(big, (deads * (n // len(deads) + 1))[:n])
    assert st == z80b.ECAPACITY
