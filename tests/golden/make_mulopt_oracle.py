"""Regenerates mulopt_oracle.json: cmd/mulopt findOptimal results of the CPU
oracle (oracle/z80_oracle_mulopt.cpp) for K = 2..32 over every pool.

    python tests/golden/make_mulopt_oracle.py [processes]

Pools and limits (the oracle walks pool^L sequences per K and length, so the
longest lengths take CPU-hours; results up to these limits are exact):
  mulopt14 (cmd/mulopt/main.go)      init zero, lengths 1..8
  wide21   (workload pool)           B, C, F from splitmix64(seed 2), lengths 1..8
  fast14   (cuda/z80_mulopt_fast.cu) init zero, lengths 1..8
  cuda21   (cuda/z80_mulopt.cu)      init zero, lengths 1..7
A constant with no sequence within its pool's limit is recorded with
length 0 ("not found up to max_len").
"""
import json
import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "..", "z80-optimizer_b200"))

POOLS = {  # name: (oracle pool id, max_len, uses the seeded init)
    "mulopt14": (0, 8, False),
    "wide21": (1, 8, True),
    "fast14": (2, 8, False),
    "cuda21": (3, 7, False),
}
KS = range(2, 33)


def seeded_init():
    import workloads
    return workloads.mul_init(2)


def task(arg):
    import oracle_lib
    name, k, b, c, f = arg
    pool, max_len, _ = POOLS[name]
    t0 = time.time()
    r = oracle_lib.mul_find_pool(pool, k, 1, max_len, b, c, f)
    dt = time.time() - t0
    if r is None:
        return name, k, {"k": k, "length": 0, "tstates": 0, "ops": []}, dt
    ln, t, ops = r
    return name, k, {"k": k, "length": ln, "tstates": t, "ops": ops}, dt


def main():
    procs = int(sys.argv[1]) if len(sys.argv) > 1 else os.cpu_count()
    b, c, f = seeded_init()
    tasks = []
    for name, (_, _, seeded) in POOLS.items():
        ib, ic, iff = (b, c, f) if seeded else (0, 0, 0)
        tasks += [(name, k, ib, ic, iff) for k in KS]
    out = {name: {} for name in POOLS}
    with mp.get_context("spawn").Pool(procs) as p:
        for name, k, r, dt in p.imap_unordered(task, tasks):
            out[name][k] = r
            print(f"{name} K={k}: length {r['length']} tstates {r['tstates']} ({dt:.1f} s)", flush=True)
    doc = {"_about": "cmd/mulopt findOptimal (shortest, then fewest T-states, then first in odometer order) "
                     "by the CPU oracle; generated by make_mulopt_oracle.py",
           "pools": {}}
    for name, (pool, max_len, seeded) in POOLS.items():
        doc["pools"][name] = {"pool": pool, "max_len": max_len,
                              "init": {"b": b, "c": c, "f": f} if seeded else {"b": 0, "c": 0, "f": 0},
                              "results": [out[name][k] for k in KS]}
    with open(os.path.join(HERE, "mulopt_oracle.json"), "w") as fh:
        json.dump(doc, fh, indent=1)


if __name__ == "__main__":
    main()
