"""Regenerates the golden fixtures derived from the reference's data files.

Usage: python tests/golden/make_fixtures.py REFERENCE_ROOT, where
REFERENCE_ROOT is a checkout of oisee/z80-optimizer.  Writes:
  peephole_top500_pairs.json -- (source, replacement, bytes_saved,
      cycles_saved) of the reference's data/peephole_top500.json, the 500
      rules its CUDA pipeline reported for length-2 targets.  Every pair is
      an equivalence the ExhaustiveCheck of pkg/search must accept.
  mulopt8_published.json -- (k, ops, length, tstates) of the reference's
      data/mulopt8_clobber.json: the shortest A*K sequences for all 254
      constants over the 14-op pool of cuda/z80_mulopt_fast.cu.  Length and
      T-states are deterministic; which of several equal-cost sequences the
      reference printed was decided by a race in its kernel.
reference_known_answers.json is transcribed by hand from the reference's
Go tests (each case cites its file:line) and is not regenerated here.
"""
import json
import os
import sys

if len(sys.argv) != 2:
    sys.exit(__doc__)
ref = sys.argv[1]
here = os.path.dirname(os.path.abspath(__file__))
src = json.load(open(os.path.join(ref, "data", "peephole_top500.json")))
pairs = [{"source": r["source"], "replacement": r["replacement"],
          "bytes_saved": r["bytes_saved"], "cycles_saved": r["cycles_saved"]} for r in src]
with open(os.path.join(here, "peephole_top500_pairs.json"), "w") as f:
    json.dump({"_about": "derived from data/peephole_top500.json of the reference by make_fixtures.py",
               "pairs": pairs}, f, indent=1)
print(len(pairs), "pairs")

mul = json.load(open(os.path.join(ref, "data", "mulopt8_clobber.json")))
rows = [{"k": r["k"], "ops": r["ops"], "length": r["length"], "tstates": r["tstates"]} for r in mul]
with open(os.path.join(here, "mulopt8_published.json"), "w") as f:
    json.dump({"_about": "derived from data/mulopt8_clobber.json of the reference by make_fixtures.py "
                         "(pool: cuda/z80_mulopt_fast.cu, 14 ops, all state zero but A)",
               "results": rows}, f, indent=1)
print(len(rows), "mulopt8 results")
