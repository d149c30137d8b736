"""bench.py's reference arm: the oracle alone, on the GPU arm's config.

The reference arm times the CPU restatement of the reference's search; it
must not load the library it is compared with, and its JSON line must name
the same workload as the GPU arm's (same metric, unit and config), with the
e2e object of a CPU run.
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import json, runpy, sys
sys.argv = ['bench.py', '--impl', 'reference', '--cpu-sample', '400', '--steps', '2', '--warmup', '1']
try:
    runpy.run_path('bench.py', run_name='__main__')
except SystemExit:
    pass
maps = open('/proc/self/maps').read()
print('MAPS', json.dumps({'product': 'libz80b200' in maps, 'oracle': 'liboracle' in maps}))
"""


def test_reference_arm_loads_only_the_oracle():
    out = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True,
                         timeout=600, check=True).stdout.splitlines()
    line = json.loads(next(x for x in out if x.startswith("{")))
    maps = json.loads(next(x for x in out if x.startswith("MAPS "))[5:])
    assert maps == {"product": False, "oracle": True}
    sys.path.insert(0, ROOT)
    import bench
    args = bench.parse(["--impl", "reference"])
    assert line["config"] == bench.workload_config(args, 1)
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["higher_is_better"] is True and line["steps"] == 2
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == line["value"] and cb["cores"] >= 1
