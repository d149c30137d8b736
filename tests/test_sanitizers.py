"""Host code under AddressSanitizer and UndefinedBehaviorSanitizer: the
JSON reader, the export and peephole functions, the ranged enumeration
(search_api.cpp) and the table code behind the compact sweep
(z80_tables.cpp), through their native checks.  No device is needed."""
import os
import subprocess

import pytest

from conftest import ROOT

SAN = ["-O1", "-g", "-std=c++17", "-fsanitize=address,undefined", "-fno-sanitize-recover=all"]
BUILD = os.path.join(ROOT, "z80-optimizer_b200", "_build")
HOST = os.path.join(ROOT, "z80-optimizer_b200", "csrc", "host")
ORACLE = [os.path.join(ROOT, "oracle", "z80_oracle_isa_cpu.cpp"), os.path.join(ROOT, "oracle", "z80_oracle_search.cpp")]


def build(tmp_path, name, srcs, with_lib):
    exe = tmp_path / (name + "_san")
    cmd = ["g++", *SAN, "-o", str(exe), os.path.join(ROOT, "tests", "native", name + ".cpp"), *srcs]
    if with_lib:
        cmd += ["-I" + HOST, "-I" + os.path.join(ROOT, "include"), "-L" + BUILD, "-lz80b200", "-Wl,-rpath," + BUILD]
    r = subprocess.run(cmd + ["-lpthread"], capture_output=True, text=True)
    if r.returncode != 0 and "sanitize" in r.stderr:
        pytest.skip("no sanitizer runtime for this compiler")
    assert r.returncode == 0, r.stderr
    return exe


def run(exe, *args):
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0", UBSAN_OPTIONS="print_stacktrace=1")
    return subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=900, env=env)


def test_search_api_under_sanitizers(tmp_path):
    exe = build(tmp_path, "export_check", [os.path.join(HOST, "search_api.cpp")], True)
    r = run(exe, tmp_path)
    assert r.returncode == 0 and r.stdout.startswith("OK"), r.stdout + r.stderr
    exe = build(tmp_path, "enum_check", [os.path.join(HOST, "search_api.cpp"), *ORACLE], True)
    r = run(exe)
    assert r.returncode == 0 and r.stdout.startswith("OK"), r.stdout + r.stderr


def test_json_reader_edge_inputs_under_sanitizers(tmp_path):
    exe = build(tmp_path, "json_echo", [os.path.join(HOST, "search_api.cpp")], True)
    cases = ['[{"source_asm": "a\\u00e9\\ud83d\\ude00\\ud800x", "bytes_saved": -3, "z": [1, {"y": null}]}, null]',
             "", " ", "[", "[{", '[{"a"', '[{"a":', '[{"a":1,', '"\\u12', '"\\ud83d\\u12"', "[" * 300 + "]" * 300,
             '[{"cycles_saved": 1e999}]', '[{"cycles_saved": -0.0}]', "[1e", "nul", "[tru]", '["\\', '["\\q"]']
    for i, text in enumerate(cases):
        f = tmp_path / f"c{i}.json"
        f.write_text(text)
        r = run(exe, f)
        assert r.returncode == 0, (text, r.stderr[-2000:])


def test_table_code_under_sanitizers(tmp_path):
    exe = build(tmp_path, "compact_check", [os.path.join(ROOT, "z80-optimizer_b200", "csrc", "z80_tables.cpp"),
                                            *ORACLE], False)
    r = run(exe)
    assert r.returncode == 0 and r.stdout.startswith("OK"), r.stdout + r.stderr
