"""Host-side parts of the enumeration and export rows: `z80opt export`
(result.WriteGoCode text and the generated peephole table package), the
JSON reader and peephole table functions of the C++ host API, and the ranged
target enumeration behind `enumerate --first-op-start/--first-op-end`.  No
device is needed."""
import json
import os
import subprocess

from conftest import ROOT

EXE = os.path.join(ROOT, "z80-optimizer_b200", "_build", "z80opt")

RULES = [
    {"source_asm": "SUB A : LD A, 00h", "replacement_asm": "SUB A", "source_bytes": 3,
     "replacement_bytes": 1, "bytes_saved": 2, "cycles_saved": 7},
    {"source_asm": "OR A : AND A", "replacement_asm": "AND A", "source_bytes": 2,
     "replacement_bytes": 1, "bytes_saved": 1, "cycles_saved": 4, "dead_flags": "10",
     "dead_flag_desc": "H"},
    {"source_asm": "LD B, 0A5h : LD C, 0FFh", "replacement_asm": "LD C, 0FFh : LD B, 0A5h",
     "source_bytes": 4, "replacement_bytes": 4, "bytes_saved": 0, "cycles_saved": 0, "dead_flags": "FF",
     "dead_flag_desc": "all"},
]

DESC = {0x10: "H", 0xFF: "all"}


def expected_go(rules):
    """output.go:95-125's text for these rules, written out independently."""
    out = ["// Code generated by z80opt. DO NOT EDIT.", "", "package optimizer", "",
           "// Z80OptRules contains peephole optimization rules discovered by the superoptimizer.",
           "var Z80OptRules = []PeepholeRule{"]
    for r in rules:
        dead = int(r.get("dead_flags", "0"), 16)
        head = f"\t// {r['source_asm']} -> {r['replacement_asm']} (-{r['bytes_saved']} bytes, -{r['cycles_saved']} cycles)"
        out.append(head + (f" [dead: {DESC[dead]}]" if dead else ""))
        out.append("\t{")
        q = lambda asm: ", ".join(json.dumps(x) for x in asm.split(" : "))
        out.append(f"\t\tMatch: []string{{{q(r['source_asm'])}}},")
        out.append(f"\t\tReplace: []string{{{q(r['replacement_asm'])}}},")
        if dead:
            out.append(f"\t\tDeadFlags: 0x{dead:02X}, // {DESC[dead]}")
        out.append("\t},")
    out.append("}")
    return "\n".join(out) + "\n"


def run(*args):
    return subprocess.run([EXE, *args], capture_output=True, text=True, timeout=60)


def test_export_go_code(tmp_path):
    f = tmp_path / "rules.json"
    f.write_text(json.dumps(RULES, indent=2))
    r = run("export", str(f))
    assert r.returncode == 0, r.stderr
    assert r.stdout == expected_go(RULES)
    out = tmp_path / "rules.go"
    r = run("export", str(f), "-f", "go", "-o", str(out))
    assert r.returncode == 0 and out.read_text() == expected_go(RULES)


def test_export_peephole_table(tmp_path):
    f = tmp_path / "top.json"
    f.write_text(json.dumps(RULES))
    r = run("export", str(f), "-f", "peephole", "--var", "Top3")
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    assert lines[0] == "// Code generated from top.json. DO NOT EDIT."
    assert lines[1] == "package peephole"
    body = lines[lines.index("var Top3 = map[string]Rule{") + 1:]
    body = body[:body.index("}")]
    assert body == [f"\t{json.dumps(x['source_asm'])}: {{{json.dumps(x['replacement_asm'])}, "
                    f"{x['cycles_saved']}, {x['bytes_saved']}}}," for x in RULES]
    assert "func Lookup(source string) *Rule {" in lines
    assert "func LoadRules(path string) (map[string]Rule, error) {" in lines


def test_export_rejects_bad_input(tmp_path):
    bad = tmp_path / "bad.json"
    bad.write_text('{"source_asm": "NOP"}')
    r = run("export", str(bad))
    assert r.returncode == 1 and "not an array" in r.stderr
    unparsable = tmp_path / "u.json"
    unparsable.write_text('[{"source_asm": "FROB A", "replacement_asm": "NOP"}]')
    r = run("export", str(unparsable))
    assert r.returncode == 1 and "cannot parse source assembly" in r.stderr
    good = tmp_path / "g.json"
    good.write_text(json.dumps(RULES))
    r = run("export", str(good), "-f", "yaml")
    assert r.returncode == 1 and "unknown format: yaml" in r.stderr


def test_json_reader_and_peephole_api(tmp_path):
    """ReadJSON follows encoding/json on rule files (case-insensitive keys,
    unknown keys skipped, null values, escapes, integers only), LoadRules
    keeps the last entry of a source, Lookup finds entries."""
    exe = tmp_path / "export_check"
    build = os.path.join(ROOT, "z80-optimizer_b200", "_build")
    subprocess.run(["g++", "-O1", "-std=c++17", "-o", str(exe),
                    os.path.join(ROOT, "tests", "native", "export_check.cpp"),
                    os.path.join(ROOT, "z80-optimizer_b200", "csrc", "host", "search_api.cpp"),
                    "-I" + os.path.join(ROOT, "z80-optimizer_b200", "csrc", "host"),
                    "-I" + os.path.join(ROOT, "include"), "-L" + build, "-lz80b200",
                    "-Wl,-rpath," + build, "-lpthread"], check=True)
    r = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("OK")


def _native(tmp_path, name, extra=()):
    exe = tmp_path / name
    build = os.path.join(ROOT, "z80-optimizer_b200", "_build")
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe),
                    os.path.join(ROOT, "tests", "native", name + ".cpp"),
                    os.path.join(ROOT, "z80-optimizer_b200", "csrc", "host", "search_api.cpp"), *extra,
                    "-I" + os.path.join(ROOT, "z80-optimizer_b200", "csrc", "host"),
                    "-I" + os.path.join(ROOT, "include"), "-L" + build, "-lz80b200",
                    "-Wl,-rpath," + build, "-lpthread"], check=True)
    return exe


def test_ranged_target_enumeration(tmp_path):
    """EnumerateTargets: whole and split ranges equal the full enumeration,
    samples follow Floyd's algorithm (length 2) or are uniform distinct
    unpruned draws (length 3), length-3 ranges match the oracle's pruner."""
    exe = _native(tmp_path, "enum_check", [os.path.join(ROOT, "oracle", "z80_oracle_isa_cpu.cpp"),
                                           os.path.join(ROOT, "oracle", "z80_oracle_search.cpp")])
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("OK")


def test_enumerate_flag_checks():
    r = run("enumerate", "--max-target", "4")
    assert r.returncode == 1 and "--max-target must be 2 or 3" in r.stderr
    r = run("enumerate", "--no-exhaust")
    assert r.returncode == 1 and "--no-exhaust needs --gpu" in r.stderr


def test_json_reader_against_python_json(tmp_path):
    """ReadJSON against Python's json module on generated rule files: random
    strings (escapes, control characters, non-ASCII, surrogate pairs),
    integers, nulls, unknown nested fields, random whitespace; and broken
    files are rejected."""
    import random
    exe = _native(tmp_path, "json_echo")
    rng = random.Random(5)
    alphabet = "ABC :,'\"\\/\t\né中\U0001F600\x01"
    fields = ["source_asm", "replacement_asm", "source_bytes", "replacement_bytes", "bytes_saved", "cycles_saved",
              "dead_flags", "dead_flag_desc"]

    def rstr():
        return "".join(rng.choice(alphabet) for _ in range(rng.randint(0, 12)))

    for case in range(40):
        rules = []
        for _ in range(rng.randint(0, 6)):
            obj = {}
            for k in fields:
                if rng.random() < 0.8:
                    if k.endswith(("bytes", "saved")):
                        obj[k] = rng.choice([None, rng.randint(-2**31, 2**31 - 1)])
                    else:
                        obj[k] = rng.choice([None, rstr()])
            if rng.random() < 0.5:
                obj["extra"] = {"x": [1, 2.5, {"y": None}], "z": rstr()}
            items = list(obj.items())
            rng.shuffle(items)
            rules.append(dict(items))
        text = json.dumps(rules, ensure_ascii=rng.random() < 0.5, indent=rng.choice([None, 1, 4]))
        f = tmp_path / f"c{case}.json"
        f.write_bytes(text.encode("utf-8"))
        r = subprocess.run([str(exe), str(f)], capture_output=True, text=True, timeout=60)
        assert r.returncode == 0
        want = []
        for obj in rules:
            row = []
            for k in fields:
                v = obj.get(k)
                if k.endswith(("bytes", "saved")):
                    row.append(str(v if v is not None else 0))
                else:
                    row.append((v or "").encode("utf-8").hex())
            want.append("\t".join(row) + "\t")
        assert r.stdout.splitlines() == want, (case, text)
    for bad in ['[{"source_asm": "A"}', '[{"bytes_saved": 1e3}]', '[{"source_asm": "\\x"}]', '{}', '[1]',
                '[{"source_asm": "a\x01"}]', '[] x', '[{"cycles_saved": 99999999999}]']:
        f = tmp_path / "bad.json"
        f.write_bytes(bad.encode())
        r = subprocess.run([str(exe), str(f)], capture_output=True, text=True, timeout=60)
        assert r.stdout.strip() == "ERROR", bad
