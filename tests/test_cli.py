"""The z80opt command-line tool (cmd/z80opt + cmd/mulopt front end)."""
import json
import os
import subprocess

import pytest

from conftest import ROOT

EXE = os.path.join(ROOT, "z80-optimizer_b200", "_build", "z80opt")


def run(*args, timeout=600):
    return subprocess.run([EXE, *args], capture_output=True, text=True, timeout=timeout)


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_cli_usage():
    r = run()
    assert r.returncode == 2 and "usage: z80opt" in r.stderr


def test_cli_fails_loudly_without_device():
    if has_gpu():
        pytest.skip("a GPU is present")
    r = run("mulopt", "--k", "3")
    assert r.returncode == 1 and "no usable CUDA device" in r.stderr


def test_cli_rejects_bad_dead_flags():
    r = run("verify-jsonl", "/dev/null", "--dead-flags", "bogus")
    assert r.returncode == 1 and "invalid dead-flags" in r.stderr


@pytest.mark.gpu
def test_cli_mulopt_single(tmp_path):
    r = run("mulopt", "--k", "3", "--json")
    assert r.returncode == 0, r.stderr
    assert json.loads(r.stdout) == {"k": 3, "ops": ["LD B,A", "ADD A,A", "ADD A,B"], "length": 3, "tstates": 12}


@pytest.mark.gpu
def test_cli_verify_jsonl_top500(tmp_path):
    """The reference's 500 top peephole rules re-verify, one JSONL line each,
    plus a wrong rule, a malformed line and an unparsable one."""
    pairs = json.load(open(os.path.join(ROOT, "tests", "golden", "peephole_top500_pairs.json")))["pairs"]
    f = tmp_path / "rules.jsonl"
    with open(f, "w") as fh:
        for p in pairs:
            fh.write(json.dumps({"source_asm": p["source"], "replacement_asm": p["replacement"],
                                 "bytes_saved": p["bytes_saved"]}) + "\n")
        fh.write(json.dumps({"source_asm": "LD A, B : LD B, A", "replacement_asm": "LD B, A"}) + "\n")
        fh.write("{not json\n")
        fh.write(json.dumps({"source_asm": "FROB A", "replacement_asm": "NOP"}) + "\n")
    r = run("verify-jsonl", str(f))
    assert r.returncode == 1
    assert "Verification complete: 503 total, 500 passed, 1 failed, 2 skipped" in r.stdout
    assert "[501] FAIL: LD A, B : LD B, A -> LD B, A" in r.stdout


@pytest.mark.gpu
def test_cli_target_and_enumerate_sample(tmp_path):
    r = run("target", "LD A, B : LD B, A", "--max-candidate", "1")
    assert r.returncode == 0, r.stderr
    assert "Replacement: LD A, B (-1 bytes, -4 cycles)" in r.stdout
    out = tmp_path / "rules.json"
    r = run("enumerate", "--max-target", "2", "--sample", "2000", "--seed", "5", "--output", str(out))
    assert r.returncode == 0, r.stderr
    rules = json.load(open(out))
    assert rules and all(x["bytes_saved"] > 0 for x in rules)


def test_cli_mulopt_resume_all_presolved(tmp_path):
    """mulopt -resume (cmd/mulopt/main.go:238-302): constants in the resume
    file are not searched again; with all 254 there, no device is needed and
    the output is the file's results."""
    res = [{"k": k, "ops": ["ADD A,A"] * (k % 5 + 1), "length": k % 5 + 1, "tstates": 4 * (k % 5 + 1)}
           for k in range(2, 256)]
    f = tmp_path / "prev.json"
    f.write_text(json.dumps(res))
    r = run("mulopt", "-resume", str(f), "-json")
    assert r.returncode == 0, r.stderr
    assert json.loads(r.stdout) == res
    assert "Resumed 254 previous results" in r.stderr and "0 constants to check (254 pre-solved)" in r.stderr
    r = run("mulopt", "--resume", str(f))
    assert r.returncode == 0
    assert r.stdout.splitlines()[0] == "×  2: " + "[ADD A,A ADD A,A ADD A,A]".ljust(80) + " (3 insts, 12T)"
    bad = tmp_path / "bad.json"
    bad.write_text('[{"k": 300, "ops": []}]')
    r = run("mulopt", "--resume", str(bad))
    assert r.returncode == 1 and "Error parsing resume file" in r.stderr
    bad.write_text('{"k": 3')
    r = run("mulopt", "--resume", str(bad))
    assert r.returncode == 1 and "Error parsing resume file" in r.stderr


@pytest.mark.gpu
def test_cli_mulopt_resume_partial(tmp_path):
    """Resuming from the first ten constants of a run gives the same output
    as the run itself."""
    r = run("mulopt", "--max-len", "4", "--json")
    assert r.returncode == 0, r.stderr
    full = json.loads(r.stdout)
    f = tmp_path / "prev.json"
    f.write_text(json.dumps(full[:10]))
    r = run("mulopt", "--max-len", "4", "--json", "--resume", str(f))
    assert r.returncode == 0, r.stderr
    assert json.loads(r.stdout) == full
    assert "(10 pre-solved)" in r.stderr
