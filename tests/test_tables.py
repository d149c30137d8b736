"""Host-side tables of the product library (catalog, masks, pruning,
enumeration order, disassembly, parsing, JSON) against the CPU oracle."""
import json
import os
import random

import pytest

import z80b
import workloads
from conftest import ROOT


def test_op_info_matches_oracle(O):
    for op in range(455):
        info = z80b.op_info(op)
        m, enc, t, size = O.catalog(op)
        assert info["mnemonic"] == m
        assert info["size"] == size and info["tstates"] == t
        assert info["reads"] == O.op_reads(op), (op, O.op_name(op))
        assert info["writes"] == O.op_writes(op), (op, O.op_name(op))


def test_pool8_order_matches_enumerator(O):
    assert z80b.pool8() == O.instructions8()


def test_opcode_names(O):
    ops = workloads.ops()
    for name, op in ops.items():
        assert O.op_name(op) == name


def test_disasm_and_prune_random(O):
    rng = random.Random(7)
    pool = z80b.pool8()
    pool16 = pool + [z80b.pack(op, rng.randrange(65536)) for op in (382, 383, 384, 385) for _ in range(4)]
    for _ in range(20000):
        n = rng.randint(1, 3)
        seq = [rng.choice(pool16) for _ in range(n)]
        assert z80b.disasm(seq) == O.disasm(seq)
        assert z80b.should_prune(seq) == O.should_prune(seq), O.disasm(seq)


def test_prune_all_pairs_sample(O):
    pool = z80b.pool8()
    rng = random.Random(3)
    for _ in range(30000):
        seq = [rng.choice(pool), rng.choice(pool)]
        assert z80b.should_prune(seq) == O.should_prune(seq), O.disasm(seq)


def test_enumerate_counts():
    c2 = workloads.c2_targets()
    assert len(c2) == 9818041
    c1 = workloads.c1_targets()
    assert len(c1) > 0 and c1.shape[1] == 2


def test_parse_and_flags(O):
    for text in ["SUB A : LD A, 0", "AND 0FFh", "ld a, 0x00 : neg", "LD (HL), 12h", "BIT 7, (HL)",
                 "EX DE, HL", "ADC HL, SP", "SLL (HL)", "LD A, 0A5h : LD C, 255"]:
        assert z80b.parse_assembly(text) == O.parse_assembly(text), text
    # as in cmd/z80opt/main.go:348-395, a 16-bit immediate never parses (the
    # mnemonic's "nn" leaves an "N" in the prefix it matches against)
    for text in ["LD HL, 0C000h", "LD BC, 1234h", "LD SP, 0", "FROB A"]:
        assert O.parse_assembly(text) is None, text
        with pytest.raises(z80b.Z80BError):
            z80b.parse_assembly(text)
    for s in ["none", "undoc", "all", "0x13", "FF", "0x00"]:
        assert z80b.parse_dead_flags(s) == O.parse_dead_flags(s)
    for m in range(256):
        assert z80b.dead_flag_desc(m) == O.dead_flag_desc(m)


def test_rules_json_matches_oracle(O):
    o = O.ops()
    targets = [[O.pack(o["AND_N"], 0xFF)], [O.pack(o["SUB_A"]), O.pack(o["LD_A_N"], 0)],
               [O.pack(o["LD_A_N"], 0)]]
    rules, _ = O.search(targets, 1, dead=0xFF)
    mine = []
    for r in rules:
        x = z80b.Rule()
        x.src_len, x.rep_len = r.src_len, r.rep_len
        for i in range(r.src_len):
            x.src[i] = r.src[i]
        for i in range(r.rep_len):
            x.rep[i] = r.rep[i]
        x.bytes_saved, x.cycles_saved, x.dead_flags = r.bytes_saved, r.cycles_saved, r.dead_flags
        mine.append(x)
    assert z80b.write_json(mine) == O.write_json(rules)
    assert any(r.dead_flags for r in rules)
    json.loads(z80b.write_json(mine))


def test_a_dependence_classes_against_oracle(tmp_path):
    """The A-dependence class of every opcode (used to sweep A-independent
    pairs at two values of A) holds under the oracle's Exec, and two values
    of A decide random A-independent pairs exactly as all 256 do."""
    import subprocess
    exe = tmp_path / "aclass_check"
    srcs = [os.path.join(ROOT, "tests", "native", "aclass_check.cpp"),
            os.path.join(ROOT, "z80-optimizer_b200", "csrc", "z80_tables.cpp"),
            os.path.join(ROOT, "oracle", "z80_oracle_isa_cpu.cpp"),
            os.path.join(ROOT, "oracle", "z80_oracle_search.cpp")]
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe)] + srcs + ["-lpthread"], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("OK")


def test_register_renaming_against_oracle(tmp_path):
    """op_rename: for every opcode and permutation of B..L, the renamed
    opcode run on the permuted state gives the permuted result (oracle's
    Exec); instructions with only 8-bit register operands always rename."""
    import subprocess
    exe = tmp_path / "rename_check"
    srcs = [os.path.join(ROOT, "tests", "native", "rename_check.cpp"),
            os.path.join(ROOT, "z80-optimizer_b200", "csrc", "z80_tables.cpp"),
            os.path.join(ROOT, "oracle", "z80_oracle_isa_cpu.cpp"),
            os.path.join(ROOT, "oracle", "z80_oracle_search.cpp")]
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe)] + srcs + ["-lpthread"], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("OK")


def test_compact_state_mapping_against_oracle(tmp_path):
    """op_regs is sound (fields an instruction does not name never matter),
    and pairs that compact_map renames onto B, C keep the oracle's
    ExhaustiveCheck[Masked] verdict over the reference's whole sweep when only
    A, F, B and C are compared."""
    import subprocess
    exe = tmp_path / "compact_check"
    srcs = [os.path.join(ROOT, "tests", "native", "compact_check.cpp"),
            os.path.join(ROOT, "z80-optimizer_b200", "csrc", "z80_tables.cpp"),
            os.path.join(ROOT, "oracle", "z80_oracle_isa_cpu.cpp"),
            os.path.join(ROOT, "oracle", "z80_oracle_search.cpp")]
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe)] + srcs + ["-lpthread"], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("OK")


def test_wide_state_against_oracle(tmp_path):
    """The wide compact state (A, F, B, C, H, L, M): its step equals the full
    bit-sliced step on every opcode it holds, the device tables rename as
    wide_map does, and the wide sweep unit with its block decoding gives the
    oracle's ExhaustiveCheck verdict (dead flags and registers) for pairs
    the A/F/B/C state does not take, memory and reduced sweeps included."""
    import subprocess
    exe = tmp_path / "wide_check"
    srcs = [os.path.join(ROOT, "tests", "native", "wide_check.cpp"),
            os.path.join(ROOT, "z80-optimizer_b200", "csrc", "z80_tables.cpp"),
            os.path.join(ROOT, "oracle", "z80_oracle_isa_cpu.cpp"),
            os.path.join(ROOT, "oracle", "z80_oracle_search.cpp")]
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe)] + srcs + ["-lpthread"], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("OK")


def test_dependency_sets_against_oracle(tmp_path):
    """The dependency sets derived from the bit-sliced step hold under the
    oracle's Exec (an output never changes with an input outside its set),
    and sweeps that leave out the swept registers no compared output depends
    on give the oracle's ExhaustiveCheck verdicts with dead flags and
    registers."""
    import subprocess
    exe = tmp_path / "deps_check"
    srcs = [os.path.join(ROOT, "tests", "native", "deps_check.cpp"),
            os.path.join(ROOT, "z80-optimizer_b200", "csrc", "z80_tables.cpp"),
            os.path.join(ROOT, "oracle", "z80_oracle_isa_cpu.cpp"),
            os.path.join(ROOT, "oracle", "z80_oracle_search.cpp")]
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe)] + srcs + ["-lpthread"], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("OK")
