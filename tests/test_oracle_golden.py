"""Pins the CPU oracle to the reference's own known answers and golden data.

Cases come from tests/golden/reference_known_answers.json (transcribed from
the reference's Go tests, each citing file:line) and
tests/golden/peephole_top500_pairs.json (the reference's data file).
"""
import json
import os

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
KA = json.load(open(os.path.join(HERE, "golden", "reference_known_answers.json")))
FLAG = {"C": 0x01, "N": 0x02, "P": 0x04, "V": 0x04, "X3": 0x08, "H": 0x10, "X5": 0x20, "Z": 0x40, "S": 0x80}


def seq(O, items):
    o = O.ops()
    return [O.pack(o[n], v) for n, v in items]


@pytest.mark.parametrize("case", KA["exec"], ids=lambda c: c["src"] + ":" + c["op"])
def test_exec_known_answers(O, case):
    st = O.state(**case["state"])
    O.exec1(st, O.ops()[case["op"]], case.get("imm", 0))
    exp = case["expect"]
    for k in "ABCDEHL":
        if k in exp:
            assert getattr(st, k) == exp[k], (k, getattr(st, k), exp[k])
    if "SP" in exp:
        assert st.SP == exp["SP"]
    if "F" in exp:
        assert st.F == exp["F"]
    for f in exp.get("F_has", []):
        assert st.F & FLAG[f], (f, hex(st.F))
    for f in exp.get("F_not", []):
        assert not st.F & FLAG[f], (f, hex(st.F))


def test_exec_sweeps(O):
    o = O.ops()
    # exec_test.go:319-343 ADD exhaustive; :466-477 CP keeps A
    for a in range(256):
        for v in range(256):
            s = O.state(A=a)
            O.exec1(s, o["ADD_A_N"], v)
            assert s.A == (a + v) & 0xFF and bool(s.F & 1) == (a + v > 0xFF) and not s.F & 2
            s = O.state(A=a)
            O.exec1(s, o["CP_N"], v)
            assert s.A == a
    # :479-500 XOR A with all flags set
    for a in range(256):
        s = O.state(A=a, F=0xFF)
        O.exec1(s, o["XOR_A"])
        assert s.A == 0 and s.F & 0x40 and not s.F & 0x13
    # :502-516 RRA preserves S, Z, P
    for f0 in (0xC4, 0x00, 0x80, 0x44):
        s = O.state(A=1, F=f0)
        O.exec1(s, o["RRA"])
        assert s.F & 0xC4 == f0 & 0xC4
    # :532-549 LD r,n
    for v in range(256):
        s = O.state()
        O.exec1(s, o["LD_A_N"], v)
        assert s.A == v
        s = O.state()
        O.exec1(s, o["LD_B_N"], v)
        assert s.B == v
    # :1155-1199 ADC/SBC HL cross-check
    for hl in range(0, 0x10000, 0x1111):
        for rr in range(0, 0x10000, 0x1111):
            for c in (0, 1):
                s = O.state(H=hl >> 8, L=hl & 0xFF, B=rr >> 8, C=rr & 0xFF, F=c)
                O.exec1(s, o["ADC_HL_BC"])
                assert not s.F & 2 and (s.H << 8 | s.L) == (hl + rr + c) & 0xFFFF
                s = O.state(H=hl >> 8, L=hl & 0xFF, D=rr >> 8, E=rr & 0xFF, F=c)
                O.exec1(s, o["SBC_HL_DE"])
                assert s.F & 2 and (s.H << 8 | s.L) == (hl - rr - c) & 0xFFFF


def test_all_opcodes_execute_deterministically(O):
    # exec_test.go:443-464 and 518-530
    for op in range(O.op_count()):
        a = O.state(A=0x42, F=0x01, B=0x13, C=0x24, D=0x35, E=0x46, H=0x57, L=0x68)
        b = O.state(A=0x42, F=0x01, B=0x13, C=0x24, D=0x35, E=0x46, H=0x57, L=0x68)
        O.exec1(a, op, 0x55)
        O.exec1(b, op, 0x55)
        assert a.tup() == b.tup()


def test_catalog(O):
    c = KA["catalog"]
    o = O.ops()
    assert O.op_count() == c["op_count"]
    for name, enc in c["encodings"].items():
        assert list(O.catalog(o[name])[1]) == enc, name
    for name, n in c["byte_size"].items():
        assert O.catalog(o[name])[3] == n
    for name, t in c["tstates"].items():
        assert O.catalog(o[name])[2] == t
    for name, imm, text in c["disassemble"]:
        assert O.disasm([O.pack(o[name], imm)]) == text
    for name in c["immediate"]:
        assert O.lib().orc_has_imm(o[name])
    for name in c["not_immediate"]:
        assert not O.lib().orc_has_imm(o[name])
    for op in range(O.op_count()):
        m, enc, t, b = O.catalog(op)
        assert m and enc and t > 0  # catalog_test.go:8-21
    items, total = c["seq_byte_size"]
    assert sum(O.catalog(o[n])[3] for n, _ in items) == total


def test_search_known(O):
    s = KA["search"]
    for case in s["single"]:
        rules, _ = O.search([seq(O, case["target"])], case["max_cand"])
        assert bool(rules) == case["expect_opt"], case["src"]
        if case["expect_opt"] and "bytes_saved" in case:
            assert rules[0].bytes_saved == case["bytes_saved"]
    for case in s["quickcheck"]:
        assert O.quickcheck(seq(O, case["t"]), seq(O, case["c"]), case["dead"]) == case["expect"], case["src"]
    for case in s["exhaustive"]:
        assert O.exhaustive(seq(O, case["t"]), seq(O, case["c"]), case["dead"]) == case["expect"], case["src"]
    for case in s["flagdiff"]:
        fd = O.flagdiff(seq(O, case["t"]), seq(O, case["c"]))
        if case.get("expect_nonzero"):
            assert fd != 0
        else:
            assert fd == case["expect"]
    for case in s["prune"]:
        assert O.should_prune(seq(O, case["seq"])) == case["expect"], case["src"]
    assert len(O.instructions8()) == s["instruction_count"]["eight_bit"]


def test_states_equal_masked_via_quickcheck(O):
    # verifier_test.go:444-468 truth table, exercised through SCF-free
    # sequences: LD A,0 vs XOR A differ in F only; masks decide
    o = O.ops()
    t = [O.pack(o["LD_A_N"], 0)]
    c = [O.pack(o["XOR_A"])]
    assert not O.quickcheck(t, c, 0x00)
    assert O.quickcheck(t, c, 0xFF)
    assert not O.quickcheck(t, c, 0x28)


def test_peephole_top500_reverify(O):
    # data/peephole_top500.json: every rule the reference's CUDA search
    # reported must pass the oracle's ExhaustiveCheck (the reference's
    # verify-jsonl step, cmd/z80opt/main.go:399-476)
    pairs = json.load(open(os.path.join(HERE, "golden", "peephole_top500_pairs.json")))["pairs"]
    bad = []
    for p in pairs:
        s = O.parse_assembly(p["source"])
        r = O.parse_assembly(p["replacement"])
        assert s is not None and r is not None, p
        if not O.exhaustive(s, r):
            bad.append(p)
        def size(q):
            return sum(O.catalog(w & 0xFFFF)[3] for w in q)
        assert size(s) - size(r) == p["bytes_saved"], p
    assert not bad, bad[:5]


def test_write_json_format(O):
    o = O.ops()
    rules, _ = O.search([[O.pack(o["AND_N"], 0xFF)]], 1)
    text = O.write_json(rules)
    assert json.loads(text) == [{"source_asm": "AND 0FFh", "replacement_asm": "AND A",
                                 "source_bytes": 2, "replacement_bytes": 1,
                                 "bytes_saved": 1, "cycles_saved": 3}]
    assert text.startswith('[\n  {\n    "source_asm": "AND 0FFh",')
    assert O.write_json([]) == "[]\n"


def test_parse_helpers(O):
    assert O.parse_dead_flags("none") == 0 and O.parse_dead_flags("undoc") == 0x28
    assert O.parse_dead_flags("ALL") == 0xFF and O.parse_dead_flags("0x13") == 0x13
    assert O.parse_dead_flags("zz") is None and O.parse_dead_flags("0x100") is None
    assert O.dead_flag_desc(0x13) == "C,N,H" and O.dead_flag_desc(0x28) == "undoc"
    o = O.ops()
    assert O.parse_assembly("SUB A : LD A, 0") == [O.pack(o["SUB_A"]), O.pack(o["LD_A_N"], 0)]
    assert O.parse_assembly("and 0FFh") == [O.pack(o["AND_N"], 0xFF)]
    assert O.parse_assembly("FOO") is None
