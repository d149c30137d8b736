"""The per-opcode tables of the oracle and of the library against the
reference's own Go source.

tests/golden/reference_tables.json is extracted mechanically from the
reference (make_table_fixture.py parses the OpCode enum and HasImmediate /
HasImm16 of pkg/inst/instruction.go, the Catalog of pkg/inst/catalog.go:147-562,
opReads of pkg/search/verifier.go:199-408 and opWrites of
pkg/search/pruner.go:66-236).  Every one of the 455 opcodes is compared field
by field: name, mnemonic, encoding, T-states, byte size, immediate kind and
the read / write register masks that pruning and the sweep shapes depend on.
"""
import json
import os

import pytest

import workloads
import z80b

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def ref():
    d = json.load(open(os.path.join(HERE, "golden", "reference_tables.json")))
    assert len(d["ops"]) == 455
    return d


def _mask(names, bits):
    m = 0
    for n in names:
        m |= 1 << bits.index(n)
    return m


def test_fixture_register_bits_match_library(ref):
    # regMask bit order of verifier.go:177-189; the library's masks use the same bits
    assert ref["reg_bits"] == ["A", "F", "B", "C", "D", "E", "H", "L", "SP", "M"]


def test_oracle_tables_equal_reference(ref, O):
    bits = ref["reg_bits"]
    for e in ref["ops"]:
        op = e["op"]
        assert O.op_name(op) == e["name"]
        mnem, enc, t, size = O.catalog(op)
        assert (mnem, list(enc), t, size) == (e["mnemonic"], e["bytes"], e["tstates"], e["size"]), e["name"]
        assert O.op_reads(op) == _mask(e["reads"], bits), e["name"]
        assert O.op_writes(op) == _mask(e["writes"], bits), e["name"]
        assert bool(O.lib().orc_has_imm(op)) == (e["imm"] != 0), e["name"]
        assert bool(O.lib().orc_has_imm16(op)) == (e["imm"] == 16), e["name"]


def test_library_tables_equal_reference(ref):
    bits = ref["reg_bits"]
    names = workloads.ops()
    for e in ref["ops"]:
        op = e["op"]
        assert names[e["name"]] == op
        info = z80b.op_info(op)
        assert info["mnemonic"] == e["mnemonic"], e["name"]
        assert (info["size"], info["tstates"]) == (e["size"], e["tstates"]), e["name"]
        assert info["imm"] == {0: 0, 8: 1, 16: 2}[e["imm"]], e["name"]
        assert info["reads"] == _mask(e["reads"], bits), e["name"]
        assert info["writes"] == _mask(e["writes"], bits), e["name"]


def test_pool8_follows_reference_immediates(ref):
    # EnumerateSequences8 (enumerator.go:319-345): non-immediate opcodes, then
    # the imm8 opcodes x 256; imm16 opcodes are not in the 8-bit list
    non = [e["op"] for e in ref["ops"] if e["imm"] == 0]
    imm8 = [e["op"] for e in ref["ops"] if e["imm"] == 8]
    want = [z80b.pack(op) for op in non] + [z80b.pack(op, v) for op in imm8 for v in range(256)]
    assert z80b.pool8() == want
    assert len(want) == 4531
