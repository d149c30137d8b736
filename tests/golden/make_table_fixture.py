"""Extracts the reference's per-opcode tables from its Go source, mechanically.

    python tests/golden/make_table_fixture.py REFERENCE_ROOT

REFERENCE_ROOT is a checkout of oisee/z80-optimizer.  Parsed, with no table
typed in by hand:

  pkg/inst/instruction.go  the OpCode enum (iota order), HasImmediate and
                           HasImm16 (their case lists)
  pkg/inst/catalog.go      Catalog: every struct-literal table and the loop
                           that files it (prefix bytes, T-states), the
                           single Catalog[...] = Info{...} lines, and the
                           BIT/RES/SET loops (evaluated: encoding base |
                           bit << 3 | register code, mnemonic text)
  pkg/search/verifier.go   opReads (case lists -> returned regMask)
  pkg/search/pruner.go     opWrites (case lists -> returned regMask)

Writes tests/golden/reference_tables.json: for each of the 455 opcodes its
name, mnemonic, encoding bytes (without immediate), T-states, byte size
(ByteSize: encoding + 1 or 2 immediate bytes), immediate kind and the
register names opReads / opWrites return.  The parser refuses anything it
does not recognise, and every opcode must be filed exactly once.
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def strip_comments(src):
    return re.sub(r"//[^\n]*", "", src)


def func_body(src, header):
    i = src.index(header)
    j = src.index("{", i)
    depth, k = 0, j
    while True:
        if src[k] == "{":
            depth += 1
        elif src[k] == "}":
            depth -= 1
            if depth == 0:
                return src[j + 1:k]
        k += 1


def parse_enum(src):
    src = strip_comments(src)
    m = re.search(r"const \(\s*(\w+) OpCode = iota(.*?)\n\)", src, re.S)
    names = [m.group(1)] + re.findall(r"^\s*(\w+)\s*$", m.group(2), re.M)
    assert names[-1] == "OpCodeCount", names[-1]
    return names[:-1]


def parse_switch(body, value):
    """case lists of a `switch op {` whose cases each `return <expr>`;
    returns {name: value(expr)}."""
    body = strip_comments(body)
    sw = body[body.index("switch op {"):]
    parts = re.split(r"\bcase\b", sw)[1:]
    out = {}
    for p in parts:
        head, _, rest = p.partition(":")
        stmt = rest.strip()
        m = re.match(r"return ([^\n]+)", stmt)
        assert m, f"unexpected case body: {stmt[:80]!r}"
        tail = stmt[m.end():].strip()
        assert tail in ("", "}") or tail.startswith("}"), f"extra statements after return: {tail[:80]!r}"
        v = value(m.group(1).strip())
        for name in re.findall(r"(?:inst\.)?(\w+)", head):
            assert name not in out, f"{name} filed twice"
            out[name] = v
    return out


REGS = ["A", "F", "B", "C", "D", "E", "H", "L", "SP", "M"]  # regMask bit order, verifier.go:177-189


def regmask(expr):
    if expr == "0":
        return []
    names = [x.strip() for x in expr.split("|")]
    for n in names:
        assert n.startswith("reg") and n[3:] in REGS, f"unexpected term {n!r}"
    return sorted({n[3:] for n in names}, key=REGS.index)


def parse_catalog(src):
    src = strip_comments(src)
    body = func_body(src, "func init()")
    cat = {}

    def put(name, mnem, enc, t):
        assert name not in cat, f"{name} filed twice"
        cat[name] = {"mnemonic": mnem, "bytes": enc, "tstates": t}

    def ints(s):
        return [int(x, 0) for x in re.findall(r"0x[0-9A-Fa-f]+|\d+", s)]

    # struct-literal tables and the loops that file them
    tables = {}
    for m in re.finditer(r"(\w+) := \[\]struct \{[^}]*\}\{(.*?)\n\t\}", body, re.S):
        tables[m.group(1)] = re.findall(r"\{(\w+), \"([^\"]*)\", (0x[0-9A-Fa-f]+)\}", m.group(2))
        assert tables[m.group(1)], m.group(1)
    loops = re.findall(r"for _, (\w+) := range (\w+) \{\s*Catalog\[\1\.op\] = Info\{Mnemonic: \1\.mnemonic, "
                       r"Bytes: \[\]uint8\{([^}]*)\}, TStates: (\d+)\}\s*\}", body)
    assert sorted(t for _, t, _, _ in loops) == sorted(tables), (sorted(tables), loops)
    for var, tname, byts, t in loops:
        prefix = [int(x, 0) for x in re.findall(r"0x[0-9A-Fa-f]+", byts)]
        assert byts.replace(" ", "").endswith(f"{var}.enc"), byts
        for name, mnem, enc in tables[tname]:
            put(name, mnem, prefix + [int(enc, 0)], int(t))
    # single lines
    for name, mnem, byts, t in re.findall(r"Catalog\[(\w+)\] = Info\{\"([^\"]*)\", \[\]uint8\{([^}]*)\}, (\d+)\}",
                                          body):
        put(name, mnem, ints(byts), int(t))
    # BIT/RES/SET n, r loops over the [7][8] opcode arrays
    reg_enc = ints(re.search(r"regEnc := \[7\]uint8\{([^}]*)\}", body).group(1))
    reg_names = re.findall(r"\"(\w)\"", re.search(r"regNames := \[7\]string\{([^}]*)\}", body).group(1))
    arrays = {}
    for m in re.finditer(r"(\w+) := \[7\]\[8\]OpCode\{(.*?)\n\t\}", body, re.S):
        rows = re.findall(r"\{([^}]*)\}", m.group(2))
        arrays[m.group(1)] = [re.findall(r"\w+", r) for r in rows]
        assert len(arrays[m.group(1)]) == 7 and all(len(r) == 8 for r in arrays[m.group(1)])
    pat2 = (r"for ri := 0; ri < 7; ri\+\+ \{\s*for bit := 0; bit < 8; bit\+\+ \{\s*"
            r"enc := (0x[0-9A-Fa-f]+) \| uint8\(bit<<3\) \| regEnc\[ri\]\s*"
            r"Catalog\[(\w+)\[ri\]\[bit\]\] = Info\{\s*Mnemonic: \"(\w+) \" \+ string\('0'\+byte\(bit\)\) \+ \", \" "
            r"\+ regNames\[ri\],\s*Bytes:\s*\[\]uint8\{(0x[0-9A-Fa-f]+), enc\},\s*TStates:\s*(\d+),")
    n2 = 0
    for base, arr, kind, pre, t in re.findall(pat2, body):
        n2 += 1
        for ri in range(7):
            for bit in range(8):
                enc = int(base, 0) | (bit << 3) | reg_enc[ri]
                put(arrays[arr][ri][bit], f"{kind} {bit}, {reg_names[ri]}", [int(pre, 0), enc], int(t))
    assert n2 == len(arrays), (n2, sorted(arrays))
    # BIT/RES/SET n, (HL) loops over consecutive opcodes
    pat1 = (r"for bit := 0; bit < 8; bit\+\+ \{\s*op := (\w+) \+ OpCode\(bit\)\s*"
            r"enc := (0x[0-9A-Fa-f]+) \| uint8\(bit<<3\)\s*Catalog\[op\] = Info\{\s*"
            r"Mnemonic: \"(\w+) \" \+ string\('0'\+byte\(bit\)\) \+ \", \(HL\)\",\s*"
            r"Bytes:\s*\[\]uint8\{(0x[0-9A-Fa-f]+), enc\},\s*TStates:\s*(\d+),")
    hli = re.findall(pat1, body)
    assert len(hli) == len(re.findall(r"for bit := 0; bit < 8; bit\+\+ \{\s*op :=", body))
    return cat, hli


def main():
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    ref = sys.argv[1]
    rd = lambda p: open(os.path.join(ref, p)).read()  # noqa: E731
    isrc = rd("pkg/inst/instruction.go")
    names = parse_enum(isrc)
    assert len(names) == 455, len(names)
    code = {n: i for i, n in enumerate(names)}
    has_imm = parse_switch(func_body(strip_comments(isrc), "func HasImmediate(op OpCode) bool"),
                           lambda e: e == "true")
    has_imm16 = parse_switch(func_body(strip_comments(isrc), "func HasImm16(op OpCode) bool"),
                             lambda e: e == "true")
    cat, hli = parse_catalog(rd("pkg/inst/catalog.go"))
    for first, base, kind, pre, t in hli:
        for bit in range(8):
            name = names[code[first] + bit]
            assert name not in cat
            cat[name] = {"mnemonic": f"{kind} {bit}, (HL)", "bytes": [int(pre, 0), int(base, 0) | (bit << 3)],
                         "tstates": int(t)}
    assert sorted(cat) == sorted(names), set(names) ^ set(cat)
    reads = parse_switch(func_body(strip_comments(rd("pkg/search/verifier.go")), "func opReads(op inst.OpCode)"),
                         regmask)
    writes = parse_switch(func_body(strip_comments(rd("pkg/search/pruner.go")), "func opWrites(op inst.OpCode)"),
                          regmask)
    for d in (reads, writes, has_imm, has_imm16):
        assert set(d) <= set(names), set(d) - set(names)
    ops = []
    for i, n in enumerate(names):
        imm16 = has_imm16.get(n, False)
        imm = imm16 or has_imm.get(n, False)
        c = cat[n]
        ops.append({"op": i, "name": n, "mnemonic": c["mnemonic"], "bytes": c["bytes"], "tstates": c["tstates"],
                    "size": len(c["bytes"]) + (2 if imm16 else 1 if imm else 0),
                    "imm": 16 if imm16 else 8 if imm else 0,
                    "reads": reads.get(n, []), "writes": writes.get(n, [])})
    out = {"source": "pkg/inst/instruction.go (enum, HasImmediate, HasImm16), pkg/inst/catalog.go (Catalog), "
                     "pkg/search/verifier.go (opReads), pkg/search/pruner.go (opWrites); extracted by "
                     "tests/golden/make_table_fixture.py",
           "reg_bits": REGS, "ops": ops}
    with open(os.path.join(HERE, "reference_tables.json"), "w") as f:
        f.write('{"source": %s,\n "reg_bits": %s,\n "ops": [\n' % (json.dumps(out["source"]),
                                                                 json.dumps(out["reg_bits"])))
        f.write(",\n".join("  " + json.dumps(o) for o in ops))
        f.write("\n]}\n")
    print(f"{len(ops)} opcodes; opReads filed {len(reads)}, opWrites filed {len(writes)}")


if __name__ == "__main__":
    main()
