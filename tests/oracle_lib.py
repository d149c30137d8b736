"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle (oracle/*.cpp) restates the reference's pkg/inst, pkg/cpu and
pkg/search behaviour; tests use it as the checker for the CUDA path.
"""
import ctypes
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "_build", "liboracle.so")


class OrcState(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint8) for n in "AFBCDEHL"] + [
        ("SP", ctypes.c_uint16), ("M", ctypes.c_uint8), ("pad", ctypes.c_uint8)]

    def tup(self):
        return (self.A, self.F, self.B, self.C, self.D, self.E, self.H, self.L, self.SP, self.M)


class OrcRule(ctypes.Structure):
    _fields_ = [("src", ctypes.c_uint32 * 4), ("rep", ctypes.c_uint32 * 4),
                ("src_len", ctypes.c_int32), ("rep_len", ctypes.c_int32),
                ("bytes_saved", ctypes.c_int32), ("cycles_saved", ctypes.c_int32),
                ("dead_flags", ctypes.c_int32), ("target_index", ctypes.c_int32),
                ("dead_regs", ctypes.c_int32)]

    def key(self):
        return (self.target_index, tuple(self.src[:self.src_len]), tuple(self.rep[:self.rep_len]),
                self.bytes_saved, self.cycles_saved, self.dead_flags)

    def key_regs(self):
        return self.key() + (self.dead_regs,)


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = ctypes.CDLL(ORACLE_SO)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        L.orc_exhaustive_states.restype = ctypes.c_ulonglong
        L.orc_search.restype = ctypes.c_longlong
        L.orc_search.argtypes = [u32p, ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_int, ctypes.POINTER(OrcRule),
                                 ctypes.c_longlong, ctypes.POINTER(ctypes.c_ulonglong)]
        L.orc_search_ext.restype = ctypes.c_longlong
        L.orc_search_ext.argtypes = [u32p, ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_uint8), ctypes.c_int,
                                     ctypes.POINTER(OrcRule), ctypes.c_longlong,
                                     ctypes.POINTER(ctypes.c_ulonglong)]
        L.orc_search_timed.restype = ctypes.c_longlong
        L.orc_search_timed.argtypes = [u32p, ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int, ctypes.POINTER(OrcRule),
                                       ctypes.c_longlong, ctypes.POINTER(ctypes.c_ulonglong),
                                       ctypes.POINTER(ctypes.c_double), ctypes.c_double]
        L.orc_enumerate_pool.restype = ctypes.c_longlong
        L.orc_enumerate_pool.argtypes = [u32p, ctypes.c_int, ctypes.c_int, u32p, ctypes.c_longlong]
        L.orc_search_gpu.restype = ctypes.c_longlong
        L.orc_search_gpu.argtypes = [u32p, ctypes.POINTER(ctypes.c_int), ctypes.c_int, u32p,
                                     ctypes.c_int, ctypes.c_int, ctypes.POINTER(OrcRule),
                                     ctypes.c_longlong]
        L.orc_mul_op_name.restype = ctypes.c_char_p
        L.orc_init()
        _lib = L
    return _lib


def pack(op, imm=0):
    return (op & 0xFFFF) | ((imm & 0xFFFF) << 16)


def arr(seq):
    return (ctypes.c_uint32 * max(1, len(seq)))(*seq)


def op_count():
    return lib().orc_op_count()


def op_name(op):
    b = ctypes.create_string_buffer(32)
    lib().orc_op_name(op, b, 32)
    return b.value.decode()


OPS = None


def ops():
    """name -> opcode"""
    global OPS
    if OPS is None:
        OPS = {op_name(i): i for i in range(op_count())}
    return OPS


def catalog(op):
    m = ctypes.create_string_buffer(64)
    enc = (ctypes.c_uint8 * 4)()
    n, t, b = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    lib().orc_catalog(op, m, 64, enc, ctypes.byref(n), ctypes.byref(t), ctypes.byref(b))
    return m.value.decode(), bytes(enc[:n.value]), t.value, b.value


def state(**kw):
    s = OrcState()
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def exec1(st, op, imm=0):
    t = lib().orc_exec(ctypes.byref(st), op, imm)
    return t


def exec_seq(st, seq):
    out = OrcState()
    lib().orc_exec_seq(ctypes.byref(st), arr(seq), len(seq), ctypes.byref(out))
    return out


def disasm(seq):
    b = ctypes.create_string_buffer(256)
    lib().orc_disasm_seq(arr(seq), len(seq), b, 256)
    return b.value.decode()


def quickcheck(t, c, dead=0):
    return bool(lib().orc_quickcheck(arr(t), len(t), arr(c), len(c), dead))


def midcheck(t, c, dead=0):
    return bool(lib().orc_midcheck(arr(t), len(t), arr(c), len(c), dead))


def exhaustive(t, c, dead=0):
    return bool(lib().orc_exhaustive(arr(t), len(t), arr(c), len(c), dead))


def exhaustive_regs(t, c, dead=0, dregs=0):
    """ExhaustiveCheckMasked with the dead-register extension."""
    return bool(lib().orc_exhaustive_regs(arr(t), len(t), arr(c), len(c), dead, dregs))


def exhaustive_states(t, c):
    return int(lib().orc_exhaustive_states(arr(t), len(t), arr(c), len(c)))


def flagdiff(t, c):
    return lib().orc_flagdiff(arr(t), len(t), arr(c), len(c))


def fingerprint(seq):
    out = (ctypes.c_uint8 * 80)()
    lib().orc_fingerprint(arr(seq), len(seq), out)
    return bytes(out)


def should_prune(seq):
    return bool(lib().orc_should_prune(arr(seq), len(seq)))


def op_reads(op):
    return lib().orc_op_reads(op)


def op_writes(op):
    return lib().orc_op_writes(op)


def instructions8():
    buf = (ctypes.c_uint32 * 8192)()
    n = lib().orc_instructions8(buf, 8192)
    return list(buf[:n])


def test_vectors():
    qc = (OrcState * 8)()
    mid = (OrcState * 32)()
    lib().orc_test_vectors(qc, mid)
    return [s.tup() for s in qc], [s.tup() for s in mid]


def _targets(targets):
    n = len(targets)
    flat = (ctypes.c_uint32 * max(1, 4 * n))()
    lens = (ctypes.c_int * max(1, n))()
    for i, t in enumerate(targets):
        lens[i] = len(t)
        for j, w in enumerate(t):
            flat[4 * i + j] = w
    return flat, lens


def search(targets, max_cand_len, dead=0, workers=0, cap=None):
    """worker.go semantics over a target list; returns (rules, checked)."""
    flat, lens = _targets(targets)
    cap = cap or (2 * len(targets) + 16)
    out = (OrcRule * cap)()
    checked = ctypes.c_ulonglong()
    w = workers or os.cpu_count() or 1
    n = lib().orc_search(flat, lens, len(targets), max_cand_len, dead, w, out, cap,
                         ctypes.byref(checked))
    assert n >= 0, "rule buffer too small"
    return [out[i] for i in range(n)], checked.value


def search_ext(targets, max_cand_len, dead=None, dregs=None, workers=0, cap=None):
    """worker.go semantics with per-target dead flags and dead registers
    (extension); returns (rules, checked)."""
    flat, lens = _targets(targets)
    cap = cap or (2 * len(targets) + 16)
    out = (OrcRule * cap)()
    checked = ctypes.c_ulonglong()
    w = workers or os.cpu_count() or 1
    d = (ctypes.c_uint8 * len(targets))(*dead) if dead is not None else None
    r = (ctypes.c_uint8 * len(targets))(*dregs) if dregs is not None else None
    n = lib().orc_search_ext(flat, lens, len(targets), max_cand_len, d, r, w, out, cap, ctypes.byref(checked))
    assert n >= 0, "rule buffer too small"
    return [out[i] for i in range(n)], checked.value


def search_gpu_semantics(targets, candidates, dead=0, cap=None):
    flat, lens = _targets(targets)
    cap = cap or (64 * len(targets) + 16)
    out = (OrcRule * cap)()
    cands = arr(candidates)
    n = lib().orc_search_gpu(flat, lens, len(targets), cands, len(candidates), dead, out, cap)
    assert n >= 0, "rule buffer too small"
    return [out[i] for i in range(n)]


def write_json(rules):
    n = len(rules)
    a = (OrcRule * max(1, n))(*rules)
    need = lib().orc_write_json(a, n, None, 0)
    b = ctypes.create_string_buffer(need + 1)
    lib().orc_write_json(a, n, b, need + 1)
    return b.value.decode()


def dead_flag_desc(mask):
    b = ctypes.create_string_buffer(64)
    lib().orc_dead_flag_desc(mask, b, 64)
    return b.value.decode()


def parse_dead_flags(s):
    v = ctypes.c_int()
    ok = lib().orc_parse_dead_flags(s.encode(), ctypes.byref(v))
    return v.value if ok else None


def parse_assembly(text):
    buf = (ctypes.c_uint32 * 64)()
    n = lib().orc_parse_assembly(text.encode(), buf, 64)
    return None if n < 0 else list(buf[:n])


def mul_find(k, min_len, max_len, b, c, f):
    ln, t = ctypes.c_int(), ctypes.c_int()
    ops_ = (ctypes.c_int * 16)()
    ok = lib().orc_mul_find(k, min_len, max_len, b, c, f, ctypes.byref(ln), ctypes.byref(t), ops_)
    if not ok:
        return None
    return ln.value, t.value, list(ops_[:ln.value])


def mul_run(seq, x, b, c, f):
    a = (ctypes.c_int * max(1, len(seq)))(*seq)
    return lib().orc_mul_run(a, len(seq), x, b, c, f)


def mul_tstates(i):
    return lib().orc_mul_tstates(i)


MUL_POOL_REFERENCE, MUL_POOL_WIDE, MUL_POOL_FAST, MUL_POOL_CUDA = 0, 1, 2, 3


def mul_pool_size(pool):
    return lib().orc_mul_pool_size(pool)


def mul_find_pool(pool, k, min_len, max_len, b=0, c=0, f=0):
    """(length, tstates, ops) of cmd/mulopt findOptimal over `pool`, or None."""
    ln, t = ctypes.c_int(), ctypes.c_int()
    ops_ = (ctypes.c_int * 16)()
    ok = lib().orc_mul_find_pool(pool, k, min_len, max_len, b, c, f, ctypes.byref(ln), ctypes.byref(t), ops_)
    if not ok:
        return None
    return ln.value, t.value, list(ops_[:ln.value])


def mul_run_pool(pool, seq, x, b=0, c=0, f=0):
    a = (ctypes.c_int * max(1, len(seq)))(*seq)
    return lib().orc_mul_run_pool(pool, a, len(seq), x, b, c, f)


def mul_tstates_pool(pool, i):
    return lib().orc_mul_tstates_pool(pool, i)


def mul_op_name(pool, i):
    return lib().orc_mul_op_name(pool, i).decode()


def qc_survivors(target, dead=0):
    buf = (ctypes.c_uint32 * 8192)()
    n = lib().orc_qc_survivors(arr(target), len(target), dead, buf, 8192)
    return list(buf[:n])


def search_timed(targets, max_cand_len, dead=0, workers=0, cap=None, target_budget=0.0):
    """search() that also returns each target's worker-thread CPU seconds:
    (rules, checked, secs list).  With target_budget > 0, a target whose
    sweeps run past that many CPU seconds is abandoned: secs = -1, and its
    rules and checked count are left out."""
    flat, lens = _targets(targets)
    cap = cap or (2 * len(targets) + 16)
    out = (OrcRule * cap)()
    checked = ctypes.c_ulonglong()
    secs = (ctypes.c_double * max(1, len(targets)))()
    w = workers or os.cpu_count() or 1
    n = lib().orc_search_timed(flat, lens, len(targets), max_cand_len, dead, w, out, cap,
                               ctypes.byref(checked), secs, float(target_budget))
    assert n >= 0, "rule buffer too small"
    return [out[i] for i in range(n)], checked.value, list(secs[:len(targets)])


def enumerate_pool(pool, length):
    """Unpruned sequences of `length` over `pool` in EnumerateSequences8
    order, as a numpy uint32 array [n, length]."""
    import numpy as np
    p = arr(pool)
    n = lib().orc_enumerate_pool(p, len(pool), length, None, 0)
    out = np.zeros((n, length), dtype=np.uint32)
    lib().orc_enumerate_pool(p, len(pool), length, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), n)
    return out


_C2 = None


def c2_targets():
    """Every unpruned length-2 sequence over the 8-bit instruction list."""
    global _C2
    if _C2 is None:
        _C2 = enumerate_pool(instructions8(), 2)
    return _C2


def c2_subset(k, seed=0):
    """k C2 targets drawn without replacement by index with numpy's seeded
    generator, in index order (the same draw as the workload generator)."""
    import numpy as np
    allt = c2_targets()
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(len(allt), size=min(k, len(allt)), replace=False))
    return allt[idx]


def splitmix64(seed):
    """The splitmix64 stream (Steele, Lea, Flood 2014)."""
    m = (1 << 64) - 1
    x = seed & m
    while True:
        x = (x + 0x9E3779B97F4A7C15) & m
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
        yield z ^ (z >> 31)


def c1_pool(seed=0):
    """The small plain pool: register LD/ALU/INC/DEC, accumulator and CB
    rotates/shifts on registers, SCF/CCF/CPL/NEG, and the immediate forms
    with imm8 in {00,01,7F,80,FF} plus three bytes of splitmix64(seed), in
    opcode order (immediate forms after the others)."""
    o = ops()
    regs = "ABCDEHL"
    names = []
    for d in regs:
        names += [f"LD_{d}_{s}" for s in ("BCDEHLA" if d == "A" else regs)]
    for pre in ["ADD_A_", "ADC_A_", "SUB_", "SBC_A_", "AND_", "XOR_", "OR_", "CP_"]:
        names += [pre + s for s in "BCDEHLA"]
    names += [f"INC_{r}" for r in regs] + [f"DEC_{r}" for r in regs]
    names += ["RLCA", "RRCA", "RLA", "RRA"]
    for k in ["RLC", "RRC", "RL", "RR", "SLA", "SRA", "SRL", "SLL"]:
        names += [f"{k}_{r}" for r in regs]
    names += ["SCF", "CCF", "CPL", "NEG"]
    non_imm = sorted(o[n] for n in names)
    imm_ops = sorted(o[n] for n in [f"LD_{d}_N" for d in regs] +
                     ["ADD_A_N", "ADC_A_N", "SUB_N", "SBC_A_N", "AND_N", "XOR_N", "OR_N", "CP_N"])
    g = splitmix64(seed)
    imms = [0x00, 0x01, 0x7F, 0x80, 0xFF] + [next(g) & 0xFF for _ in range(3)]
    return [pack(op) for op in non_imm] + [pack(op, v) for op in imm_ops for v in imms]


def c1_targets(seed=0):
    return enumerate_pool(c1_pool(seed), 2)


def eligible_checks(targets):
    """QuickCheck units of a target array (numpy uint32 [n, L]): for each
    target, the 8-bit instructions with a shorter encoding than the target
    that ShouldPrune keeps."""
    import numpy as np
    sizes = np.array([catalog(op)[3] for op in range(op_count())], dtype=np.int64)
    pool = np.array(instructions8(), dtype=np.uint32)
    psize = sizes[pool & 0xFFFF]
    prune = np.array([should_prune([int(w)]) for w in pool])
    tb = sizes[(targets & 0xFFFF)].sum(axis=1)
    counts = np.array([np.count_nonzero((psize < b) & ~prune) for b in range(0, 16)], dtype=np.int64)
    return int(counts[tb].sum())

