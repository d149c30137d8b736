"""Seeded synthetic workloads of the benchmark configurations.

C1  small plain: targets = every unpruned length-2 sequence over a reduced
    8-bit pool (register LD/ALU/INC/DEC, accumulator and CB rotates/shifts on
    registers, SCF/CCF/CPL/NEG, and the immediate forms with imm8 in
    {00,01,7F,80,FF} plus three bytes from splitmix64(seed 0)); candidates
    are the reference's length-1 enumeration (4,531 instructions).
C2  full length-2: every unpruned length-2 sequence over the reference's
    8-bit instruction list (9,818,041 targets); subsets are drawn by index
    with a seeded generator.
C3  batched uneven: unpruned targets drawn instruction by instruction from
    the 8-bit list (60% length 2, 40% length 3), each with a dead-register
    mask over B,C,D,E,H,L and a dead-flag mask over the six documented flags
    S,Z,H,P/V,N,C; candidates up to 2 instructions.
The reference publishes no benchmark dataset for this path; these
generators are the inputs of the parity tests and of bench.py.
"""
import ctypes

import numpy as np

import z80b

MASK64 = (1 << 64) - 1


def splitmix64(seed):
    """Yields the splitmix64 stream (Steele, Lea, Flood 2014)."""
    x = seed & MASK64
    while True:
        x = (x + 0x9E3779B97F4A7C15) & MASK64
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        yield z ^ (z >> 31)


_OPS = None


def ops():
    """opcode name -> number, from the library's catalog."""
    global _OPS
    if _OPS is None:
        names = {}
        regs = "ABCDEHL"
        # derive names from mnemonics is ambiguous; build the enum order the
        # same way the reference lists it (pkg/inst/instruction.go:50-595)
        order = []
        for d in regs:
            srcs = "BCDEHLA" if d == "A" else regs
            order += [f"LD_{d}_{s}" for s in srcs]
        order += [f"LD_{d}_N" for d in regs]
        for pre in ["ADD_A_", "ADC_A_", "SUB_", "SBC_A_", "AND_", "XOR_", "OR_", "CP_"]:
            order += [pre + s for s in "BCDEHLAN"]
        order += [f"INC_{r}" for r in regs] + [f"DEC_{r}" for r in regs]
        order += ["RLCA", "RRCA", "RLA", "RRA", "DAA", "CPL", "SCF", "CCF", "NEG", "NOP"]
        for k in ["RLC", "RRC", "RL", "RR", "SLA", "SRA", "SRL"]:
            order += [f"{k}_{r}" for r in regs]
        order += ["SLL_A"] + [f"SLL_{r}" for r in regs[1:]]
        for k in ["BIT", "RES", "SET"]:
            for n in range(8):
                order += [f"{k}_{n}_{r}" for r in regs]
        order += ["INC_BC", "INC_DE", "INC_HL", "INC_SP", "DEC_BC", "DEC_DE", "DEC_HL", "DEC_SP",
                  "ADD_HL_BC", "ADD_HL_DE", "ADD_HL_HL", "ADD_HL_SP", "EX_DE_HL", "LD_SP_HL",
                  "LD_BC_NN", "LD_DE_NN", "LD_HL_NN", "LD_SP_NN",
                  "ADC_HL_BC", "ADC_HL_DE", "ADC_HL_HL", "ADC_HL_SP",
                  "SBC_HL_BC", "SBC_HL_DE", "SBC_HL_HL", "SBC_HL_SP"]
        order += [f"LD_{r}_HLI" for r in regs] + [f"LD_HLI_{r}" for r in regs]
        order += ["LD_HLI_N", "LD_A_BCI", "LD_A_DEI", "LD_BCI_A", "LD_DEI_A",
                  "ADD_A_HLI", "ADC_A_HLI", "SUB_HLI", "SBC_A_HLI", "AND_HLI", "XOR_HLI", "OR_HLI",
                  "CP_HLI", "INC_HLI", "DEC_HLI",
                  "RLC_HLI", "RRC_HLI", "RL_HLI", "RR_HLI", "SLA_HLI", "SRA_HLI", "SRL_HLI", "SLL_HLI"]
        for k in ["BIT", "RES", "SET"]:
            order += [f"{k}_{n}_HLI" for n in range(8)]
        assert len(order) == 455
        names = {n: i for i, n in enumerate(order)}
        _OPS = names
    return _OPS


def c1_imm8(seed=0):
    g = splitmix64(seed)
    return [0x00, 0x01, 0x7F, 0x80, 0xFF] + [next(g) & 0xFF for _ in range(3)]


def c1_pool(seed=0):
    """The C1 instruction pool, in opcode order (immediate forms x imm8 set)."""
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
    imms = c1_imm8(seed)
    return [z80b.pack(op) for op in non_imm] + [z80b.pack(op, v) for op in imm_ops for v in imms]


def enumerate_targets(pool, length):
    """Unpruned sequences of `length` over `pool` in odometer order (numpy uint32 [n, length])."""
    L = z80b.lib()
    L.z80b_enumerate.restype = ctypes.c_uint64
    L.z80b_enumerate.argtypes = [ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint32, ctypes.c_uint32,
                                 ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint64]
    p = (ctypes.c_uint32 * len(pool))(*pool)
    n = L.z80b_enumerate(p, len(pool), length, None, 0)
    out = np.zeros((n, length), dtype=np.uint32)
    L.z80b_enumerate(p, len(pool), length, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), n)
    return out


def c1_targets(seed=0):
    return enumerate_targets(c1_pool(seed), 2)


_C2 = None


def c2_targets():
    global _C2
    if _C2 is None:
        _C2 = enumerate_targets(z80b.pool8(), 2)
    return _C2


def c2_subset(k, seed=0):
    """k targets of C2 drawn without replacement by index (seeded), in index order."""
    allt = c2_targets()
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(len(allt), size=min(k, len(allt)), replace=False))
    return allt[idx]


def to_lists(arr):
    return [list(map(int, row)) for row in arr]


def shard_bounds(n, rank, world):
    """Contiguous shard [lo, hi) of n independent targets for one rank (the
    reference splits its outer target loop the same way across processes)."""
    return n * rank // world, n * (rank + 1) // world


def mul_init(seed=2):
    """Initial B, C, F of the constant-multiply workload: the low bytes of the
    first three splitmix64 outputs of `seed`."""
    g = splitmix64(seed)
    return next(g) & 0xFF, next(g) & 0xFF, next(g) & 0xFF


DOC_FLAGS = (0x80, 0x40, 0x10, 0x04, 0x02, 0x01)  # S, Z, H, P/V, N, C


def prune_mask(arr, lens):
    """ShouldPrune of every row of arr (uint32 [n, stride]) with lengths lens."""
    L = z80b.lib()
    arr = np.ascontiguousarray(arr, dtype=np.uint32)
    lens = np.ascontiguousarray(lens, dtype=np.uint8)
    out = np.zeros(len(arr), dtype=np.uint8)
    st = L.z80b_should_prune_batch(arr.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                   lens.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), arr.shape[1], len(arr),
                                   out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
    assert st == 0 and not (out == 0xFF).any()
    return out.astype(bool)


def c3_targets(n, seed=1):
    """n C3 targets: (targets uint32 [n, 4], lens uint8 [n], dead_flags uint8 [n],
    dead_regs uint8 [n]).  Length 2 with probability 0.6, else 3; every
    instruction uniform over the 4,531-entry 8-bit list; pruned draws are
    redrawn; masks uniform over their 64 subsets."""
    pool = np.array(z80b.pool8(), dtype=np.uint32)
    rng = np.random.default_rng(seed)
    out = np.zeros((n, 4), dtype=np.uint32)
    lens = np.where(rng.random(n) < 0.6, 2, 3).astype(np.uint8)
    todo = np.arange(n)
    while len(todo):
        out[todo, :3] = pool[rng.integers(0, len(pool), size=(len(todo), 3))]
        out[todo[lens[todo] == 2], 2] = 0
        bad = prune_mask(out[todo], lens[todo])
        todo = todo[bad]
    bits = rng.integers(0, 64, size=n)
    dead = np.zeros(n, dtype=np.uint8)
    for i, f in enumerate(DOC_FLAGS):
        dead |= np.where((bits >> i) & 1, f, 0).astype(np.uint8)
    dregs = rng.integers(0, 64, size=n).astype(np.uint8)
    return out, lens, dead, dregs
