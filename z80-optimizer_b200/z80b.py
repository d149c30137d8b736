"""Python binding of libz80b200.so (the sm_100a candidate-verification path).

Mirrors the reference's host interface for this path:
  * ``Context.load_candidates`` / ``Context.quickcheck_gpu`` --
    gpu.NewCUDAProcess / CUDAProcess.QuickCheckGPU (pkg/gpu/cuda.go:32-107)
  * ``Context.fingerprints`` -- search.Fingerprint (pkg/search/verifier.go:134)
  * ``Context.verify_pairs`` -- QuickCheck / MidCheck / ExhaustiveCheck
    [Masked] and FlagDiff over pairs (pkg/search/verifier.go)
  * ``Context.search`` -- search.Run worker semantics (mode "first",
    pkg/search/worker.go:124-265) or gpu.SearchGPU semantics (mode "all",
    pkg/gpu/search.go:80-199) over a batch of targets
  * ``search_single`` / ``search_single_masked`` -- search.SearchSingle[Masked]
    (pkg/search/search.go:82-110)
  * ``write_json`` -- result.WriteJSON (pkg/result/output.go:70-90)

Errors raise ``Z80BError`` with the library's status and message; the module
never falls back to a CPU implementation.  Instructions are packed as
``op | imm << 16`` (pkg/gpu/cuda.go:310).
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libz80b200.so")

OK, EINVAL, ENOMEM, ECUDA, ETIMEOUT, ECAPACITY, ENODEV, ESTATE = range(8)
MODE_FIRST, MODE_ALL = 0, 1
PATH_BATCHED, PATH_PLAIN = 0, 1
TIER_QC, TIER_MID, TIER_EXH = 1, 2, 4
DEAD_NONE, DEAD_UNDOC, DEAD_ALL = 0x00, 0x28, 0xFF


class Z80BError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"z80b status {status}: {msg}")
        self.status = status


class State(ctypes.Structure):
    """cpu.State (pkg/cpu/state.go:11-15)."""
    _fields_ = [(n, ctypes.c_uint8) for n in "afbcdehl"] + [
        ("sp", ctypes.c_uint16), ("m", ctypes.c_uint8), ("pad", ctypes.c_uint8)]

    def tup(self):
        return (self.a, self.f, self.b, self.c, self.d, self.e, self.h, self.l, self.sp, self.m)


class Rule(ctypes.Structure):
    """result.Rule (pkg/result/table.go:11-17) + target index."""
    _fields_ = [("src", ctypes.c_uint32 * 4), ("rep", ctypes.c_uint32 * 4),
                ("src_len", ctypes.c_int32), ("rep_len", ctypes.c_int32),
                ("bytes_saved", ctypes.c_int32), ("cycles_saved", ctypes.c_int32),
                ("dead_flags", ctypes.c_int32), ("target_index", ctypes.c_int32),
                ("dead_regs", ctypes.c_int32), ("reserved", ctypes.c_int32)]

    @property
    def source(self):
        return list(self.src[:self.src_len])

    @property
    def replacement(self):
        return list(self.rep[:self.rep_len])

    def key(self):
        return (self.target_index, tuple(self.source), tuple(self.replacement),
                self.bytes_saved, self.cycles_saved, self.dead_flags, self.dead_regs)


class Stats(ctypes.Structure):
    _fields_ = [("targets", ctypes.c_uint64), ("checks", ctypes.c_uint64),
                ("checked_ref", ctypes.c_uint64), ("qc_survivors", ctypes.c_uint64),
                ("mid_survivors", ctypes.c_uint64), ("exhaustive_pairs", ctypes.c_uint64),
                ("exhaustive_states", ctypes.c_uint64), ("rules", ctypes.c_uint64),
                ("rounds", ctypes.c_uint32), ("launches", ctypes.c_uint32),
                ("device_ms", ctypes.c_double), ("qc_ms", ctypes.c_double),
                ("exh_ms", ctypes.c_double), ("exhaustive_evaluated", ctypes.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Job(ctypes.Structure):
    _fields_ = [("targets", ctypes.POINTER(ctypes.c_uint32)),
                ("target_lens", ctypes.POINTER(ctypes.c_uint8)),
                ("dead_flags", ctypes.POINTER(ctypes.c_uint8)),
                ("dead_regs", ctypes.POINTER(ctypes.c_uint8)),
                ("n_targets", ctypes.c_uint32), ("target_len", ctypes.c_uint32),
                ("target_stride", ctypes.c_uint32), ("max_cand_len", ctypes.c_uint32),
                ("global_dead_flags", ctypes.c_uint32), ("mode", ctypes.c_uint32),
                ("path", ctypes.c_uint32), ("flags", ctypes.c_uint32)]


_lib = None
EXPORTS = [
    "z80b_init", "z80b_destroy", "z80b_last_error", "z80b_status_string", "z80b_version",
    "z80b_fingerprints", "z80b_exec", "z80b_load_candidates", "z80b_quickcheck",
    "z80b_verify_pairs", "z80b_search", "z80b_stage_job", "z80b_run_staged", "z80b_fetch_rules",
    "z80b_op_info", "z80b_disasm_seq", "z80b_parse_assembly", "z80b_parse_dead_flags",
    "z80b_dead_flag_desc", "z80b_should_prune", "z80b_pool8", "z80b_rules_json",
    "z80b_set_option", "z80b_get_option", "z80b_autotune", "z80b_enumerate",
    "z80b_mul_pool", "z80b_mul_search", "z80b_should_prune_batch",
    "z80b_server_start", "z80b_server_submit", "z80b_server_poll", "z80b_server_get_stats", "z80b_server_stop",
    "z80b_search_cb",
]
RULE_CB = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint32)
OPT_EXH_LANE_STATES, OPT_EXH_CHUNK_BLOCKS, OPT_STREAM_PRIORITY, OPT_QC_INDEX, OPT_XINDEP_BITS = 1, 2, 3, 4, 5
OPT_COMPACT_SWEEP = 6
OPT_GRAPH_ROUNDS = 7
OPT_WIDE_SWEEP = 8
OPT_CONCURRENT_SWEEPS = 9
OPT_QC_SINGLE_PASS = 10
JOB_NO_EXHAUSTIVE = 1
ANSWER_TRUNCATED = 1


MULPOOL_MULOPT, MULPOOL_WIDE21, MULPOOL_FAST14, MULPOOL_CUDA21 = 0, 1, 2, 3


class MulResult(ctypes.Structure):
    """MulResult (cmd/mulopt/main.go:162-167) with pool indices for ops."""
    _fields_ = [("k", ctypes.c_int32), ("found", ctypes.c_int32), ("length", ctypes.c_int32),
                ("tstates", ctypes.c_int32), ("ops", ctypes.c_uint8 * 16), ("index", ctypes.c_uint64)]


class MulStats(ctypes.Structure):
    _fields_ = [("sequences", ctypes.c_uint64), ("per_k_sequences", ctypes.c_uint64),
                ("filter_nodes", ctypes.c_uint64), ("full_checks", ctypes.c_uint64),
                ("full_pass", ctypes.c_uint64), ("lengths", ctypes.c_int32),
                ("launches", ctypes.c_int32), ("device_ms", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Query(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint64), ("target", ctypes.c_uint32 * 4), ("len", ctypes.c_uint8),
                ("dead_flags", ctypes.c_uint8), ("dead_regs", ctypes.c_uint8), ("reserved", ctypes.c_uint8)]


class Answer(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint64), ("status", ctypes.c_int32), ("n_rules", ctypes.c_int32),
                ("rules", Rule * 2), ("queued_ms", ctypes.c_double), ("service_ms", ctypes.c_double),
                ("latency_ms", ctypes.c_double), ("batch_size", ctypes.c_uint32), ("flags", ctypes.c_uint32)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("workers", ctypes.c_int), ("max_batch", ctypes.c_uint32),
                ("memory_budget", ctypes.c_uint64), ("max_cand_len", ctypes.c_uint32)]


class ServerStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_uint64) for k in ("submitted", "answered", "errors", "batches", "max_batch_seen",
                                               "pending", "inflight_bytes")] + [("device_ms", ctypes.c_double),
                                                                                 ("peak_inflight_bytes", ctypes.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TuneTrial(ctypes.Structure):
    _fields_ = [("xindep_bits", ctypes.c_int), ("lane_states", ctypes.c_int), ("chunk_blocks", ctypes.c_int),
                ("compact", ctypes.c_int), ("ms", ctypes.c_double), ("kernels", ctypes.c_char * 96)]

    def as_dict(self):
        return {"xindep_bits": self.xindep_bits, "lane_states": self.lane_states,
                "chunk_blocks": self.chunk_blocks, "compact": self.compact, "ms": self.ms,
                "kernels": self.kernels.decode()}


TUNE_MAX_TRIALS = 64


class TuneResult(ctypes.Structure):
    _fields_ = [("lane_states", ctypes.c_int), ("chunk_blocks", ctypes.c_int), ("xindep_bits", ctypes.c_int),
                ("compact", ctypes.c_int), ("n_trials", ctypes.c_int), ("trials", TuneTrial * TUNE_MAX_TRIALS)]

    def trial_list(self):
        return [self.trials[i].as_dict() for i in range(self.n_trials)]


def lib():
    """Loads libz80b200.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise Z80BError(ENODEV, f"{LIB_PATH} not built (run make in {_HERE})")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        u32p = ctypes.POINTER(ctypes.c_uint32)
        u8p = ctypes.POINTER(ctypes.c_uint8)
        L.z80b_init.argtypes = [ctypes.c_int, ctypes.POINTER(vp)]
        L.z80b_destroy.argtypes = [vp]
        L.z80b_destroy.restype = None
        L.z80b_last_error.argtypes = [vp]
        L.z80b_last_error.restype = ctypes.c_char_p
        L.z80b_status_string.restype = ctypes.c_char_p
        L.z80b_fingerprints.argtypes = [vp, u32p, ctypes.c_uint32, ctypes.c_uint32, u8p]
        L.z80b_exec.argtypes = [vp, ctypes.POINTER(State), u32p, u8p, ctypes.c_uint32,
                                ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(State)]
        L.z80b_load_candidates.argtypes = [vp, u32p, ctypes.c_uint32, ctypes.c_uint32]
        L.z80b_quickcheck.argtypes = [vp, u8p, ctypes.c_uint32, u32p, ctypes.c_uint32, u32p]
        L.z80b_verify_pairs.argtypes = [vp, u32p, u8p, u32p, u8p, ctypes.c_uint32, ctypes.c_uint32,
                                        u8p, ctypes.c_uint32, u8p, u8p]
        L.z80b_search.argtypes = [vp, ctypes.POINTER(Job), ctypes.POINTER(Rule), ctypes.c_uint64,
                                  ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(Stats)]
        L.z80b_stage_job.argtypes = [vp, ctypes.POINTER(Job)]
        L.z80b_run_staged.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(Stats)]
        L.z80b_fetch_rules.argtypes = [vp, ctypes.POINTER(Rule), ctypes.c_uint64,
                                       ctypes.POINTER(ctypes.c_uint64)]
        L.z80b_op_info.argtypes = [ctypes.c_uint32, ctypes.c_char_p, ctypes.c_uint32] + \
            [ctypes.POINTER(ctypes.c_int)] * 5
        L.z80b_disasm_seq.argtypes = [u32p, ctypes.c_uint32, ctypes.c_char_p, ctypes.c_uint32]
        L.z80b_parse_assembly.argtypes = [ctypes.c_char_p, u32p, ctypes.c_uint32]
        L.z80b_parse_dead_flags.argtypes = [ctypes.c_char_p, u32p]
        L.z80b_dead_flag_desc.argtypes = [ctypes.c_uint32, ctypes.c_char_p, ctypes.c_uint32]
        L.z80b_should_prune.argtypes = [u32p, ctypes.c_uint32]
        L.z80b_pool8.argtypes = [u32p, ctypes.c_uint32]
        L.z80b_pool8.restype = ctypes.c_uint32
        L.z80b_rules_json.argtypes = [ctypes.POINTER(Rule), ctypes.c_uint64, ctypes.c_char_p,
                                      ctypes.c_uint64]
        L.z80b_rules_json.restype = ctypes.c_longlong
        L.z80b_set_option.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.z80b_get_option.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.z80b_autotune.argtypes = [vp, ctypes.POINTER(Job), ctypes.POINTER(TuneResult)]
        L.z80b_enumerate.restype = ctypes.c_uint64
        L.z80b_enumerate.argtypes = [u32p, ctypes.c_uint32, ctypes.c_uint32, u32p, ctypes.c_uint64]
        L.z80b_should_prune_batch.argtypes = [u32p, u8p, ctypes.c_uint32, ctypes.c_uint64, u8p]
        L.z80b_search_cb.argtypes = [vp, ctypes.POINTER(Job), ctypes.POINTER(Rule), ctypes.c_uint64,
                                     ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(Stats), RULE_CB, vp]
        L.z80b_server_start.argtypes = [ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]
        L.z80b_server_submit.argtypes = [vp, ctypes.POINTER(Query), ctypes.c_uint32]
        L.z80b_server_poll.argtypes = [vp, ctypes.POINTER(Answer), ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32),
                                       ctypes.c_int]
        L.z80b_server_get_stats.argtypes = [vp, ctypes.POINTER(ServerStats)]
        L.z80b_server_stop.argtypes = [vp]
        ip = ctypes.POINTER(ctypes.c_int)
        L.z80b_mul_pool.argtypes = [ctypes.c_int, ip, ip, ctypes.POINTER(ctypes.c_char_p), ip, ctypes.c_int]
        L.z80b_mul_search.argtypes = [vp, ctypes.c_int, ctypes.c_uint8, ctypes.c_uint8, ctypes.c_uint8,
                                      ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int32),
                                      ctypes.c_uint32, ctypes.POINTER(MulResult), ctypes.POINTER(MulStats)]
        _lib = L
    return _lib


def pack(op, imm=0):
    return (op & 0xFFFF) | ((imm & 0xFFFF) << 16)


def _u32(seq):
    return (ctypes.c_uint32 * max(1, len(seq)))(*seq)


def _u8(seq):
    return (ctypes.c_uint8 * max(1, len(seq)))(*seq)


# ------------------------------------------------------------ host helpers

def op_info(op):
    m = ctypes.create_string_buffer(32)
    vals = [ctypes.c_int() for _ in range(5)]
    st = lib().z80b_op_info(op, m, 32, *[ctypes.byref(v) for v in vals])
    if st != OK:
        raise Z80BError(st, f"opcode {op}")
    size, t, imm, rd, wr = (v.value for v in vals)
    return {"mnemonic": m.value.decode(), "size": size, "tstates": t, "imm": imm,
            "reads": rd, "writes": wr}


def disasm(seq):
    n = lib().z80b_disasm_seq(_u32(seq), len(seq), None, 0)
    if n < 0:
        raise Z80BError(EINVAL, "bad opcode")
    b = ctypes.create_string_buffer(n + 1)
    lib().z80b_disasm_seq(_u32(seq), len(seq), b, n + 1)
    return b.value.decode()


def parse_assembly(text):
    buf = (ctypes.c_uint32 * 256)()
    n = lib().z80b_parse_assembly(text.encode(), buf, 256)
    if n < 0:
        raise Z80BError(EINVAL, f"cannot parse {text!r}")
    return list(buf[:n])


def parse_dead_flags(text):
    v = ctypes.c_uint32()
    st = lib().z80b_parse_dead_flags(text.encode(), ctypes.byref(v))
    if st != OK:
        raise Z80BError(st, f"invalid --dead-flags value {text!r}")
    return v.value


def dead_flag_desc(mask):
    b = ctypes.create_string_buffer(64)
    lib().z80b_dead_flag_desc(mask, b, 64)
    return b.value.decode()


def should_prune(seq):
    r = lib().z80b_should_prune(_u32(seq), len(seq))
    if r < 0:
        raise Z80BError(EINVAL, "bad opcode")
    return bool(r)


def pool8():
    buf = (ctypes.c_uint32 * 8192)()
    n = lib().z80b_pool8(buf, 8192)
    return list(buf[:n])


def write_json(rules):
    arr = (Rule * max(1, len(rules)))(*rules)
    n = lib().z80b_rules_json(arr, len(rules), None, 0)
    if n < 0:
        raise Z80BError(EINVAL, "bad rule")
    b = ctypes.create_string_buffer(n + 1)
    lib().z80b_rules_json(arr, len(rules), b, n + 1)
    return b.value.decode()


# ----------------------------------------------------------------- context

class Context:
    """One device context (z80b_init).  Not thread-safe; one per thread."""

    def __init__(self, device=0):
        self._h = ctypes.c_void_p()
        st = lib().z80b_init(device, ctypes.byref(self._h))
        if st != OK:
            raise Z80BError(st, lib().z80b_status_string(st).decode())

    def close(self):
        if self._h:
            lib().z80b_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != OK:
            raise Z80BError(st, lib().z80b_last_error(self._h).decode())

    # search.Fingerprint
    def fingerprints(self, seqs, length):
        flat = [w for s in seqs for w in s]
        out = (ctypes.c_uint8 * (80 * max(1, len(seqs))))()
        self._check(lib().z80b_fingerprints(self._h, _u32(flat), len(seqs), length, out))
        return [bytes(out[80 * i:80 * i + 80]) for i in range(len(seqs))]

    def exec(self, states, seqs, stride=4):
        n = len(seqs)
        flat = []
        lens = []
        for s in seqs:
            flat += list(s) + [0] * (stride - len(s))
            lens.append(len(s))
        ins = (State * max(1, n))(*states)
        outs = (State * max(1, n))()
        self._check(lib().z80b_exec(self._h, ins, _u32(flat), _u8(lens), 0, stride, n, outs))
        return [outs[i] for i in range(n)]

    # gpu.NewCUDAProcess
    def load_candidates(self, cands, seq_len=1):
        flat = [w for c in cands for w in (c if isinstance(c, (list, tuple)) else [c])]
        n = len(flat) // seq_len
        self._check(lib().z80b_load_candidates(self._h, _u32(flat), n, seq_len))

    # CUDAProcess.QuickCheckGPU
    def quickcheck_gpu(self, fp, dead_flags=0, cap=1 << 20):
        hits = (ctypes.c_uint32 * cap)()
        nh = ctypes.c_uint32()
        fpb = (ctypes.c_uint8 * 80)(*fp)
        self._check(lib().z80b_quickcheck(self._h, fpb, dead_flags, hits, cap, ctypes.byref(nh)))
        return list(hits[:nh.value])

    def verify_pairs(self, pairs, dead=None, tiers=TIER_QC | TIER_MID | TIER_EXH, stride=4):
        """pairs: [(target_seq, cand_seq)]; returns [(tier_bits, flagdiff)]."""
        n = len(pairs)
        t, c, tl, cl = [], [], [], []
        for a, b in pairs:
            t += list(a) + [0] * (stride - len(a))
            c += list(b) + [0] * (stride - len(b))
            tl.append(len(a))
            cl.append(len(b))
        out = (ctypes.c_uint8 * max(1, n))()
        fd = (ctypes.c_uint8 * max(1, n))()
        dd = _u8(dead) if dead is not None else None
        self._check(lib().z80b_verify_pairs(self._h, _u32(t), _u8(tl), _u32(c), _u8(cl), stride, n,
                                            dd, tiers, out, fd))
        return [(out[i], fd[i]) for i in range(n)]

    @staticmethod
    def make_job(targets, dead_flags=0, mode=MODE_FIRST, path=PATH_BATCHED, per_target_dead=None,
                 dead_regs=None, stride=4, max_cand_len=1, no_exhaustive=False):
        """Builds a Job plus the ctypes buffers it points to."""
        n = len(targets)
        stride = max([stride] + [len(t) for t in targets])
        flat = (ctypes.c_uint32 * max(1, n * stride))()
        lens = (ctypes.c_uint8 * max(1, n))()
        for i, t in enumerate(targets):
            lens[i] = len(t)
            for j, w in enumerate(t):
                flat[i * stride + j] = w
        job = Job()
        job.targets = ctypes.cast(flat, ctypes.POINTER(ctypes.c_uint32))
        job.target_lens = ctypes.cast(lens, ctypes.POINTER(ctypes.c_uint8))
        keep = [flat, lens]
        if per_target_dead is not None:
            d = _u8(per_target_dead)
            keep.append(d)
            job.dead_flags = ctypes.cast(d, ctypes.POINTER(ctypes.c_uint8))
        if dead_regs is not None:
            r = _u8(dead_regs)
            keep.append(r)
            job.dead_regs = ctypes.cast(r, ctypes.POINTER(ctypes.c_uint8))
        job.n_targets = n
        job.target_len = 0
        job.target_stride = stride
        job.max_cand_len = max_cand_len
        job.global_dead_flags = dead_flags
        job.mode = mode
        job.path = path
        job.flags = JOB_NO_EXHAUSTIVE if no_exhaustive else 0
        return job, keep

    def search(self, targets, dead_flags=0, mode=MODE_FIRST, path=PATH_BATCHED,
               per_target_dead=None, dead_regs=None, max_cand_len=1, no_exhaustive=False):
        job, keep = self.make_job(targets, dead_flags, mode, path, per_target_dead, dead_regs,
                                  max_cand_len=max_cand_len, no_exhaustive=no_exhaustive)
        return self.run_job(job)

    def run_job(self, job, cap=None):
        cap = cap or (2 * job.n_targets + 1024)
        while True:
            out = (Rule * cap)()
            nr = ctypes.c_uint64()
            st = Stats()
            s = lib().z80b_search(self._h, ctypes.byref(job), out, cap, ctypes.byref(nr),
                                  ctypes.byref(st))
            if s == ECAPACITY and nr.value > cap:
                cap = nr.value
                continue
            self._check(s)
            return [out[i] for i in range(nr.value)], st

    def search_streaming(self, targets, per_target_dead=None, dead_regs=None, max_cand_len=1):
        """z80b_search_cb: returns (rules, stats, events) where events lists
        (target_index, [rule keys]) in the order the callback delivered them."""
        job, keep = self.make_job(targets, 0, MODE_FIRST, PATH_BATCHED, per_target_dead, dead_regs,
                                  max_cand_len=max_cand_len)
        events = []

        def cb(user, t, rules, n):
            rs = ctypes.cast(rules, ctypes.POINTER(Rule))
            events.append((t, [rs[i].key() for i in range(n)]))

        fn = RULE_CB(cb)
        cap = 2 * len(targets) + 16
        out = (Rule * cap)()
        nr = ctypes.c_uint64()
        st = Stats()
        self._check(lib().z80b_search_cb(self._h, ctypes.byref(job), out, cap, ctypes.byref(nr), ctypes.byref(st),
                                         fn, None))
        return [out[i] for i in range(nr.value)], st, events

    def set_option(self, option, value):
        self._check(lib().z80b_set_option(self._h, option, value))

    def get_option(self, option):
        v = ctypes.c_int()
        self._check(lib().z80b_get_option(self._h, option, ctypes.byref(v)))
        return v.value

    def autotune(self, job):
        """Tries every (lane states, chunk size) on a sample job; keeps the fastest."""
        r = TuneResult()
        self._check(lib().z80b_autotune(self._h, ctypes.byref(job), ctypes.byref(r)))
        return r

    def mul_search(self, pool, init=(0, 0, 0), min_len=1, max_len=8, ks=None):
        """cmd/mulopt findOptimal for the constants ks (default 2..255) at once.
        Returns ([{k, found, length, tstates, ops, index}], MulStats)."""
        kl = list(range(2, 256)) if ks is None else list(ks)
        karr = (ctypes.c_int32 * max(1, len(kl)))(*kl)
        out = (MulResult * max(1, len(kl)))()
        st = MulStats()
        b, c, f = init
        self._check(lib().z80b_mul_search(self._h, pool, b, c, f, min_len, max_len,
                                          None if ks is None else karr, len(kl), out, ctypes.byref(st)))
        res = [{"k": out[i].k, "found": bool(out[i].found), "length": out[i].length,
                "tstates": out[i].tstates, "ops": list(out[i].ops[:out[i].length]),
                "index": out[i].index} for i in range(len(kl))]
        return res, st

    def stage(self, job):
        self._check(lib().z80b_stage_job(self._h, ctypes.byref(job)))

    def run_staged(self):
        nr = ctypes.c_uint64()
        st = Stats()
        self._check(lib().z80b_run_staged(self._h, ctypes.byref(nr), ctypes.byref(st)))
        return nr.value, st

    def fetch_rules(self, n):
        out = (Rule * max(1, n))()
        nr = ctypes.c_uint64()
        self._check(lib().z80b_fetch_rules(self._h, out, max(1, n), ctypes.byref(nr)))
        return [out[i] for i in range(nr.value)]


def mul_pool(pool):
    """(names, tstates, max_len) of a constant-multiply pool."""
    n, ml = ctypes.c_int(), ctypes.c_int()
    names = (ctypes.c_char_p * 32)()
    ts = (ctypes.c_int * 32)()
    st = lib().z80b_mul_pool(pool, ctypes.byref(n), ctypes.byref(ml), names, ts, 32)
    if st != OK:
        raise Z80BError(st, f"unknown pool {pool}")
    return [names[i].decode() for i in range(n.value)], list(ts[:n.value]), ml.value


def mul_results_json(results, pool):
    """cmd/mulopt -json output (main.go:336-350): the found results as a JSON
    array of {k, ops, length, tstates}, two-space indent."""
    import json
    names = mul_pool(pool)[0]
    out = [{"k": r["k"], "ops": [names[i] for i in r["ops"]], "length": r["length"],
            "tstates": r["tstates"]} for r in results if r["found"]]
    return json.dumps(out, indent=2) + "\n"


class Server:
    """Serving loop (z80b_server_*): submit queries from any thread, poll answers."""

    def __init__(self, device=0, workers=4, max_batch=512, memory_budget=0, max_cand_len=2):
        cfg = ServerConfig(device, workers, max_batch, memory_budget, max_cand_len)
        h = ctypes.c_void_p()
        st = lib().z80b_server_start(ctypes.byref(cfg), ctypes.byref(h))
        if st != OK:
            raise Z80BError(st, "z80b_server_start failed")
        self._h = h

    def submit(self, queries):
        """queries: iterable of (id, target instruction list, dead_flags, dead_regs)."""
        qs = list(queries)
        arr = (Query * max(1, len(qs)))()
        for i, (qid, tgt, df, dr) in enumerate(qs):
            if not 1 <= len(tgt) <= 4:
                raise Z80BError(EINVAL, f"query {qid}: target length {len(tgt)} outside 1..4")
            arr[i].id = qid
            arr[i].len = len(tgt)
            for k, w in enumerate(tgt):
                arr[i].target[k] = w
            arr[i].dead_flags = df
            arr[i].dead_regs = dr
        st = lib().z80b_server_submit(self._h, arr, len(qs))
        if st != OK:
            raise Z80BError(st, "z80b_server_submit failed")

    def poll(self, cap=4096, timeout_ms=10):
        out = (Answer * cap)()
        n = ctypes.c_uint32()
        st = lib().z80b_server_poll(self._h, out, cap, ctypes.byref(n), timeout_ms)
        if st != OK:
            raise Z80BError(st, "z80b_server_poll failed")
        return [out[i] for i in range(n.value)]

    def stats(self):
        s = ServerStats()
        lib().z80b_server_get_stats(self._h, ctypes.byref(s))
        return s

    def stop(self):
        if self._h:
            lib().z80b_server_stop(self._h)
            self._h = None


def _sort_rules(rules):
    # result.Table.Rules (pkg/result/table.go:38-50): bytes saved, then cycles
    # saved, both descending; insertion order breaks ties (full rule first)
    return sorted(rules, key=lambda r: (-r.bytes_saved, -r.cycles_saved))


def search_single(ctx, target, max_cand_len=1):
    """search.SearchSingle (pkg/search/search.go:82-94)."""
    rules, _ = ctx.search([target], max_cand_len=max_cand_len)
    rules = _sort_rules(rules)
    return rules[0] if rules else None


def search_single_masked(ctx, target, max_cand_len, dead_flags):
    """search.SearchSingleMasked (pkg/search/search.go:97-110)."""
    rules, _ = ctx.search([target], dead_flags=dead_flags, max_cand_len=max_cand_len)
    rules = _sort_rules(rules)
    return rules[0] if rules else None
