/* z80b200.h -- C ABI of libz80b200.so, the B200 (sm_100a) implementation of
 * the Z80 superoptimizer's candidate-verification path.
 *
 * Drop-in boundary: these entry points replace the child process
 * `cuda/z80qc --server` and its stdin/stdout protocol (pkg/gpu/cuda.go:32-113,
 * cuda/z80_quickcheck.cu:823-923) with in-process calls, and expose the whole
 * verification pipeline of pkg/search (QuickCheck -> [MidCheck] ->
 * ExhaustiveCheck, first-found or all-hits) for a batch of targets.
 *
 * Conventions
 *  - Instructions are packed as uint32 op | imm << 16, the packing of
 *    pkg/gpu/cuda.go:310 (op = the reference's OpCode enum, 0..454).
 *  - The caller owns every host buffer; the library copies in and out.  The
 *    library owns all device memory.
 *  - Every call returns a status (Z80B_OK = 0).  z80b_last_error() gives the
 *    message of the last failure on a context.
 *  - A context is bound to one device and is not thread-safe: use one
 *    context per host thread (queries of one context are serialized, as
 *    pkg/gpu/cuda.go:80 serializes queries with a mutex).
 */
#ifndef Z80B200_H_
#define Z80B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define Z80B_OK 0
#define Z80B_EINVAL 1     /* bad argument (null pointer, opcode > 454, length) */
#define Z80B_ENOMEM 2     /* device allocation failed */
#define Z80B_ECUDA 3      /* CUDA runtime error */
#define Z80B_ETIMEOUT 4   /* a bounded device wait ran out */
#define Z80B_ECAPACITY 5  /* caller's output buffer too small (count reported) */
#define Z80B_ENODEV 6     /* no CUDA device / wrong architecture */
#define Z80B_ESTATE 7     /* call order (e.g. quickcheck before load) */

#define Z80B_NUM_OPS 455
#define Z80B_FP_LEN 80    /* search.FingerprintLen (pkg/search/verifier.go:130) */

typedef struct z80b_ctx z80b_ctx;

/* cpu.State (pkg/cpu/state.go:11-15) in C layout (12 bytes). */
typedef struct z80b_state {
  uint8_t a, f, b, c, d, e, h, l;
  uint16_t sp;
  uint8_t m, pad;
} z80b_state;

/* result.Rule (pkg/result/table.go:11-17) plus the index of its target in
 * the job.  dead_regs is the register extension (bit 0..5 = B,C,D,E,H,L):
 * 0 for every rule of the reference semantics. */
typedef struct z80b_rule {
  uint32_t src[4];
  uint32_t rep[4];
  int32_t src_len, rep_len;
  int32_t bytes_saved, cycles_saved;
  int32_t dead_flags;
  int32_t target_index;
  int32_t dead_regs;
  int32_t reserved;
} z80b_rule;

typedef struct z80b_stats {
  uint64_t targets;
  uint64_t checks;          /* (target, candidate) QuickCheck evaluations after the
                               byte-size and prune filters */
  uint64_t checked_ref;     /* the reference's 'checked' counter (worker.go:134) */
  uint64_t qc_survivors;
  uint64_t mid_survivors;   /* Z80B_MODE_ALL only */
  uint64_t exhaustive_pairs;
  uint64_t exhaustive_states;
  uint64_t rules;
  uint32_t rounds;          /* ExhaustiveCheck rounds of the first-found pass */
  uint32_t launches;        /* kernels launched by this call */
  double device_ms;         /* whole pipeline, first to last event on the context's stream */
  double qc_ms, exh_ms;     /* summed durations of the QuickCheck scan kernels and of the
                               ExhaustiveCheck kernels (CUDA events around each launch) */
  uint64_t exhaustive_evaluated; /* states the sweep kernel ran: exhaustive_states less what
                               the A-independent sweeps skip (2 of 256 values of A decide) */
} z80b_stats;

/* Semantics of a search job. */
#define Z80B_MODE_FIRST 0 /* pkg/search worker.go:124-265: per target the first
                             candidate (enumeration order, shortest length first)
                             passing QuickCheck + ExhaustiveCheck; then, if dead
                             flags are set, the masked pass */
#define Z80B_MODE_ALL 1   /* pkg/gpu/search.go:80-199: fingerprint QuickCheck,
                             byte filter, prune, MidCheck, ExhaustiveCheck; every
                             passing length-1 candidate kept */
/* Execution path. */
#define Z80B_PATH_BATCHED 0 /* every target of the job in one pipeline */
#define Z80B_PATH_PLAIN 1   /* one target per launch, synchronizing per target */

typedef struct z80b_job {
  const uint32_t* targets;      /* n_targets * target_stride packed instructions */
  const uint8_t* target_lens;   /* per-target length 1..4, or NULL: target_len */
  const uint8_t* dead_flags;    /* per-target dead-flag mask or NULL: global_dead_flags */
  const uint8_t* dead_regs;     /* per-target dead-register mask (extension) or NULL */
  uint32_t n_targets;
  uint32_t target_len;
  uint32_t target_stride;       /* words per target, >= the longest target */
  uint32_t max_cand_len;        /* 1: candidates are the 4,531 8-bit instructions;
                                   2 (Z80B_MODE_FIRST): then, for targets without a
                                   length-1 winner, the 4,531^2 instruction pairs in
                                   EnumerateSequences8(2) order */
  uint32_t global_dead_flags;   /* search.FlagMask applied to every target */
  uint32_t mode;                /* Z80B_MODE_* */
  uint32_t path;                /* Z80B_PATH_* */
  uint32_t flags;               /* Z80B_JOB_* bits, 0 for the default pipeline */
} z80b_job;
/* Z80B_MODE_ALL only: report every MidCheck survivor without the
 * ExhaustiveCheck tier (cuda/z80_search_v2.cu --no-exhaust,
 * z80_search_v2.cu:944-948); such rules are candidates, not proofs. */
#define Z80B_JOB_NO_EXHAUSTIVE 1u

/* ---- context ---------------------------------------------------------- */
int z80b_init(int device, z80b_ctx** out);
void z80b_destroy(z80b_ctx* ctx);
const char* z80b_last_error(const z80b_ctx* ctx);
const char* z80b_status_string(int status);
int z80b_version(void);

/* ---- primitives --------------------------------------------------------- */
/* search.Fingerprint (pkg/search/verifier.go:134-151) of n sequences of
 * `len` instructions each: 80 bytes per sequence into out. */
int z80b_fingerprints(z80b_ctx* ctx, const uint32_t* seqs, uint32_t n, uint32_t len, uint8_t* out);

/* Runs n sequences (stride words, lengths lens[] or len) from initial states
 * in[] and writes the final states (execSeq, pkg/search/verifier.go:75-81). */
int z80b_exec(z80b_ctx* ctx, const z80b_state* in, const uint32_t* seqs, const uint8_t* lens,
              uint32_t len, uint32_t stride, uint32_t n, z80b_state* out);

/* gpu.NewCUDAProcess (pkg/gpu/cuda.go:32-75): uploads the candidate list
 * once; count * seq_len packed instructions. */
int z80b_load_candidates(z80b_ctx* ctx, const uint32_t* cands, uint32_t count, uint32_t seq_len);

/* CUDAProcess.QuickCheckGPU (pkg/gpu/cuda.go:79-107): indices (ascending) of
 * the loaded candidates whose 80-byte fingerprint equals fp with the flag
 * bits of dead_flags ignored in every F byte.  Writes up to cap indices and
 * the full count to *n_hits (Z80B_ECAPACITY if count > cap). */
int z80b_quickcheck(z80b_ctx* ctx, const uint8_t* fp80, uint32_t dead_flags, uint32_t* hits,
                    uint32_t cap, uint32_t* n_hits);

/* Batched verifier tiers over n (target, candidate) pairs: for pair i,
 * tgt[i*stride..] (tlens[i]) vs cand[i*stride..] (clens[i]).
 * tiers: bit0 QuickCheck[Masked], bit1 MidCheck[Masked], bit2
 * ExhaustiveCheck[Masked] (verifier.go:85-123,159-171,626-654); out[i] has
 * bit k set when tier k passed (tiers not requested are left 0).
 * dead: per-pair dead-flag masks or NULL (0).  flagdiff: optional out,
 * FlagDiff (verifier.go:658-673) per pair. */
int z80b_verify_pairs(z80b_ctx* ctx, const uint32_t* tgt, const uint8_t* tlens,
                      const uint32_t* cand, const uint8_t* clens, uint32_t stride, uint32_t n,
                      const uint8_t* dead, uint32_t tiers, uint8_t* out, uint8_t* flagdiff);

/* ---- whole pipeline ------------------------------------------------------ */
/* Runs the job and writes its rules (grouped by target index; within a
 * target the full-equivalence rule precedes the masked one, and all-hits
 * rules follow candidate order).  Writes up to cap rules and the total to
 * *n_rules (Z80B_ECAPACITY if it did not fit).  stats may be NULL.  The
 * job's arrays are read during the call only (targets in page-locked memory
 * are copied by DMA, in chunks for large jobs, while the host checks them);
 * the call returns after its GPU work has finished. */
int z80b_search(z80b_ctx* ctx, const z80b_job* job, z80b_rule* out, uint64_t cap,
                uint64_t* n_rules, z80b_stats* stats);

/* z80b_search with each target's answer handed to cb as soon as it is final
 * (both its full and its masked lane have a winner or have no candidate left
 * to try), before the whole job ends: cb(user, target_index, rules, n) with
 * the target's 0..2 rules in z80b_search's order; called once per target, on
 * the calling thread.  Batched first-found jobs only.  For callers that
 * answer queries individually (the serving loop), so one slow target does
 * not hold the answers of the others. */
typedef void (*z80b_rule_cb)(void* user, uint32_t target_index, const z80b_rule* rules, uint32_t n_rules);
int z80b_search_cb(z80b_ctx* ctx, const z80b_job* job, z80b_rule* out, uint64_t cap, uint64_t* n_rules,
                   z80b_stats* stats, z80b_rule_cb cb, void* user);

/* Device-resident variant for timing the pipeline without host copies:
 * z80b_stage_job uploads the job's targets once; z80b_run_staged runs the
 * pipeline on them and keeps the rules on the device (count in *n_rules);
 * z80b_fetch_rules copies them out. */
int z80b_stage_job(z80b_ctx* ctx, const z80b_job* job);
int z80b_run_staged(z80b_ctx* ctx, uint64_t* n_rules, z80b_stats* stats);
int z80b_fetch_rules(z80b_ctx* ctx, z80b_rule* out, uint64_t cap, uint64_t* n_rules);

/* ---- allocation-free ExhaustiveCheck -------------------------------------- */
/* No counterpart in the reference: an entry point for callers that cannot
 * allocate device memory -- a process whose GPU memory is budgeted by another
 * component, a latency path that must not pay for an allocation or for the
 * synchronization cudaFree implies, a plugin host that forbids allocator
 * calls.  It needs no context and allocates nothing (device or host heap):
 * its device scratch is a fixed 316 KiB array inside the library that every
 * GPU loading the library keeps until the process exits.
 *
 * ExhaustiveCheck[Masked] (pkg/search/verifier.go:159-171,642-654) of n
 * (target, candidate) pairs given as host arrays (as z80b_verify_pairs):
 * pass[i] = 1 when pair i is equivalent over the sweep, else 0.  At most
 * Z80B_NOALLOC_MAX_PAIRS pairs per call (larger n returns Z80B_ECAPACITY and
 * does nothing); stride <= 4.  stream may be NULL (default stream).  The
 * work runs on `device`; the calling thread's current device is the same
 * after the call as before it.
 * The first call on a device sets the scratch up on that device (symbol
 * address, lookup tables); make that first call before any stream capture.
 * Every call reuses the same scratch array (one per process and device, its
 * contents left over from the previous call; what must start at zero is
 * cleared by each call).  Calls in one process are serialized on the host and
 * return only after their GPU work has finished, so they never overlap; GPU
 * work that reaches the array by another route while a call runs (a captured
 * copy of a call replayed later) would race with it. */
#define Z80B_NOALLOC_MAX_PAIRS 4096
int z80b_exhaustive_noalloc(int device, const uint32_t* tgt, const uint8_t* tlens, const uint32_t* cand,
                            const uint8_t* clens, uint32_t stride, uint32_t n, const uint8_t* dead,
                            uint8_t* pass, void* stream);

/* ---- tuning -------------------------------------------------------------- */
#define Z80B_OPT_EXH_LANE_STATES 1  /* ExhaustiveCheck states per lane per dispatch: 1, 2, 4, 8 */
#define Z80B_OPT_EXH_CHUNK_BLOCKS 2 /* A-blocks (256 states) per work chunk: 1..4096 */
#define Z80B_OPT_STREAM_PRIORITY 3  /* the context's stream: -1 high, 0 default, 1 low priority */
#define Z80B_OPT_QC_INDEX 4         /* QuickCheck through the pool's bucket index: 1 (default) or 0 (scan every candidate) */
#define Z80B_OPT_XINDEP_BITS 5      /* A-independent sweeps bit-sliced (1, default) or one state per lane slot (0) */
#define Z80B_OPT_COMPACT_SWEEP 6    /* pairs naming at most two of B..L on the A/F/B/C-state kernel (1, default) or not (0) */
#define Z80B_OPT_GRAPH_ROUNDS 7     /* first-found ExhaustiveCheck rounds driven on the device by one CUDA graph (1, default;
                                       not for z80b_search_cb, whose callbacks follow the rounds) or from the host (0) */
#define Z80B_OPT_WIDE_SWEEP 8       /* other A-dependent pairs naming at most four of B..L and not SP on the
                                       A/F/B/C/H/L/M-state kernel, and the rest that name neither SP nor the memory
                                       byte on the A/F/B..L-state kernel (1, default), or neither (0) */
#define Z80B_OPT_CONCURRENT_SWEEPS 9 /* device-driven rounds: the sweep classes' kernels on parallel branches of the
                                       round graph (1, default) or one after another (0) */
#define Z80B_OPT_QC_SINGLE_PASS 10  /* bucket-index QuickCheck: the count pass keeps the survivors of targets with at
                                       most 8 and the collect pass runs for the others alone (1, default), or the
                                       collect pass runs for every target (0) */
int z80b_set_option(z80b_ctx* ctx, int option, int value);
int z80b_get_option(const z80b_ctx* ctx, int option, int* value);

typedef struct z80b_tune_trial {
  int xindep_bits;            /* Z80B_OPT_XINDEP_BITS of the trial */
  int lane_states;            /* Z80B_OPT_EXH_LANE_STATES (scalar A-independent kernel); 0 when bit-sliced */
  int chunk_blocks;           /* Z80B_OPT_EXH_CHUNK_BLOCKS: sweep units per work chunk */
  int compact;                /* Z80B_OPT_COMPACT_SWEEP and Z80B_OPT_WIDE_SWEEP (set together) */
  double ms;                  /* device ms of the pipeline on the sample */
  char kernels[96];           /* the sweep kernels it launched, "k_exhaustive<K,CLS>" joined by '+' */
} z80b_tune_trial;
#define Z80B_TUNE_MAX_TRIALS 64
typedef struct z80b_tune_result {
  int lane_states;            /* the chosen setting, now the context's */
  int chunk_blocks;
  int xindep_bits;
  int compact;
  int n_trials;
  z80b_tune_trial trials[Z80B_TUNE_MAX_TRIALS];
} z80b_tune_result;
/* Runs the job (a representative sample) once per sweep configuration --
 * A-independent kernel (bit-sliced, or scalar with 1/2/4/8 states per lane
 * per dispatch) x units per chunk (8, 32, 128, 512) x compact kernels off/on,
 * 40 distinct kernel configurations -- keeps the fastest for this context
 * and reports every trial with the kernels it launched.  The rules of the
 * trials are discarded.  No counterpart in the reference (its launch shape
 * is fixed, cuda/z80_search_v2.cu:900-948). */
int z80b_autotune(z80b_ctx* ctx, const z80b_job* sample, z80b_tune_result* out);

/* ---- constant-multiply search (cmd/mulopt) ---------------------------------
 * Replaces findOptimal (cmd/mulopt/main.go:186-229) for every requested
 * constant at once, and the reference's per-K CUDA searchers
 * (cuda/z80_mulopt.cu:232-303, cuda/z80_mulopt_fast.cu).  Per K the result is
 * the shortest sequence with A_out = A_in * K (mod 256) for all 256 inputs,
 * then the fewest T-states, then the first in odometer order (main.go:194-207),
 * so ops are deterministic (the CUDA searchers pick among equal-cost ties by a
 * race). */
#define Z80B_MULPOOL_MULOPT 0 /* cmd/mulopt/main.go:25-49, 14 ops, state zero but A */
#define Z80B_MULPOOL_WIDE21 1 /* the 21-op constant-multiply workload pool (pkg/cpu semantics) */
#define Z80B_MULPOOL_FAST14 2 /* cuda/z80_mulopt_fast.cu:20-51, 14 ops */
#define Z80B_MULPOOL_CUDA21 3 /* cuda/z80_mulopt.cu:19-48, 21 ops */

typedef struct z80b_mul_result {   /* MulResult (cmd/mulopt/main.go:162-167) */
  int32_t k;
  int32_t found;       /* 0: no sequence up to max_len ("NOT FOUND") */
  int32_t length;
  int32_t tstates;
  uint8_t ops[16];     /* pool indices, `length` entries (names: z80b_mul_pool) */
  uint64_t index;      /* odometer index of ops among the pool^length sequences */
} z80b_mul_result;

typedef struct z80b_mul_stats {
  uint64_t sequences;      /* sequences walked: sum of pool^L over the lengths searched */
  uint64_t per_k_sequences;/* sequences the per-K odometers would test: sum over K of its lengths' pool^L */
  uint64_t filter_nodes;   /* warp-level tree nodes whose leaves passed the x=2/x=255 filter */
  uint64_t full_checks;    /* all-256-input tests run */
  uint64_t full_pass;      /* tests passed */
  int32_t lengths;         /* lengths searched */
  int32_t launches;
  double device_ms;        /* device time of the search kernels */
} z80b_mul_stats;

/* Pool description: instruction count, longest searchable length, and (when
 * names / tstates are not NULL) up to `cap` names and T-state costs. */
int z80b_mul_pool(int pool, int* n_ops, int* max_len, const char** names, int* tstates, int cap);
/* Searches lengths min_len..max_len for the constants ks[0..n_k) (each 2..255;
 * ks = NULL searches 2..255 and writes 254 results).  init_b, init_c, init_f
 * are the initial B, C, F (0, 0, 0 for the reference's pools); A', F' and
 * the shadow B' start at 0.  out[i] answers ks[i]. */
int z80b_mul_search(z80b_ctx* ctx, int pool, uint8_t init_b, uint8_t init_c, uint8_t init_f, int min_len,
                    int max_len, const int32_t* ks, uint32_t n_k, z80b_mul_result* out, z80b_mul_stats* stats);

/* ---- serving loop ---------------------------------------------------------
 * Queries (a target of 1..4 instructions plus its dead flags and dead
 * registers) are answered like SearchSingle[Masked] (pkg/search/search.go:
 * 82-110) with candidates shorter than the target, up to max_cand_len
 * instructions.  Several workers, each with its own context and stream, run
 * batches of waiting queries concurrently (continuous batching: queries that
 * arrive while batches are in flight are admitted by the next free worker;
 * queries whose target alone implies an ExhaustiveCheck sweep of 2^32
 * states or more run alone on a low-priority stream);
 * admission charges each query the device memory its batch holds for it
 * (lanes, survivor records at their bound for its target's size and passes,
 * pair slots, length-2 slots, rule records) against memory_budget, and a
 * query waits until its charge fits; z80b_server_submit returns
 * Z80B_ECAPACITY for a query whose charge alone exceeds the budget.
 * Answers of length-4 targets carry Z80B_ANSWER_TRUNCATED (candidates of 3
 * instructions are not searched).  No counterpart in the reference (its
 * serving is one query per z80opt target call). */
typedef struct z80b_server z80b_server;
typedef struct z80b_server_config {
  int device;
  int workers;               /* concurrent batches (contexts); 0: 4 */
  uint32_t max_batch;        /* queries per batch; 0: 512 */
  uint64_t memory_budget;    /* device bytes of admitted query frontiers; 0: 64 GiB */
  uint32_t max_cand_len;     /* 1 or 2; 0: 2 */
} z80b_server_config;
typedef struct z80b_query {
  uint64_t id;
  uint32_t target[4];        /* packed op | imm << 16 */
  uint8_t len;               /* 1..4 */
  uint8_t dead_flags;
  uint8_t dead_regs;         /* bit0..5 = B,C,D,E,H,L */
  uint8_t reserved;
} z80b_query;
typedef struct z80b_answer {
  uint64_t id;
  int32_t status;            /* Z80B_OK or the status of the query's batch */
  int32_t n_rules;           /* 0..2: the full-equivalence rule first, then the masked one */
  z80b_rule rules[2];
  double queued_ms;          /* submit -> batch start */
  double service_ms;         /* batch start -> answer */
  double latency_ms;         /* submit -> answer */
  uint32_t batch_size;       /* 0: answered without device work (length-1 target) */
  uint32_t flags;            /* Z80B_ANSWER_* */
} z80b_answer;
/* The query's own candidate limit (target length - 1, SearchSingle's
 * MaxCandLen, pkg/search/search.go:27-29) is above the server's
 * max_cand_len: only candidates of up to max_cand_len instructions were
 * searched (length-4 targets: 3-instruction candidates were not), so a
 * shorter 3-instruction equivalent may exist that the answer does not give. */
#define Z80B_ANSWER_TRUNCATED 1u
typedef struct z80b_server_stats {
  uint64_t submitted, answered, errors, batches, max_batch_seen, pending, inflight_bytes;
  double device_ms;          /* summed pipeline device time of the batches */
  uint64_t peak_inflight_bytes; /* most frontier bytes admitted at once (never above memory_budget) */
} z80b_server_stats;
int z80b_server_start(const z80b_server_config* cfg, z80b_server** out);
int z80b_server_submit(z80b_server* s, const z80b_query* q, uint32_t n);  /* thread-safe */
/* Completed answers (any order), up to cap; waits up to timeout_ms for the first. */
int z80b_server_poll(z80b_server* s, z80b_answer* out, uint32_t cap, uint32_t* n, int timeout_ms);
int z80b_server_get_stats(z80b_server* s, z80b_server_stats* out);
/* Answers every submitted query, joins the workers and frees the server. */
int z80b_server_stop(z80b_server* s);

/* ---- host helpers (no device work) ---------------------------------------- */
/* inst.Catalog entry (pkg/inst/catalog.go:4-145): mnemonic with n/nn
 * placeholders, encoded size incl. immediate, T-states, immediate kind
 * (0 none, 1 imm8, 2 imm16) and the opReads/opWrites register masks
 * (pkg/search/verifier.go:199-408, pruner.go:66-236). */
int z80b_op_info(uint32_t op, char* mnemonic, uint32_t cap, int* size, int* tstates, int* imm_kind,
                 int* reads, int* writes);
/* inst.Disassemble of a sequence joined by " : " (pkg/search/worker.go:273-282);
 * returns the text length, -1 on a bad opcode. */
int z80b_disasm_seq(const uint32_t* seq, uint32_t n, char* buf, uint32_t cap);
/* parseAssembly (cmd/z80opt/main.go:325-397): returns the instruction count
 * (writing up to cap) or -1 when the text does not parse. */
int z80b_parse_assembly(const char* text, uint32_t* out, uint32_t cap);
/* parseDeadFlags (cmd/z80opt/main.go:305-322). */
int z80b_parse_dead_flags(const char* text, uint32_t* out);
/* result.DeadFlagDesc (pkg/result/output.go:93-129). */
int z80b_dead_flag_desc(uint32_t mask, char* buf, uint32_t cap);
/* search.ShouldPrune (pkg/search/pruner.go:7-35): 1, 0, or -1 on a bad opcode. */
int z80b_should_prune(const uint32_t* seq, uint32_t n);
/* ShouldPrune of n sequences (lens[i] words at seqs + i*stride): out[i] = 1, 0,
 * or 0xFF on a bad opcode or length. */
int z80b_should_prune_batch(const uint32_t* seqs, const uint8_t* lens, uint32_t stride, uint64_t n, uint8_t* out);
/* The 8-bit instruction list in EnumerateSequences8 order
 * (pkg/search/enumerator.go:319-345); returns its length (4531). */
uint32_t z80b_pool8(uint32_t* out, uint32_t cap);
/* EnumerateSequences + ShouldPrune over a caller's instruction pool
 * (pkg/search/enumerator.go:280-345, search.go:341-361): the unpruned
 * sequences of length len (1..4) in odometer order, len words each; writes up
 * to cap sequences and returns the total. */
uint64_t z80b_enumerate(const uint32_t* pool, uint32_t npool, uint32_t len, uint32_t* out, uint64_t cap);
/* result.WriteJSON (pkg/result/output.go:70-90). */
long long z80b_rules_json(const z80b_rule* rules, uint64_t n, char* buf, uint64_t cap);

#ifdef __cplusplus
}
#endif
#endif /* Z80B200_H_ */
