// z80b_kernels.cu -- the CUDA kernels of the verification pipeline (sm_100a).
//
// Tier 1, QuickCheck (pkg/search/verifier.go:85-94,626-638): one warp per
// target.  Lanes 0..7 run the target on the eight test vectors (same opcode
// in every lane), the outputs are broadcast with shuffles, then the warp
// scans the candidate table 32 candidates at a time.  Candidate outputs are
// precomputed once (k_pool_outputs), so a check is a compare of vector 0
// (one 16-byte shared-memory load) and, on the rare match, of vectors 1..7.
// __ballot_sync turns the per-lane verdicts into ordered survivor slots.
//
// Tier 2, MidCheck (verifier.go:98-123): one warp per pair, lane v runs both
// sequences on MidCheck vector v, __all_sync decides.
//
// Tier 3, ExhaustiveCheck (verifier.go:159-612,642-853): the sweep of a pair
// is cut into chunks of "A-blocks" (the 256 values of A for one carry and
// one assignment of the swept registers).  A persistent grid pulls chunks
// from an atomic dispenser; within a chunk the 32 lanes take 32 consecutive
// A values, so every lane executes the same opcode and the swept registers
// are warp-uniform.  A mismatch sets the pair's rejected flag, which the
// other chunks of the pair poll to stop early.  The reference's sweep order
// only matters for its early exit; the verdict (all states equal) does not
// depend on it.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>

#include "z80_bits.cuh"
#include "z80_tables.h"
#include "z80b_kernels.cuh"

namespace z80b {

namespace {
constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr uint32_t kResolved = 0x80000000u;
constexpr int kBlock = 256;

// Tables that lanes index with different values live in global memory (L1
// cached; lane-indexed __constant__ loads would serialise); __constant__ is
// kept for the reduced-sweep values, whose index is the same in every lane
// of a warp.  Every kernel that runs z_step gives all lanes of a warp the
// same opcode (a per-lane 455-way switch serialises by opcode).  A flag that
// other warps write (the pair's rejection flag) is read by lane 0 and
// broadcast, never read per lane in front of a warp collective: lanes that
// read it at different times would leave the warp split at the next
// __shfl_sync / __any_sync, which is undefined.
__device__ OpInfo g_ops[kNumOps];
__device__ uint32_t g_vec[32][3];  // MidCheck vectors; the first 8 are the QuickCheck vectors
__constant__ uint8_t c_rep[32];
__constant__ uint16_t c_repsp[16];
// Lane-indexed copies of the sweep values and the A-dependence class per
// opcode (AClass of z80_tables.h).
__device__ uint8_t g_rep[32];
__device__ uint16_t g_repsp[16];
__device__ uint8_t g_aclass[kNumOps];
// compact sweep: renamed opcodes and register places per register set
// (compact_tables), the registers each opcode names
__device__ int16_t g_cren[kCompactSets][kNumOps];
__device__ int8_t g_corig[kCompactSets][2];
__device__ uint8_t g_cid[64];
__device__ uint8_t g_opregs[kNumOps];
// wide compact sweep: the same per register set of at most four registers
// (wide_tables)
// input fields each output field of an opcode depends on (op_deps), and
// whether it leaves A exactly as it was (op_keeps_a)
__device__ uint32_t g_dep[kNumOps][kDepFields];
__device__ uint8_t g_keepa[kNumOps];
__device__ uint16_t g_keeps[kNumOps];  // fields (read-mask bits) an opcode leaves exactly as they were
__device__ int16_t g_wren[kWideSets][kNumOps];
__device__ int8_t g_worig[kWideSets][4];
__device__ uint8_t g_wid[64];

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Runs n instructions held one per lane (lane first+i holds instruction i).
// Every lane of the warp must call this with the same n.
__device__ __forceinline__ void run_lanes(Z80S& s, uint32_t lane_word, int first, int n) {
#pragma unroll 1
  for (int i = 0; i < n; i++) {
    uint32_t w = __shfl_sync(kFull, lane_word, first + i);
    z_step(s, w & 0xFFFFu, w >> 16);
  }
}

__device__ __forceinline__ Z80S vec_state(int v) {
  return z_unpack(g_vec[v][0], g_vec[v][1], g_vec[v][2]);
}

// Byte masks of compared registers from keepR bits (B,C,D,E,H,L).
struct Keep {
  uint32_t f, b, c, d, e, h, l, sp, m;
};
__device__ __forceinline__ Keep make_keep(uint32_t keepF, uint32_t keepR, bool cmpM) {
  Keep k;
  k.f = keepF & 0xFFu;
  k.b = (keepR & 1u) ? 0xFFu : 0u;
  k.c = (keepR & 2u) ? 0xFFu : 0u;
  k.d = (keepR & 4u) ? 0xFFu : 0u;
  k.e = (keepR & 8u) ? 0xFFu : 0u;
  k.h = (keepR & 16u) ? 0xFFu : 0u;
  k.l = (keepR & 32u) ? 0xFFu : 0u;
  k.sp = 0xFFFFu;
  k.m = cmpM ? 0xFFu : 0u;
  return k;
}
__device__ __forceinline__ bool eq_keep(const Z80S& x, const Z80S& y, const Keep& k) {
  uint32_t d = (x.a ^ y.a) | ((x.f ^ y.f) & k.f) | ((x.b ^ y.b) & k.b) | ((x.c ^ y.c) & k.c) |
               ((x.d ^ y.d) & k.d) | ((x.e ^ y.e) & k.e) | ((x.h ^ y.h) & k.h) | ((x.l ^ y.l) & k.l) |
               ((x.sp ^ y.sp) & k.sp) | ((x.m ^ y.m) & k.m);
  return d == 0;
}
// Registers (B,C,D,E,H,L -> bit 0..5) differing between packed words.
__device__ __forceinline__ uint32_t reg_diff(uint32_t d0, uint32_t d1) {
  return ((d0 >> 16) & 0xFFu ? 1u : 0u) | ((d0 >> 24) ? 2u : 0u) | ((d1 & 0xFFu) ? 4u : 0u) |
         ((d1 >> 8) & 0xFFu ? 8u : 0u) | ((d1 >> 16) & 0xFFu ? 16u : 0u) | ((d1 >> 24) ? 32u : 0u);
}

// Number of A-blocks of the ExhaustiveCheck sweep for a read mask
// (verifier.go:159-171,428-476); reduced: the reference's sweep of the pair
// is a reduced one although these reads alone would not make it so (swept
// registers left out, see put_pair).
__device__ __forceinline__ unsigned long long sweep_blocks(uint32_t reads, bool reduced = false) {
  uint32_t ext = reads & (kRegB | kRegC | kRegD | kRegE | kRegH | kRegL | kRegM);
  int n = __popc(ext);
  bool sp = (reads & kRegSP) != 0;
  if (n == 0 && !sp && !reduced) return 2ull;
  if (n <= 2 && !sp && !reduced) return 2ull << (8 * n);
  return (2ull << (5 * n)) * (sp ? 16ull : 1ull);
}
// Input fields (op_deps layout) that the outputs in `out` of a program can
// depend on: the dependency sets of its instructions, walked backwards.
__device__ __forceinline__ uint32_t dev_seq_relevant(const uint32_t* w, uint32_t n, uint32_t out) {
  for (int i = int(n) - 1; i >= 0; i--) {
    const uint32_t* d = g_dep[w[i] & 0xFFFFu];
    uint32_t in = 0;
    for (uint32_t o = out; o; o &= o - 1) in |= d[__ffs(o) - 1];
    out = in;
  }
  return out;
}
__device__ __forceinline__ uint32_t dev_seq_keeps(const uint32_t* w, uint32_t n) {
  uint32_t k = 0xFFFFu;
  for (uint32_t i = 0; i < n; i++) k &= g_keeps[w[i] & 0xFFFFu];
  return k;
}
__device__ __forceinline__ bool dev_seq_keeps_a(const uint32_t* w, uint32_t n) {
  for (uint32_t i = 0; i < n; i++)
    if (!g_keepa[w[i] & 0xFFFFu]) return false;
  return true;
}
// A-independent sweeps.  When no output of either sequence depends on the
// input A except A itself passing through (AClass folds of both sequences),
// every output but A is the same for all 256 values of A, and A_out is
// either A_in or a value independent of A_in in each sequence; two values of
// A then decide the verdict of all 256 (equal outputs at A = 0 and A = 1
// imply equal non-A outputs and either both pass A through or both write the
// same constant; a sequence passing A through against one writing a
// constant differs at one of the two).  Such a pair is swept as "units" of
// 128 A-blocks with A in {0, 1}: 256 states evaluated per unit instead of
// 32,768.  PairRec.keepR bit 6 marks it.
constexpr uint32_t kXIndep = 0x40u;
constexpr unsigned long long kUnitBlocks = 128;
__device__ __forceinline__ uint32_t dev_seq_aflow(const uint32_t* w, uint32_t n) {
  bool a_is_x = true;
  for (uint32_t i = 0; i < n; i++) {
    const uint32_t k = g_aclass[w[i] & 0xFFFFu];
    if (k == 0u && a_is_x) return 0u;
    if (k == 2u) a_is_x = false;
  }
  return a_is_x ? 3u : 1u;
}
__device__ __forceinline__ bool pair_xindep(const DevTargets& T, uint32_t t, const DevPool& P, uint32_t c) {
  return dev_seq_aflow(T.insn + (size_t)t * T.stride, target_len(T, t)) != 0u &&
         dev_seq_aflow(P.insn + (size_t)c * P.stride, pool_len(P, c)) != 0u;
}
// Compact sweep: 1 + the register-set entry when the pair's instructions
// name at most two of B..L, neither SP nor the memory byte, and all rename
// onto B and C (compact_map); 0 otherwise.
__device__ __forceinline__ uint8_t pair_cmap(const DevTargets& T, uint32_t t, const DevPool& P, uint32_t c) {
  const uint32_t tl = target_len(T, t), cl = pool_len(P, c);
  const uint32_t* tw = T.insn + (size_t)t * T.stride;
  const uint32_t* cw = P.insn + (size_t)c * P.stride;
  uint32_t fp = 0;
  for (uint32_t i = 0; i < tl; i++) fp |= g_opregs[tw[i] & 0xFFFFu];
  for (uint32_t i = 0; i < cl; i++) fp |= g_opregs[cw[i] & 0xFFFFu];
  if (fp & 0xC0u) return 0;
  const uint32_t id = g_cid[fp & 0x3Fu];
  if (!id) return 0;
  for (uint32_t i = 0; i < tl; i++)
    if (g_cren[id - 1][tw[i] & 0xFFFFu] < 0) return 0;
  for (uint32_t i = 0; i < cl; i++)
    if (g_cren[id - 1][cw[i] & 0xFFFFu] < 0) return 0;
  return uint8_t(id);
}
// Wide compact sweep: kWideClass | (1 + the register-set entry) when the
// pair's instructions name at most four of B..L and not SP, and all rename
// onto B, C, H and L (wide_map); 0 otherwise.
constexpr uint8_t kWideClass = 0x80u;
// Register-state sweep: the pair's instructions name neither SP nor the
// memory byte.
constexpr uint8_t kRegClass = 0x40u;
__device__ __forceinline__ bool pair_regstate(const DevTargets& T, uint32_t t, const DevPool& P, uint32_t c) {
  const uint32_t tl = target_len(T, t), cl = pool_len(P, c);
  uint32_t fp = 0;
  for (uint32_t i = 0; i < tl; i++) fp |= g_opregs[T.insn[(size_t)t * T.stride + i] & 0xFFFFu];
  for (uint32_t i = 0; i < cl; i++) fp |= g_opregs[P.insn[(size_t)c * P.stride + i] & 0xFFFFu];
  return (fp & 0xC0u) == 0u;
}
__device__ __forceinline__ uint8_t pair_wmap(const DevTargets& T, uint32_t t, const DevPool& P, uint32_t c) {
  const uint32_t tl = target_len(T, t), cl = pool_len(P, c);
  const uint32_t* tw = T.insn + (size_t)t * T.stride;
  const uint32_t* cw = P.insn + (size_t)c * P.stride;
  uint32_t fp = 0;
  for (uint32_t i = 0; i < tl; i++) fp |= g_opregs[tw[i] & 0xFFFFu];
  for (uint32_t i = 0; i < cl; i++) fp |= g_opregs[cw[i] & 0xFFFFu];
  if (fp & 0x80u) return 0;
  const uint32_t id = g_wid[fp & 0x3Fu];
  if (!id) return 0;
  for (uint32_t i = 0; i < tl; i++)
    if (g_wren[id - 1][tw[i] & 0xFFFFu] < 0) return 0;
  for (uint32_t i = 0; i < cl; i++)
    if (g_wren[id - 1][cw[i] & 0xFFFFu] < 0) return 0;
  return uint8_t(kWideClass | id);
}
// A-dependent pairs run bit-sliced (z80_bits.cuh): a unit is 4 A-blocks, a
// lane takes 32 consecutive values of A of one block.
constexpr unsigned long long kBitsBlocks = 4;
constexpr int kBitsWords = 88;  // planes of one ZB (A F B C D E H L M: 8 each, SP: 16)
__device__ __forceinline__ unsigned long long pair_units(unsigned long long nblocks, uint32_t keepR,
                                                         uint32_t xunit) {
  const unsigned long long xu = xunit ? xunit : kUnitBlocks;
  return (keepR & kXIndep) ? (nblocks + xu - 1) / xu : (nblocks + kBitsBlocks - 1) / kBitsBlocks;
}
constexpr unsigned long long kMaxChunks = 1ull << 20;
constexpr int kChunksPerWarp = 16;
// Work chunks of a sweep: cb A-blocks each (cb is the tuning option), at
// most kMaxChunks per pair.
__device__ __forceinline__ unsigned long long chunks_for(unsigned long long nb, uint32_t cb);
// Chunks of pair p in the numbering of its class (zero in the other one).
__device__ __forceinline__ void set_chunks(const RoundBuf& R, uint32_t p, const PairRec& pr) {
  const unsigned long long c = chunks_for(pair_units(pr.nblocks, pr.keepR, R.xunit), R.chunk_blocks);
  const bool xind = (pr.keepR & kXIndep) != 0;
  const bool wide = (pr.cmap & kWideClass) != 0;     // only set when R.wide
  const bool regs = pr.cmap == kRegClass;            // only set when R.wide
  const bool comp = pr.cmap != 0 && !wide && !regs;  // only set when R.compact
  const bool other = comp || wide || regs;
  R.nchunks[p] = (xind || other) ? 0ull : c;
  R.nchunks_x[p] = (xind && !other) ? c : 0ull;
  if (R.compact) R.nchunks_c[p] = comp ? c : 0ull;
  if (R.wide) {
    R.nchunks_w[p] = wide ? c : 0ull;
    R.nchunks_r[p] = regs ? c : 0ull;
  }
}
__device__ __forceinline__ unsigned long long chunks_for(unsigned long long nb, uint32_t cb) {
  unsigned long long c = (nb + cb - 1) / cb;
  return c > kMaxChunks ? kMaxChunks : c;
}

// ------------------------------------------------------------------ kernels

// Warp per candidate, lane v runs the candidate on vector v (lanes 0..7
// QuickCheck, 0..31 MidCheck); the opcode is the same in every lane.
__global__ void k_pool_outputs(const uint32_t* __restrict__ insn, uint32_t n, uint32_t len,
                               uint4* __restrict__ qc, uint4* __restrict__ mid) {
  const unsigned lane = lane_id();
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t c = gw; c < n; c += nw) {
    const uint32_t pw = lane < len ? insn[(size_t)c * len + lane] : 0u;
    Z80S s = vec_state(int(lane));
    run_lanes(s, pw, 0, int(len));
    uint32_t w[3];
    z_pack(s, w);
    const uint4 q = make_uint4(w[0], w[1], w[2], 0u);
    if (lane < 8) qc[(size_t)lane * n + c] = q;
    if (mid) mid[(size_t)lane * n + c] = q;
  }
}

// One warp per sequence; lane 0 runs it (arbitrary per-item opcodes would
// otherwise diverge inside the dispatch loop).
__global__ void k_exec(const uint32_t* __restrict__ in, const uint32_t* __restrict__ seqs,
                       const uint8_t* __restrict__ lens, uint32_t len, uint32_t stride, uint32_t n,
                       uint32_t* __restrict__ out) {
  const unsigned lane = lane_id();
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = gw; i < n; i += nw) {
    const uint32_t l = lens ? lens[i] : len;
    const uint32_t pw = lane < l ? seqs[(size_t)i * stride + lane] : 0u;
    Z80S s = z_unpack(in[3 * i], in[3 * i + 1], in[3 * i + 2]);
    run_lanes(s, pw, 0, int(l));
    if (lane == 0) {
      uint32_t w[3];
      z_pack(s, w);
      out[3 * i] = w[0];
      out[3 * i + 1] = w[1];
      out[3 * i + 2] = w[2];
    }
  }
}

// search.Fingerprint: 8 x {A,F,B,C,D,E,H,L,SP_hi,SP_lo}; warp per sequence,
// lane v (< 8) on test vector v.
__global__ void k_fingerprints(const uint32_t* __restrict__ seqs, uint32_t n, uint32_t len,
                               uint8_t* __restrict__ out) {
  const unsigned lane = lane_id();
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = gw; i < n; i += nw) {
    const uint32_t pw = lane < len ? seqs[(size_t)i * len + lane] : 0u;
    Z80S s = vec_state(int(lane & 7u));
    run_lanes(s, pw, 0, int(len));
    if (lane < 8) {
      uint8_t* p = out + (size_t)i * 80 + lane * 10;
      p[0] = uint8_t(s.a); p[1] = uint8_t(s.f); p[2] = uint8_t(s.b); p[3] = uint8_t(s.c);
      p[4] = uint8_t(s.d); p[5] = uint8_t(s.e); p[6] = uint8_t(s.h); p[7] = uint8_t(s.l);
      p[8] = uint8_t(s.sp >> 8); p[9] = uint8_t(s.sp);
    }
  }
}

// z80qc query semantics (cuda/z80_quickcheck.cu:666-681 over pkg/cpu
// outputs): candidate c matches when its fingerprint equals the query with
// the dead flag bits cleared in every F byte.
__global__ void k_fp_query(DevPool P, const uint32_t* __restrict__ fp, uint32_t dead,
                           uint32_t* __restrict__ hits, uint32_t* __restrict__ nhits, uint32_t cap) {
  uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  bool hit = false;
  if (c < P.n) {
    uint32_t keep0 = ~(dead << 8);
    hit = true;
#pragma unroll
    for (int v = 0; v < 8; v++) {
      uint4 q = P.qc[(size_t)v * P.n + c];
      uint32_t d0 = (q.x ^ fp[3 * v]) & keep0, d1 = q.y ^ fp[3 * v + 1], d2 = (q.z ^ fp[3 * v + 2]) & 0xFFFFu;
      hit = hit && ((d0 | d1 | d2) == 0);
    }
  }
  unsigned b = __ballot_sync(kFull, hit);
  if (b) {
    uint32_t base = 0;
    if (lane_id() == 0) base = atomicAdd(nhits, (uint32_t)__popc(b));
    base = __shfl_sync(kFull, base, 0);
    uint32_t idx = base + __popc(b & lanemask_lt());
    if (hit && idx < cap) hits[idx] = c;
  }
}

// Target side of a QuickCheck: encoded bytes, T-states and reads of the
// target (summed over its lanes), its outputs on the 8 vectors (warp-uniform
// copies) and the compared bytes of the packed words under its dead masks.
struct QCTarget {
  uint32_t tb, tts, trd, tl;
  uint32_t tw[8][3];
  uint32_t keep0, keep1;
};
__device__ __forceinline__ void qc_target(const DevTargets& T, uint32_t t, QCTarget& g) {
  const unsigned lane = lane_id();
  const uint32_t tl = target_len(T, t);
  const uint32_t pw = lane < tl ? T.insn[(size_t)t * T.stride + lane] : 0u;
  uint32_t sz = 0, ts = 0, rd = 0;
  if (lane < tl) {
    const OpInfo oi = g_ops[pw & 0xFFFFu];
    sz = oi.size;
    ts = oi.tstates;
    rd = oi.reads;
  }
#pragma unroll
  for (int off = 2; off >= 1; off >>= 1) {
    sz += __shfl_down_sync(kFull, sz, off);
    ts += __shfl_down_sync(kFull, ts, off);
    rd |= __shfl_down_sync(kFull, rd, off);
  }
  g.tl = tl;
  g.tb = __shfl_sync(kFull, sz, 0);
  g.tts = __shfl_sync(kFull, ts, 0);
  g.trd = __shfl_sync(kFull, rd, 0);
  Z80S s = vec_state(int(lane & 7u));
  run_lanes(s, pw, 0, int(tl));
  uint32_t w[3];
  z_pack(s, w);
#pragma unroll
  for (int v = 0; v < 8; v++) {
    g.tw[v][0] = __shfl_sync(kFull, w[0], v);
    g.tw[v][1] = __shfl_sync(kFull, w[1], v);
    g.tw[v][2] = __shfl_sync(kFull, w[2], v);
  }
  const uint32_t dead = target_dead(T, t) & 0xFFu;
  const uint32_t dregs = target_dead_regs(T, t) & 0x3Fu;
  g.keep0 = 0xFFu | ((~dead & 0xFFu) << 8) | ((dregs & 1u) ? 0u : 0xFF0000u) | ((dregs & 2u) ? 0u : 0xFF000000u);
  g.keep1 = ((dregs & 4u) ? 0u : 0xFFu) | ((dregs & 8u) ? 0u : 0xFF00u) | ((dregs & 16u) ? 0u : 0xFF0000u) |
            ((dregs & 32u) ? 0u : 0xFF000000u);
}

// QuickCheck of candidate c (vector-0 output q) against the target: fp
// (full equivalence; every pass in all-hits mode), mp (passes only under the
// dead masks), diff (FlagDiff | differing registers << 8 over the vectors).
__device__ __forceinline__ void qc_candidate(const DevPool& P, uint4 q, uint32_t c, const QCTarget& g,
                                             uint32_t keep2, bool all_hits, bool& fp, bool& mp, uint32_t& diff) {
  const uint32_t d0 = q.x ^ g.tw[0][0], d1 = q.y ^ g.tw[0][1], d2 = q.z ^ g.tw[0][2];
  if (((d0 & g.keep0) | (d1 & g.keep1) | (d2 & keep2)) != 0) return;
  bool full = (d0 | d1 | (d2 & keep2)) == 0;
  uint32_t fd = (d0 >> 8) & 0xFFu, rdf = reg_diff(d0, d1);
  bool ok = true;
#pragma unroll
  for (int v = 1; v < 8; v++) {
    const uint4 qv = P.qc[(size_t)v * P.n + c];
    const uint32_t e0 = qv.x ^ g.tw[v][0], e1 = qv.y ^ g.tw[v][1], e2 = qv.z ^ g.tw[v][2];
    ok = ok && (((e0 & g.keep0) | (e1 & g.keep1) | (e2 & keep2)) == 0);
    full = full && ((e0 | e1 | (e2 & keep2)) == 0);
    fd |= (e0 >> 8) & 0xFFu;
    rdf |= reg_diff(e0, e1);
  }
  if (!ok) return;
  if (all_hits) {
    fp = true;
  } else {
    fp = full;
    mp = !full;
  }
  diff = fd | (rdf << 8);
}

// Appends this warp's survivors of one 32-candidate step in enumeration
// order (collect pass) or tallies them per lane (count pass).
template <bool COLLECT>
__device__ __forceinline__ void qc_emit(const QCOut& o, bool fp, bool mp, uint32_t c, uint32_t diff, uint32_t obase,
                                        uint32_t nf_total, uint32_t& nf, uint32_t& nm, uint32_t& lf,
                                        uint32_t& lm) {
  if constexpr (!COLLECT) {
    lf += fp ? 1u : 0u;
    lm += mp ? 1u : 0u;
  } else {
    const unsigned bf = __ballot_sync(kFull, fp);
    const unsigned bm = __ballot_sync(kFull, mp);
    if (fp) {
      const uint32_t idx = obase + nf + __popc(bf & lanemask_lt());
      o.surv[idx] = c;
      o.sdiff[idx] = uint16_t(diff);
    }
    if (mp) {
      const uint32_t idx = obase + nf_total + nm + __popc(bm & lanemask_lt());
      o.surv[idx] = c;
      o.sdiff[idx] = uint16_t(diff);
    }
    nf += __popc(bf);
    nm += __popc(bm);
  }
}

// Count-pass epilogue: survivor counts and the target's metadata.
__device__ __forceinline__ void qc_count_out(const QCOut& o, uint32_t t, const QCTarget& g, uint32_t nf,
                                             uint32_t nm) {
  o.cnt_f[t] = nf;
  o.cnt_m[t] = nm;
  o.cnt_all[t] = nf + nm;
  TargetMeta m;
  m.tstates = uint16_t(g.tts);
  m.bytes = uint8_t(g.tb);
  m.len = uint8_t(g.tl);
  m.reads = uint16_t(g.trd);
  m.pad = 0;
  o.meta[t] = m;
}

template <bool COLLECT>
__global__ void __launch_bounds__(kBlock) k_qc_scan(DevTargets T, DevPool P, QCConfig cfg, QCOut o) {
  extern __shared__ uint4 smem[];
  uint4* s_q0 = smem;
  uint8_t* s_el = reinterpret_cast<uint8_t*>(smem + (cfg.use_smem ? P.n : 0));
  if (cfg.use_smem) {
    for (uint32_t i = threadIdx.x; i < P.n; i += blockDim.x) {
      s_q0[i] = P.qc[i];
      s_el[i] = uint8_t(P.size[i] | (P.prune[i] ? 0x80u : 0u));
    }
    __syncthreads();
  }
  const unsigned lane = lane_id();
  const uint32_t warps_per_block = blockDim.x >> 5;
  const uint32_t gw = blockIdx.x * warps_per_block + (threadIdx.x >> 5);
  const uint32_t nw = gridDim.x * warps_per_block;
  unsigned long long my_checks = 0;

  for (uint32_t t = gw; t < T.n; t += nw) {
    uint32_t nf_total = 0, obase = 0;
    if (COLLECT) {
      nf_total = o.cnt_f[t];
      if (nf_total + o.cnt_m[t] == 0) continue;
      obase = o.base[t];
    }
    QCTarget g;
    qc_target(T, t, g);
    uint32_t nf = 0, nm = 0;
    uint32_t lf = 0, lm = 0, lc = 0;  // count pass: per-lane tallies, reduced once per target
    for (uint32_t base = 0; base < P.n; base += 32) {
      const uint32_t c = base + lane;
      bool el = false;
      if (c < P.n) {
        uint32_t e = cfg.use_smem ? s_el[c] : (P.size[c] | (P.prune[c] ? 0x80u : 0u));
        el = (e & 0x7Fu) < g.tb && !(e & 0x80u);
      }
      bool fp = false, mp = false;
      uint32_t diff = 0;
      if (el) qc_candidate(P, cfg.use_smem ? s_q0[c] : P.qc[c], c, g, cfg.w2mask, cfg.all_hits != 0, fp, mp, diff);
      if constexpr (!COLLECT) lc += el ? 1u : 0u;
      qc_emit<COLLECT>(o, fp, mp, c, diff, obase, nf_total, nf, nm, lf, lm);
    }
    if constexpr (!COLLECT) {
      nf = __reduce_add_sync(kFull, lf);
      nm = __reduce_add_sync(kFull, lm);
      const uint32_t nc = __reduce_add_sync(kFull, lc);
      if (lane == 0) {
        my_checks += nc;
        qc_count_out(o, t, g, nf, nm);
      }
    }
  }
  if (!COLLECT && lane == 0 && my_checks) atomicAdd(o.checks, my_checks);
}

// Appends one pair per unresolved (target, kind) lane with an untried survivor.
// Allocates w consecutive pair slots for this thread (one atomic per warp;
// every lane of the warp takes part); returns the first slot.
__device__ __forceinline__ uint32_t alloc_pairs(uint32_t* counter, uint32_t w) {
  const unsigned lane = lane_id();
  uint32_t incl = w;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t v = __shfl_up_sync(kFull, incl, off);
    if (lane >= unsigned(off)) incl += v;
  }
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  uint32_t base = 0;
  if (lane == 31 && total) base = atomicAdd(counter, total);
  base = __shfl_sync(kFull, base, 31);
  return base + incl - w;
}

// Writes one pair of a round.
__device__ __forceinline__ void put_pair(const RoundBuf& R, uint32_t p, const DevTargets& T, const DevPool& P,
                                         const QCOut& q, uint32_t t, uint32_t kind, uint32_t c, uint32_t src,
                                         uint8_t wlen, uint32_t wend) {
  PairRec pr;
  const uint32_t reads = q.meta[t].reads | P.reads[c];
  pr.target = t;
  pr.cand = c;
  pr.keepF = kind ? uint8_t(~target_dead(T, t)) : uint8_t(0xFFu);
  pr.keepR = kind ? uint8_t((~target_dead_regs(T, t) & 0x3Fu) | 0x80u) : uint8_t(0x3Fu);
  if (pair_xindep(T, t, P, c)) pr.keepR |= uint8_t(kXIndep);
  // A swept register that no compared output of either program depends on
  // (dead registers and flags make this common in masked passes: SET 6, B
  // with B dead) cannot change the verdict, so one value of it stands for
  // all the reference sweeps: it is left out of the sweep, whose other
  // registers keep the reference's values (a reduced sweep stays reduced).
  // The same holds for the carry, the most significant field of the block
  // index: when no compared output depends on it, the first half of the
  // blocks (carry 0) decides.
  uint32_t swept = reads;
  pr.sweepf = 0;
  const uint32_t ext = reads & (kRegB | kRegC | kRegD | kRegE | kRegH | kRegL | kRegM);
  const uint32_t cmp = kRegA | kRegSP | kRegM | ((uint32_t(pr.keepR) & 0x3Fu) << 2) |
                       (uint32_t(pr.keepF) << kDepF0);
  const uint32_t* tw = T.insn + (size_t)t * T.stride;
  const uint32_t* cw = P.insn + (size_t)c * P.stride;
  const uint32_t tl = target_len(T, t), cl = pool_len(P, c);
  // what the compared outputs other than A, and A itself, depend on
  const uint32_t rest = dev_seq_relevant(tw, tl, cmp & ~uint32_t(kRegA)) | dev_seq_relevant(cw, cl, cmp & ~uint32_t(kRegA));
  const uint32_t at = dev_seq_relevant(tw, tl, kRegA), ac = dev_seq_relevant(cw, cl, kRegA);
  const uint32_t rel = rest | at | ac;
  uint32_t drop = ext & ~rel;
  // a swept register both programs keep exactly, on which no other compared
  // output depends, compares equal whatever its value: one value decides
  const uint32_t both = dev_seq_keeps(tw, tl) & dev_seq_keeps(cw, cl) & ext & ~drop;
  for (uint32_t b = both; b; b &= b - 1) {
    const uint32_t r = b & (0u - b);
    if (!((dev_seq_relevant(tw, tl, cmp & ~r) | dev_seq_relevant(cw, cl, cmp & ~r)) & r)) drop |= r;
  }
  const bool carry_out = (rel & (1u << kDepF0)) == 0;
  if (drop) {
    const bool red = (reads & kRegSP) != 0 || __popc(ext) > 2;
    swept = reads & ~drop;
    pr.sweepf = uint8_t((red ? 0x80u : 0u) | uint32_t(__popc(drop)) * (red ? 5u : 8u));
  }
  pr.reads = uint16_t(swept);
  pr.nblocks = sweep_blocks(swept, (pr.sweepf & 0x80u) != 0);
  if (carry_out) {
    pr.nblocks >>= 1;
    pr.sweepf += 1;
  }
  // Two values of A decide the pair when no compared output but A depends
  // on the input A (a comparison whose flags are dead or overwritten, A
  // copied into a dead register) and each program keeps A or computes its A
  // from other inputs: the argument of the A-independent sweeps under the
  // pair's masks.
  if (!(rest & kRegA) && (!(at & kRegA) || dev_seq_keeps_a(tw, tl)) && (!(ac & kRegA) || dev_seq_keeps_a(cw, cl)))
    pr.keepR |= uint8_t(kXIndep);
  // compact classes: A-dependent pairs, and A-independent ones when those
  // are swept bit-sliced (units of kXBitsBlocks); the narrow state first
  pr.cmap = 0;
  if (!(pr.keepR & kXIndep) || R.xunit == kXBitsBlocks) {
    if (R.compact) pr.cmap = pair_cmap(T, t, P, c);
    // the wide state: A-dependent pairs only
    if (!pr.cmap && R.wide && !(pr.keepR & kXIndep)) pr.cmap = pair_wmap(T, t, P, c);
    // the register state: the rest that name neither SP nor the memory byte
    if (!pr.cmap && R.wide && pair_regstate(T, t, P, c)) pr.cmap = kRegClass;
  }
  R.pairs[p] = pr;
  R.pair_src[p] = src;
  set_chunks(R, p, pr);
  R.rejected[p] = 0;
  R.wlen[p] = wlen;
  if (R.wend) {
    R.wend[p] = wend;
    R.cdone[p] = 0;
  }
}

// Lane 0, after a warp's chunk of pair p ran to its end without a mismatch:
// counts the chunk; the warp that counts the last one of a pair that still
// stands (its whole sweep passed) cancels the pairs after it in its survivor
// window (rejected 0 -> 2): the first passing pair of a window wins, so
// their sweeps cannot change the result.  A chunk with a mismatch rejects
// the pair and is not counted, so a rejected pair never reaches its count.
// nch = the pair's chunks.
__device__ __forceinline__ void chunk_passed(uint32_t* rejected, const uint32_t* wend, uint32_t* cdone, uint32_t p,
                                          uint32_t nch) {
  __threadfence();
  const uint32_t before = atomicAdd(&cdone[p], 1u);
  if (before + 1u != nch) return;
  __threadfence();
  if (atomicAdd(&rejected[p], 0u) != 0u) return;
  // windows hold at most 64 pairs; an unrolled, guarded run keeps a loop
  // out of the sweep kernels' loop nest (which made them spill)
  const uint32_t e = wend[p];
#pragma unroll
  for (uint32_t i = 1; i < 64; i++)
    if (p + i < e) atomicCAS(&rejected[p + i], 0u, 2u);
}

// One round of the length-1 pass: each unresolved (target, kind) lane puts
// its window of next survivors into the round (pairs past the buffer's
// capacity wait for the next round).
__global__ void k_round_build(DevTargets T, DevPool P, QCOut q, Lanes L, RoundBuf R) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
  for (uint32_t kind = 0; kind < 2; kind++) {
    uint32_t w = 0, nx = 0, sbase = 0;
    if (t < T.n) {
      const uint32_t cf = q.cnt_f[t], cm = q.cnt_m[t];
      const uint32_t idx = 2 * t + kind;
      nx = L.next[idx];
      if (!(nx & kResolved)) {
        const uint32_t cnt = kind ? cm : cf;
        if (nx >= cnt) {
          L.next[idx] = nx | kResolved;
        } else {
          w = min(1u << L.spec[idx], cnt - nx);
          sbase = q.base[t] + (kind ? cf : 0u) + nx;
        }
      }
    }
    if (!__any_sync(kFull, w != 0)) continue;
    const uint32_t p0 = alloc_pairs(R.npairs, w);
    const uint32_t fit = p0 >= R.cap ? 0u : min(w, R.cap - p0);
    for (uint32_t j = 0; j < fit; j++)
      put_pair(R, p0 + j, T, P, q, t, kind, q.surv[sbase + j], sbase + j, j == 0 ? uint8_t(fit) : uint8_t(0),
               p0 + fit);
  }
}

// pkg/gpu semantics: one pair per MidCheck survivor (all survivors when
// midpass is null).
__global__ void k_pairs_from_survivors(DevTargets T, DevPool P, QCOut q, const uint8_t* __restrict__ midpass,
                                       uint32_t nsurv, const uint32_t* __restrict__ surv_target,
                                       RoundBuf R) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  bool have = false;
  PairRec pr;
  if (i < nsurv && (!midpass || midpass[i])) {
    const uint32_t t = surv_target[i], c = q.surv[i];
    const uint32_t reads = q.meta[t].reads | P.reads[c];
    pr.target = t;
    pr.cand = c;
    pr.reads = uint16_t(reads);
    pr.nblocks = sweep_blocks(reads);
    pr.keepF = uint8_t(~target_dead(T, t));
    pr.keepR = uint8_t(~target_dead_regs(T, t) & 0x3Fu);
    if (pair_xindep(T, t, P, c)) pr.keepR |= uint8_t(kXIndep);
    pr.cmap = 0;
    pr.sweepf = 0;
    have = true;
  }
  unsigned b = __ballot_sync(kFull, have);
  if (!b) return;
  uint32_t base = 0;
  if (lane_id() == 0) base = atomicAdd(R.npairs, (uint32_t)__popc(b));
  base = __shfl_sync(kFull, base, 0);
  if (have) {
    uint32_t p = base + __popc(b & lanemask_lt());
    R.pairs[p] = pr;
    R.pair_src[p] = i;
    set_chunks(R, p, pr);
    R.rejected[p] = 0;
  }
}

// K = states per lane per dispatch ("vectors per lane").  One warp
// iteration covers 32*K values of A; an A-block (256 states) takes 8/K
// iterations.
// Initial register values of A-block ab (everything but A and F's carry),
// decoded field by field from the sweep shape: the same values as
// bdec_state, in a form that keeps the bit-sliced A-independent unit within
// its registers.  Block index fields fastest first: SP (reduced sweeps), the
// swept registers from the last to the first, carry.  UNIFORM selects the
// __constant__ tables (the index is the same in every lane) or their global
// copies (lane-dependent index).
template <bool UNIFORM>
__device__ __forceinline__ void decode_block(unsigned long long ab, bool spw, bool reduced, int nx, int fw,
                                             const int (&slot)[7], Z80S& init) {
  unsigned long long rest = ab;
  uint32_t sp = 0;
  if (spw) {
    sp = UNIFORM ? c_repsp[uint32_t(rest & 15ull)] : g_repsp[uint32_t(rest & 15ull)];
    rest >>= 4;
  }
  uint32_t fieldv[7];
#pragma unroll
  for (int f = 6; f >= 0; f--) {
    fieldv[f] = 0;
    if (f < nx) {
      const uint32_t x = uint32_t(rest) & (reduced ? 31u : 255u);
      fieldv[f] = reduced ? (UNIFORM ? c_rep[x] : g_rep[x]) : x;
      rest >>= fw;
    }
  }
  uint32_t rv[7];
#pragma unroll
  for (int r = 0; r < 7; r++) {
    uint32_t v = 0;
#pragma unroll
    for (int f = 0; f < 7; f++)
      if (slot[r] == f) v = fieldv[f];
    rv[r] = v;
  }
  init.a = 0;
  init.f = uint32_t(rest & 1ull);
  init.b = rv[0]; init.c = rv[1]; init.d = rv[2]; init.e = rv[3];
  init.h = rv[4]; init.l = rv[5]; init.m = rv[6];
  init.sp = sp;
}

// Runs the candidate then the target from K initial states (init(q, x)
// writes state q) and reports whether any compared output differs (only
// states with valid[q]).
template <int K, class Init>
__device__ __forceinline__ bool run_compare(const Init& init, const bool (&valid)[K], uint32_t pw, int tl, int cl,
                                            uint32_t keep0, uint32_t keep1) {
  Z80S X[K];
  uint32_t P0[K], P1[K], P2[K];
  const int nsteps = tl + cl;
  // one dispatch site: the candidate runs first; its output is packed into
  // three words per state, the registers are re-initialised and the target
  // runs on them
#pragma unroll 1
  for (int st = -1; st < nsteps; st++) {
    if (st == -1 || st == cl) {
      if (st == cl) {
#pragma unroll
        for (int q = 0; q < K; q++) {
          P0[q] = X[q].a | (X[q].f << 8) | (X[q].b << 16) | (X[q].c << 24);
          P1[q] = X[q].d | (X[q].e << 8) | (X[q].h << 16) | (X[q].l << 24);
          P2[q] = X[q].sp | (X[q].m << 16);
        }
      }
#pragma unroll
      for (int q = 0; q < K; q++) init(q, X[q]);
      if (st == -1) continue;
    }
    // lanes tl.. hold the candidate, lanes 0.. the target
    const int src = st < cl ? tl + st : st - cl;
    const uint32_t w = __shfl_sync(kFull, pw, src);
    z_stepK<K>(X, w & 0xFFFFu, w >> 16);
  }
  bool bad = false;
#pragma unroll
  for (int q = 0; q < K; q++) {
    const uint32_t d0 = (X[q].a | (X[q].f << 8) | (X[q].b << 16) | (X[q].c << 24)) ^ P0[q];
    const uint32_t d1 = (X[q].d | (X[q].e << 8) | (X[q].h << 16) | (X[q].l << 24)) ^ P1[q];
    const uint32_t d2 = (X[q].sp | (X[q].m << 16)) ^ P2[q];
    bad = bad || (valid[q] && ((d0 & keep0) | (d1 & keep1) | d2) != 0);
  }
  return bad;
}

// Planes of the 32 states A = a0 .. a0+31 (a0 a multiple of 32) with the
// other registers of x.
__device__ __forceinline__ void zb_init(ZB& z, const Z80S& x, uint32_t a0) {
  z.a[0] = 0xAAAAAAAAu;
  z.a[1] = 0xCCCCCCCCu;
  z.a[2] = 0xF0F0F0F0u;
  z.a[3] = 0xFF00FF00u;
  z.a[4] = 0xFFFF0000u;
  z.a[5] = (a0 & 32u) ? kZBOnes : 0u;
  z.a[6] = (a0 & 64u) ? kZBOnes : 0u;
  z.a[7] = (a0 & 128u) ? kZBOnes : 0u;
  zb_set8(z.f, x.f);
  zb_set8(z.b, x.b);
  zb_set8(z.c, x.c);
  zb_set8(z.d, x.d);
  zb_set8(z.e, x.e);
  zb_set8(z.h, x.h);
  zb_set8(z.l, x.l);
  zb_set8(z.m, x.m);
#pragma unroll
  for (int i = 0; i < 16; i++) z.sp[i] = ((x.sp >> i) & 1u) ? kZBOnes : 0u;
}
// Saves / compares the planes (s: this lane's column, stride 32 words).
__device__ __forceinline__ void zb_save(const ZB& z, uint32_t* s) {
#pragma unroll
  for (int i = 0; i < 8; i++) {
    s[(0 + i) * 32] = z.a[i];
    s[(8 + i) * 32] = z.f[i];
    s[(16 + i) * 32] = z.b[i];
    s[(24 + i) * 32] = z.c[i];
    s[(32 + i) * 32] = z.d[i];
    s[(40 + i) * 32] = z.e[i];
    s[(48 + i) * 32] = z.h[i];
    s[(56 + i) * 32] = z.l[i];
    s[(64 + i) * 32] = z.m[i];
  }
#pragma unroll
  for (int i = 0; i < 16; i++) s[(72 + i) * 32] = z.sp[i];
}
__device__ __forceinline__ uint32_t zb_diff(const ZB& z, const uint32_t* s, uint32_t keepF, uint32_t keepR) {
  uint32_t d = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    d |= z.a[i] ^ s[(0 + i) * 32];
    if ((keepF >> i) & 1u) d |= z.f[i] ^ s[(8 + i) * 32];
    if (keepR & 1u) d |= z.b[i] ^ s[(16 + i) * 32];
    if (keepR & 2u) d |= z.c[i] ^ s[(24 + i) * 32];
    if (keepR & 4u) d |= z.d[i] ^ s[(32 + i) * 32];
    if (keepR & 8u) d |= z.e[i] ^ s[(40 + i) * 32];
    if (keepR & 16u) d |= z.h[i] ^ s[(48 + i) * 32];
    if (keepR & 32u) d |= z.l[i] ^ s[(56 + i) * 32];
    d |= z.m[i] ^ s[(64 + i) * 32];
  }
#pragma unroll
  for (int i = 0; i < 16; i++) d |= z.sp[i] ^ s[(72 + i) * 32];
  return d;
}
// One unit (4 A-blocks) of an A-dependent sweep, bit-sliced: lane l takes
// block unit*4 + l/8 and A = (l%8)*32 .. +31; the candidate's outputs wait in
// shared memory while the target runs.  One dispatch site for both programs.
__device__ __forceinline__ bool bits_unit(unsigned long long u, unsigned long long nblocks, const BDec& bd,
                                          uint32_t pw, int tl, int cl, uint32_t keepF, uint32_t keepR, uint32_t* sm) {
  const unsigned lane = lane_id();
  const unsigned long long blk = u * kBitsBlocks + (lane >> 3);
  const bool valid = blk < nblocks;
  const Z80S x = bdec_state(bd, valid ? blk : u * kBitsBlocks, g_rep, g_repsp);
  const uint32_t a0 = (lane & 7u) * 32u;
  ZB z;
#pragma unroll 1
  for (int st = -1; st < tl + cl; st++) {
    if (st == -1 || st == cl) {
      if (st == cl) zb_save(z, sm);
      zb_init(z, x, a0);
      if (st == -1) continue;
    }
    const int src = st < cl ? tl + st : st - cl;
    const uint32_t w = __shfl_sync(kFull, pw, src);
    zb_step(z, w & 0xFFFFu, w >> 16);
  }
  return valid && zb_diff(z, sm, keepF, keepR) != 0u;
}

// One unit of a compact sweep: the layout of bits_unit (lane l: block 4u +
// l/8, A = 32(l % 8) .. +31) on the compact state (A, F, B, C; ZB4).  The
// pair's programs arrive renamed onto B and C; o0 / o1 are the original
// registers (0..5 = B..L) that B and C stand for, or -1 where none does.
// Only A, F (under keepF) and those registers (under keepR) can differ.
constexpr int kCompactWords = 32;  // planes saved per lane: A, F, B, C
__device__ __forceinline__ bool cbits_unit(unsigned long long u, unsigned long long nblocks, const CDec& dec,
                                           uint32_t pw, int tl, int cl, uint32_t keepF, uint32_t keepR, int o0, int o1,
                                           uint32_t* sm) {
  const unsigned lane = lane_id();
  const unsigned long long blk = u * kBitsBlocks + (lane >> 3);
  const bool valid = blk < nblocks;
  uint32_t vb, vc, carry;
  cdec_vals(dec, valid ? blk : u * kBitsBlocks, vb, vc, carry);
  const uint32_t a0 = (lane & 7u) * 32u;
  ZB4 z;
  auto init = [&]() {
    z.a[0] = 0xAAAAAAAAu;
    z.a[1] = 0xCCCCCCCCu;
    z.a[2] = 0xF0F0F0F0u;
    z.a[3] = 0xFF00FF00u;
    z.a[4] = 0xFFFF0000u;
    z.a[5] = (a0 & 32u) ? kZBOnes : 0u;
    z.a[6] = (a0 & 64u) ? kZBOnes : 0u;
    z.a[7] = (a0 & 128u) ? kZBOnes : 0u;
    zb_set8(z.f, carry);
    zb_set8(z.b, vb);
    zb_set8(z.c, vc);
  };
  init();
#pragma unroll 1
  for (int st = 0; st < tl + cl; st++) {
    if (st == cl) {
#pragma unroll
      for (int i = 0; i < 8; i++) {
        sm[(0 + i) * 32] = z.a[i];
        sm[(8 + i) * 32] = z.f[i];
        sm[(16 + i) * 32] = z.b[i];
        sm[(24 + i) * 32] = z.c[i];
      }
      init();
    }
    const int src = st < cl ? tl + st : st - cl;
    const uint32_t w = __shfl_sync(kFull, pw, src);
    zb4_step(z, w & 0xFFFFu, w >> 16);
  }
  const bool cmp_b = o0 >= 0 && ((keepR >> o0) & 1u), cmp_c = o1 >= 0 && ((keepR >> o1) & 1u);
  uint32_t d = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    d |= z.a[i] ^ sm[(0 + i) * 32];
    if ((keepF >> i) & 1u) d |= z.f[i] ^ sm[(8 + i) * 32];
    if (cmp_b) d |= z.b[i] ^ sm[(16 + i) * 32];
    if (cmp_c) d |= z.c[i] ^ sm[(24 + i) * 32];
  }
  return valid && d != 0u;
}

// A-independent sweeps, bit-sliced: lane l of a unit takes the 32 A-blocks
// u*1024 + 32l .. +31 as one state word (block j in bit j), first at A = 0,
// then at A = 1 (two values decide these pairs).  In an aligned group of 32
// blocks only the low 5 bits of the block index change, and they move one
// thing: the last swept register's low 5 bits (full sweep), its 32
// representative values (reduced sweep), SP's 16 representatives and one bit
// of the next field (SP sweep), or the carry (no extra register).
__device__ __forceinline__ void zb_set_reg(ZB& z, int r, const uint32_t (&pl)[8]) {
  switch (r) {
    case 0: zb_copy8(z.b, pl); break;
    case 1: zb_copy8(z.c, pl); break;
    case 2: zb_copy8(z.d, pl); break;
    case 3: zb_copy8(z.e, pl); break;
    case 4: zb_copy8(z.h, pl); break;
    case 5: zb_copy8(z.l, pl); break;
    case 6: zb_copy8(z.m, pl); break;
    default: break;
  }
}
__device__ __forceinline__ bool xbits_unit(unsigned long long u, unsigned long long nblocks, bool spw, bool reduced,
                                           int nx, int fw, const int (&slot)[7], int rlast, uint32_t pw, int tl,
                                           int cl, uint32_t keepF, uint32_t keepR, uint32_t* sm) {
  const unsigned lane = lane_id();
  const unsigned long long g0 = u * kXBitsBlocks + (unsigned long long)lane * 32ull;
  const uint32_t valid = g0 >= nblocks ? 0u
                         : (nblocks - g0 >= 32ull ? 0xFFFFFFFFu : ((1u << uint32_t(nblocks - g0)) - 1u));
  Z80S x;
  decode_block<false>(g0 < nblocks ? g0 : 0ull, spw, reduced, nx, fw, slot, x);
  // planes of what the low 5 bits of the block index move
  uint32_t vp[8], spp[16];
  uint32_t fp0 = 0u;
#pragma unroll
  for (int i = 0; i < 16; i++) spp[i] = 0u;
  if (spw) {
    // SP: state j takes representative j mod 16; bit 4: the last field's x
    // (even x0 in states 0-15, x0 + 1 in 16-31) or, with no field, the carry
#pragma unroll
    for (int i = 0; i < 16; i++) spp[i] = __ballot_sync(kFull, (g_repsp[lane & 15u] >> i) & 1u);
    const uint32_t x0 = uint32_t(g0 >> 4) & 31u;
    const uint32_t lo = g_rep[x0], hi = g_rep[(x0 + 1u) & 31u];
#pragma unroll
    for (int i = 0; i < 8; i++)
      vp[i] = (((lo >> i) & 1u) ? 0x0000FFFFu : 0u) | (((hi >> i) & 1u) ? 0xFFFF0000u : 0u);
    fp0 = 0xFFFF0000u;
  } else if (reduced) {
    // the last field's 32 representatives, state j = representative j
#pragma unroll
    for (int i = 0; i < 8; i++) vp[i] = __ballot_sync(kFull, (g_rep[lane] >> i) & 1u);
  } else {
    // full sweep: the last field's low 5 bits count the states, the rest is
    // the group's value; with no extra register the carry is bit 0
    uint32_t v = 0u;
    switch (rlast) {
      case 0: v = x.b; break;
      case 1: v = x.c; break;
      case 2: v = x.d; break;
      case 3: v = x.e; break;
      case 4: v = x.h; break;
      case 5: v = x.l; break;
      case 6: v = x.m; break;
      default: break;
    }
    vp[0] = 0xAAAAAAAAu;
    vp[1] = 0xCCCCCCCCu;
    vp[2] = 0xF0F0F0F0u;
    vp[3] = 0xFF00FF00u;
    vp[4] = 0xFFFF0000u;
#pragma unroll
    for (int i = 5; i < 8; i++) vp[i] = ((v >> i) & 1u) ? kZBOnes : 0u;
    fp0 = 0xAAAAAAAAu;
  }
  ZB z;
  bool bad = false;
#pragma unroll 1
  for (uint32_t abit = 0; abit < 2u; abit++) {
    auto init = [&]() {
      zb_set8(z.a, abit);
      zb_set8(z.f, x.f);
      zb_set8(z.b, x.b);
      zb_set8(z.c, x.c);
      zb_set8(z.d, x.d);
      zb_set8(z.e, x.e);
      zb_set8(z.h, x.h);
      zb_set8(z.l, x.l);
      zb_set8(z.m, x.m);
#pragma unroll
      for (int i = 0; i < 16; i++) z.sp[i] = spw ? spp[i] : (((x.sp >> i) & 1u) ? kZBOnes : 0u);
      if (nx >= 1) zb_set_reg(z, rlast, vp);
      else z.f[0] = fp0;
    };
    init();
#pragma unroll 1
    for (int st = 0; st < tl + cl; st++) {
      if (st == cl) {
        zb_save(z, sm);
        init();
      }
      const int src = st < cl ? tl + st : st - cl;
      const uint32_t w = __shfl_sync(kFull, pw, src);
      zb_step(z, w & 0xFFFFu, w >> 16);
    }
    bad = bad || (zb_diff(z, sm, keepF, keepR) & valid) != 0u;
  }
  return bad;
}

// One unit of a compact A-independent sweep: xbits_unit's layout (lane l:
// the 32 A-blocks u*1024 + 32l .. +31 as one state word, at A = 0 then
// A = 1) on the A/F/B/C state with renamed programs.  A compact pair reads
// neither SP nor more than two registers, so its sweep is a full one over
// at most two fields, and the field the low 5 block bits move is the last
// swept register, now B (o0) or C (o1), or with no swept register the carry.
__device__ __forceinline__ bool cxbits_unit(unsigned long long u, unsigned long long nblocks, int nx, const CDec& dec,
                                            int rlast, uint32_t pw, int tl, int cl, uint32_t keepF, uint32_t keepR,
                                            int o0, int o1, uint32_t* sm) {
  const unsigned lane = lane_id();
  const unsigned long long g0 = u * kXBitsBlocks + (unsigned long long)lane * 32ull;
  const uint32_t valid = g0 >= nblocks ? 0u
                         : (nblocks - g0 >= 32ull ? 0xFFFFFFFFu : ((1u << uint32_t(nblocks - g0)) - 1u));
  uint32_t vb, vc, carry;
  cdec_vals(dec, g0 < nblocks ? g0 : 0ull, vb, vc, carry);
  // the moving field's planes: state j has j in its low 5 bits, the group's
  // value above them
  const uint32_t v = rlast == o0 ? vb : vc;
  uint32_t vp[8];
  vp[0] = 0xAAAAAAAAu;
  vp[1] = 0xCCCCCCCCu;
  vp[2] = 0xF0F0F0F0u;
  vp[3] = 0xFF00FF00u;
  vp[4] = 0xFFFF0000u;
#pragma unroll
  for (int i = 5; i < 8; i++) vp[i] = ((v >> i) & 1u) ? kZBOnes : 0u;
  ZB4 z;
  bool bad = false;
#pragma unroll 1
  for (uint32_t abit = 0; abit < 2u; abit++) {
    auto init = [&]() {
      zb_set8(z.a, abit);
      zb_set8(z.f, carry);
      zb_set8(z.b, vb);
      zb_set8(z.c, vc);
      if (nx == 0) z.f[0] = 0xAAAAAAAAu;
      else if (rlast == o0) zb_copy8(z.b, vp);
      else zb_copy8(z.c, vp);
    };
    init();
#pragma unroll 1
    for (int st = 0; st < tl + cl; st++) {
      if (st == cl) {
#pragma unroll
        for (int i = 0; i < 8; i++) {
          sm[(0 + i) * 32] = z.a[i];
          sm[(8 + i) * 32] = z.f[i];
          sm[(16 + i) * 32] = z.b[i];
          sm[(24 + i) * 32] = z.c[i];
        }
        init();
      }
      const int src = st < cl ? tl + st : st - cl;
      const uint32_t w = __shfl_sync(kFull, pw, src);
      zb4_step(z, w & 0xFFFFu, w >> 16);
    }
    const bool cmp_b = o0 >= 0 && ((keepR >> o0) & 1u), cmp_c = o1 >= 0 && ((keepR >> o1) & 1u);
    uint32_t d = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      d |= z.a[i] ^ sm[(0 + i) * 32];
      if ((keepF >> i) & 1u) d |= z.f[i] ^ sm[(8 + i) * 32];
      if (cmp_b) d |= z.b[i] ^ sm[(16 + i) * 32];
      if (cmp_c) d |= z.c[i] ^ sm[(24 + i) * 32];
    }
    bad = bad || (d & valid) != 0u;
  }
  return bad;
}

// Wide compact sweeps (A-dependent pairs): the layout of bits_unit on the
// wide state (A, F, B, C, H, L, M; ZBW) with renamed programs.  Fields 0..3 are
// B, C, H, L (standing for the registers the pair's set puts there), field
// 4 is M; cmp bit s: field s is compared (it stands for a register under
// keepR).  A and M are always compared, F under keepF.
constexpr int kWideWords = 56;  // planes saved per lane
__device__ __forceinline__ void zbw_init(ZBW& z, const uint32_t (&v)[5], uint32_t carry) {
  zb_set8(z.f, carry);
  zb_set8(z.b, v[0]);
  zb_set8(z.c, v[1]);
  zb_set8(z.h, v[2]);
  zb_set8(z.l, v[3]);
  zb_set8(z.m, v[4]);
}
__device__ __forceinline__ void zbw_save(const ZBW& z, uint32_t* s) {
#pragma unroll
  for (int i = 0; i < 8; i++) {
    s[(0 + i) * 32] = z.a[i];
    s[(8 + i) * 32] = z.f[i];
    s[(16 + i) * 32] = z.b[i];
    s[(24 + i) * 32] = z.c[i];
    s[(32 + i) * 32] = z.h[i];
    s[(40 + i) * 32] = z.l[i];
    s[(48 + i) * 32] = z.m[i];
  }
}
__device__ __forceinline__ uint32_t zbw_diff(const ZBW& z, const uint32_t* s, uint32_t keepF, uint32_t cmp) {
  uint32_t d = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    d |= z.a[i] ^ s[(0 + i) * 32];
    if ((keepF >> i) & 1u) d |= z.f[i] ^ s[(8 + i) * 32];
    if (cmp & 1u) d |= z.b[i] ^ s[(16 + i) * 32];
    if (cmp & 2u) d |= z.c[i] ^ s[(24 + i) * 32];
    if (cmp & 4u) d |= z.h[i] ^ s[(32 + i) * 32];
    if (cmp & 8u) d |= z.l[i] ^ s[(40 + i) * 32];
    d |= z.m[i] ^ s[(48 + i) * 32];
  }
  return d;
}
// A-dependent: lane l takes block 4u + l/8 and A = 32(l % 8) .. +31.
__device__ __forceinline__ bool wbits_unit(unsigned long long u, unsigned long long nblocks, const WDec& dec,
                                           uint32_t pw, int tl, int cl, uint32_t keepF, uint32_t cmp, uint32_t* sm) {
  const unsigned lane = lane_id();
  const unsigned long long blk = u * kBitsBlocks + (lane >> 3);
  const bool valid = blk < nblocks;
  uint32_t v[5], carry;
  wdec_vals(dec, uint32_t(valid ? blk : u * kBitsBlocks), g_rep, v, carry);
  const uint32_t a0 = (lane & 7u) * 32u;
  ZBW z;
  auto init = [&]() {
    z.a[0] = 0xAAAAAAAAu;
    z.a[1] = 0xCCCCCCCCu;
    z.a[2] = 0xF0F0F0F0u;
    z.a[3] = 0xFF00FF00u;
    z.a[4] = 0xFFFF0000u;
    z.a[5] = (a0 & 32u) ? kZBOnes : 0u;
    z.a[6] = (a0 & 64u) ? kZBOnes : 0u;
    z.a[7] = (a0 & 128u) ? kZBOnes : 0u;
    zbw_init(z, v, carry);
  };
  init();
#pragma unroll 1
  for (int st = 0; st < tl + cl; st++) {
    if (st == cl) {
      zbw_save(z, sm);
      init();
    }
    const int src = st < cl ? tl + st : st - cl;
    const uint32_t w = __shfl_sync(kFull, pw, src);
    zbw_step(z, w & 0xFFFFu, w >> 16);
  }
  return valid && zbw_diff(z, sm, keepF, cmp) != 0u;
}
// Register-state sweeps (pairs naming neither SP nor the memory byte that
// no compact state takes): the layouts of bits_unit (A-dependent pairs) and
// xbits_unit (A-independent ones) on ZB6 (A, F, B..L), no renaming.
constexpr int kRegWords = 64;  // planes saved per lane
__device__ __forceinline__ void zb6_init(ZB6& z, const Z80S& x) {
  zb_set8(z.f, x.f);
  zb_set8(z.b, x.b);
  zb_set8(z.c, x.c);
  zb_set8(z.d, x.d);
  zb_set8(z.e, x.e);
  zb_set8(z.h, x.h);
  zb_set8(z.l, x.l);
}
__device__ __forceinline__ void zb6_save(const ZB6& z, uint32_t* s) {
#pragma unroll
  for (int i = 0; i < 8; i++) {
    s[(0 + i) * 32] = z.a[i];
    s[(8 + i) * 32] = z.f[i];
    s[(16 + i) * 32] = z.b[i];
    s[(24 + i) * 32] = z.c[i];
    s[(32 + i) * 32] = z.d[i];
    s[(40 + i) * 32] = z.e[i];
    s[(48 + i) * 32] = z.h[i];
    s[(56 + i) * 32] = z.l[i];
  }
}
__device__ __forceinline__ uint32_t zb6_diff(const ZB6& z, const uint32_t* s, uint32_t keepF, uint32_t keepR) {
  uint32_t d = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    d |= z.a[i] ^ s[(0 + i) * 32];
    if ((keepF >> i) & 1u) d |= z.f[i] ^ s[(8 + i) * 32];
    if (keepR & 1u) d |= z.b[i] ^ s[(16 + i) * 32];
    if (keepR & 2u) d |= z.c[i] ^ s[(24 + i) * 32];
    if (keepR & 4u) d |= z.d[i] ^ s[(32 + i) * 32];
    if (keepR & 8u) d |= z.e[i] ^ s[(40 + i) * 32];
    if (keepR & 16u) d |= z.h[i] ^ s[(48 + i) * 32];
    if (keepR & 32u) d |= z.l[i] ^ s[(56 + i) * 32];
  }
  return d;
}
// A-dependent: lane l takes block 4u + l/8 and A = 32(l % 8) .. +31.
__device__ __forceinline__ bool rbits_unit(unsigned long long u, unsigned long long nblocks, const BDec& bd,
                                           uint32_t pw, int tl, int cl, uint32_t keepF, uint32_t keepR, uint32_t* sm) {
  const unsigned lane = lane_id();
  const unsigned long long blk = u * kBitsBlocks + (lane >> 3);
  const bool valid = blk < nblocks;
  const Z80S x = bdec_state(bd, valid ? blk : u * kBitsBlocks, g_rep, g_repsp);
  const uint32_t a0 = (lane & 7u) * 32u;
  ZB6 z;
  auto init = [&]() {
    z.a[0] = 0xAAAAAAAAu;
    z.a[1] = 0xCCCCCCCCu;
    z.a[2] = 0xF0F0F0F0u;
    z.a[3] = 0xFF00FF00u;
    z.a[4] = 0xFFFF0000u;
    z.a[5] = (a0 & 32u) ? kZBOnes : 0u;
    z.a[6] = (a0 & 64u) ? kZBOnes : 0u;
    z.a[7] = (a0 & 128u) ? kZBOnes : 0u;
    zb6_init(z, x);
  };
  init();
#pragma unroll 1
  for (int st = 0; st < tl + cl; st++) {
    if (st == cl) {
      zb6_save(z, sm);
      init();
    }
    const int src = st < cl ? tl + st : st - cl;
    const uint32_t w = __shfl_sync(kFull, pw, src);
    zb6_step(z, w & 0xFFFFu, w >> 16);
  }
  return valid && zb6_diff(z, sm, keepF, keepR) != 0u;
}
// A-independent: lane l takes the 32 A-blocks u*1024 + 32l .. +31 as one
// state word, at A = 0 and then A = 1; the low 5 bits of the block index
// move the last swept register rlast (its low 5 bits in a full sweep, its
// 32 representative values in a reduced one) or, with none, the carry.
__device__ __forceinline__ void zb6_set_reg(ZB6& z, int r, const uint32_t (&pl)[8]) {
  switch (r) {
    case 0: zb_copy8(z.b, pl); break;
    case 1: zb_copy8(z.c, pl); break;
    case 2: zb_copy8(z.d, pl); break;
    case 3: zb_copy8(z.e, pl); break;
    case 4: zb_copy8(z.h, pl); break;
    case 5: zb_copy8(z.l, pl); break;
    default: break;
  }
}
__device__ __forceinline__ bool rxbits_unit(unsigned long long u, unsigned long long nblocks, bool reduced, int nx,
                                            int rlast, const BDec& bd, uint32_t pw, int tl, int cl, uint32_t keepF,
                                            uint32_t keepR, uint32_t* sm) {
  const unsigned lane = lane_id();
  const unsigned long long g0 = u * kXBitsBlocks + (unsigned long long)lane * 32ull;
  const uint32_t valid = g0 >= nblocks ? 0u
                         : (nblocks - g0 >= 32ull ? 0xFFFFFFFFu : ((1u << uint32_t(nblocks - g0)) - 1u));
  const Z80S x = bdec_state(bd, g0 < nblocks ? g0 : 0ull, g_rep, g_repsp);
  uint32_t vp[8];
  if (reduced) {
#pragma unroll
    for (int i = 0; i < 8; i++) vp[i] = __ballot_sync(kFull, (g_rep[lane] >> i) & 1u);
  } else {
    uint32_t v = 0u;
    switch (rlast) {
      case 0: v = x.b; break;
      case 1: v = x.c; break;
      case 2: v = x.d; break;
      case 3: v = x.e; break;
      case 4: v = x.h; break;
      case 5: v = x.l; break;
      default: break;
    }
    vp[0] = 0xAAAAAAAAu;
    vp[1] = 0xCCCCCCCCu;
    vp[2] = 0xF0F0F0F0u;
    vp[3] = 0xFF00FF00u;
    vp[4] = 0xFFFF0000u;
#pragma unroll
    for (int i = 5; i < 8; i++) vp[i] = ((v >> i) & 1u) ? kZBOnes : 0u;
  }
  ZB6 z;
  bool bad = false;
#pragma unroll 1
  for (uint32_t abit = 0; abit < 2u; abit++) {
    auto init = [&]() {
      zb_set8(z.a, abit);
      zb6_init(z, x);
      if (nx >= 1) zb6_set_reg(z, rlast, vp);
      else z.f[0] = 0xAAAAAAAAu;
    };
    init();
#pragma unroll 1
    for (int st = 0; st < tl + cl; st++) {
      if (st == cl) {
        zb6_save(z, sm);
        init();
      }
      const int src = st < cl ? tl + st : st - cl;
      const uint32_t w = __shfl_sync(kFull, pw, src);
      zb6_step(z, w & 0xFFFFu, w >> 16);
    }
    bad = bad || (zb6_diff(z, sm, keepF, keepR) & valid) != 0u;
  }
  return bad;
}

// One unit (128 A-blocks at A = 0, 1) of an A-independent sweep, for the
// A-independent sweep kernel; kept out of line (that kernel compiles without
// register spills at every K this way).
template <int K>
__device__ __noinline__ bool xindep_unit(unsigned long long first, unsigned long long nb, const BDec bd, uint32_t pw,
                                         int tl, int cl, uint32_t keep0, uint32_t keep1) {
  const unsigned lane = lane_id();
  bool bad = false;
#pragma unroll 1
  for (uint32_t i = 0; i < 8u / K; i++) {
    uint32_t W[K][3];  // initial states, packed
    bool valid[K];
#pragma unroll
    for (int q = 0; q < K; q++) {
      const uint32_t sl = (i * K + q) * 32u + lane;
      valid[q] = (sl >> 1) < nb;
      Z80S x = bdec_state(bd, valid[q] ? first + (sl >> 1) : first, g_rep, g_repsp);
      x.a = sl & 1u;
      z_pack(x, W[q]);
    }
    auto init = [&](int q, Z80S& x) { x = z_unpack(W[q][0], W[q][1], W[q][2]); };
    bad = run_compare<K>(init, valid, pw, tl, cl, keep0, keep1) || bad;
  }
  return bad;
}

// One kernel per pair class: CLS 0 runs the bit-sliced pairs (outputs
// depend on A), CLS 1 the A-independent ones (K states per lane per
// dispatch), CLS 2 the A-independent ones bit-sliced, CLS 3 the pairs whose
// registers fit the compact state (three blocks per SM), CLS 4 the
// A-dependent ones that fit the wide compact state (two blocks per SM), CLS
// 5 the rest that name neither SP nor the memory byte, on A, F and B..L; each class
// draws chunks from its own numbering and dispenser.  Kept apart so that
// neither path's registers weigh on the other.
// dev_total / dev_np (device-driven rounds): the class's chunk total and the
// round's pair count are read from the device instead of total / npairs.
// chunks_per_warp: chunks a warp takes before its block retires.
#ifndef Z80B_REG_BLOCKS
#define Z80B_REG_BLOCKS 2
#endif
// The pair whose chunk range holds chunk k: the last p with cbase[p] <= k
// (cbase ascending from cbase[0] = 0; pairs without chunks in the class
// repeat their successor's base).  Warp-wide, k the same in every lane: each
// step the 32 lanes probe 32 evenly spaced pairs of the range left and a
// ballot keeps the span after the last probe that is <= k, so a round of n
// pairs takes ceil(log32 n) dependent loads instead of log2 n.
__device__ __forceinline__ uint32_t chunk_pair(const unsigned long long* __restrict__ cbase, uint32_t npairs,
                                               unsigned long long k, unsigned lane) {
  uint32_t lo = 0, n = npairs;  // the answer lies in [lo, lo + n); cbase[lo] <= k
  while (n > 1) {
    const uint32_t step = (n + 31u) / 32u;
    const uint32_t off = lane * step;
    const bool le = off < n && cbase[lo + off] <= k;
    const unsigned b = __ballot_sync(kFull, le);  // a prefix of the lanes, lane 0 always
    const uint32_t last = 31u - uint32_t(__clz(b));
    lo += last * step;
    n = min(step, n - last * step);
  }
  return lo;
}
template <int K, int CLS>
__global__ void __launch_bounds__(kBlock, CLS == 3 ? 3 : (CLS == 4 ? 2 : (CLS == 5 ? Z80B_REG_BLOCKS : 1)))
    k_exhaustive(DevTargets T, DevPool P, RoundBuf R, uint32_t npairs, unsigned long long total,
                 const unsigned long long* __restrict__ dev_total, const uint32_t* __restrict__ dev_np,
                 int chunks_per_warp) {
  static_assert(K == 1 || K == 2 || K == 4 || K == 8, "K divides 8");
  if (dev_total) {
    total = *dev_total;
    npairs = *dev_np;
  }
  constexpr bool XI = CLS != 0;
  const unsigned long long* __restrict__ cbase =
      CLS == 5 ? R.cbase_r : (CLS == 4 ? R.cbase_w : (CLS == 3 ? R.cbase_c : (XI ? R.cbase_x : R.cbase)));
  const unsigned lane = lane_id();
  unsigned long long my_states = 0, my_eval = 0;
  // At most kChunksPerWarp chunks per warp, then the block retires: the grid
  // covers all chunks, and blocks of kernels on other streams (with a higher
  // priority) get SMs as soon as blocks of a long sweep retire.
  for (int taken = 0; taken < chunks_per_warp; taken++) {
    unsigned long long k = 0;
    if (lane == 0) k = atomicAdd(R.counter + (CLS >= 3 ? CLS - 1 : (XI ? 1 : 0)), 1ull);
    k = __shfl_sync(kFull, k, 0);
    if (k >= total) break;
    // pair p: cbase[p] <= k < cbase[p + 1]
    const uint32_t p = chunk_pair(cbase, npairs, k, lane);
    // lane 0 reads the flag and the warp acts on one value, so the
    // shuffles below always see all 32 lanes
    if (__shfl_sync(kFull, lane == 0 ? *reinterpret_cast<volatile uint32_t*>(&R.rejected[p]) : 0u, 0))
      continue;
    const PairRec pr = R.pairs[p];
    const unsigned long long nunits = pair_units(pr.nblocks, pr.keepR, R.xunit);
    const unsigned long long nch = (p + 1 < npairs ? cbase[p + 1] : total) - cbase[p];
    const unsigned long long upc = (nunits + nch - 1) / nch;
    const unsigned long long j = k - cbase[p];
    const unsigned long long u0 = j * upc;
    unsigned long long u1 = u0 + upc;
    if (u1 > nunits) u1 = nunits;

    // programs: lanes 0..tl-1 target, tl..tl+cl-1 candidate
    const uint32_t tl = target_len(T, pr.target), cl = pool_len(P, pr.cand);
    uint32_t pw = 0;
    if (lane < tl) pw = T.insn[(size_t)pr.target * T.stride + lane];
    else if (lane < tl + cl) pw = P.insn[(size_t)pr.cand * P.stride + (lane - tl)];

    // sweep shape (verifier.go:428-476): extra registers in B,C,D,E,H,L,M order
    const uint32_t ext = pr.reads & (kRegB | kRegC | kRegD | kRegE | kRegH | kRegL | kRegM);
    const int nx = __popc(ext);
    const bool spw = (pr.reads & kRegSP) != 0;
    const bool reduced = spw || nx > 2 || (pr.sweepf & 0x80u) != 0;
    const uint32_t xs = pr.sweepf & 0x3Fu;  // reference states per evaluated state, log2
    const int fw = reduced ? 5 : 8;  // bits per swept register in the block index
    int slot[7];
    {
      int k2 = 0;
      const uint32_t bits[7] = {kRegB, kRegC, kRegD, kRegE, kRegH, kRegL, kRegM};
#pragma unroll
      for (int r = 0; r < 7; r++) slot[r] = (ext & bits[r]) ? k2++ : -1;
    }
    const BDec bd = bdec_make(spw, reduced, nx, fw, slot);
    // compared bytes of the packed words (A F B C / D E H L / SP M)
    const uint32_t keep0 = 0xFFu | (uint32_t(pr.keepF) << 8) | ((pr.keepR & 1u) ? 0xFF0000u : 0u) |
                           ((pr.keepR & 2u) ? 0xFF000000u : 0u);
    const uint32_t keep1 = ((pr.keepR & 4u) ? 0xFFu : 0u) | ((pr.keepR & 8u) ? 0xFF00u : 0u) |
                           ((pr.keepR & 16u) ? 0xFF0000u : 0u) | ((pr.keepR & 32u) ? 0xFF000000u : 0u);

    bool bad = false;
    bool stopped = false;  // left the loop on the pair's flag (rejected or cancelled elsewhere)
    if constexpr (CLS == 5) {
      // the register state (A, F, B..L), programs as they are
      extern __shared__ uint32_t zsm[];
      uint32_t* sm = zsm + (threadIdx.x >> 5) * (kRegWords * 32) + lane;
      if (pr.keepR & kXIndep) {
        int rlast = -1;  // the register of the last swept field (the fastest)
#pragma unroll
        for (int r = 0; r < 6; r++)
          if (slot[r] == nx - 1) rlast = r;
        for (unsigned long long u = u0; u < u1; u++) {
          const unsigned long long first = u * kXBitsBlocks;
          const unsigned long long nb = (pr.nblocks - first < kXBitsBlocks) ? pr.nblocks - first : kXBitsBlocks;
          bad = rxbits_unit(u, pr.nblocks, reduced, nx, rlast, bd, pw, int(tl), int(cl), pr.keepF, pr.keepR, sm) ||
                bad;
          my_states += (256ull * nb) << xs;
          my_eval += 2ull * nb;
          if (__any_sync(kFull, bad)) break;
          if (__shfl_sync(kFull, lane == 0 ? *reinterpret_cast<volatile uint32_t*>(&R.rejected[p]) : 0u, 0)) {
            stopped = true;
            break;
          }
        }
      } else {
        for (unsigned long long u = u0; u < u1; u++) {
          const unsigned long long first = u * kBitsBlocks;
          const unsigned long long nb = (pr.nblocks - first < kBitsBlocks) ? pr.nblocks - first : kBitsBlocks;
          bad = rbits_unit(u, pr.nblocks, bd, pw, int(tl), int(cl), pr.keepF, pr.keepR, sm) || bad;
          my_states += (256ull * nb) << xs;
          my_eval += 256ull * nb;
          if (__any_sync(kFull, bad)) break;
          if ((u & 15ull) == 15ull &&
              __shfl_sync(kFull, lane == 0 ? *reinterpret_cast<volatile uint32_t*>(&R.rejected[p]) : 0u, 0)) {
            stopped = true;
            break;
          }
        }
      }
    } else if constexpr (CLS == 4) {
      // the wide compact state, the programs renamed onto B, C, H and L
      const uint32_t e = (pr.cmap & ~uint32_t(kWideClass)) - 1u;
      if (lane < tl + cl) pw = (uint32_t(uint16_t(g_wren[e][pw & 0xFFFFu]))) | (pw & 0xFFFF0000u);
      int o[4];
      uint32_t cmp = 0;
#pragma unroll
      for (int f = 0; f < 4; f++) {
        o[f] = g_worig[e][f];
        if (o[f] >= 0 && ((pr.keepR >> o[f]) & 1u)) cmp |= 1u << f;
      }
      extern __shared__ uint32_t zsm[];
      uint32_t* sm = zsm + (threadIdx.x >> 5) * (kWideWords * 32) + lane;
      const WDec dec = wdec_make(nx, reduced, slot, o);
      for (unsigned long long u = u0; u < u1; u++) {
        const unsigned long long first = u * kBitsBlocks;
        const unsigned long long nb = (pr.nblocks - first < kBitsBlocks) ? pr.nblocks - first : kBitsBlocks;
        bad = wbits_unit(u, pr.nblocks, dec, pw, int(tl), int(cl), pr.keepF, cmp, sm) || bad;
        my_states += (256ull * nb) << xs;
        my_eval += 256ull * nb;
        if (__any_sync(kFull, bad)) break;
        if ((u & 15ull) == 15ull &&
            __shfl_sync(kFull, lane == 0 ? *reinterpret_cast<volatile uint32_t*>(&R.rejected[p]) : 0u, 0)) {
          stopped = true;
          break;
        }
      }
    } else if constexpr (CLS == 3) {
      // the compact state, the programs renamed onto B and C
      const uint32_t e = pr.cmap - 1u;
      if (lane < tl + cl) pw = (uint32_t(uint16_t(g_cren[e][pw & 0xFFFFu]))) | (pw & 0xFFFF0000u);
      const int o0 = g_corig[e][0], o1 = g_corig[e][1];
      extern __shared__ uint32_t zsm[];
      uint32_t* sm = zsm + (threadIdx.x >> 5) * (kCompactWords * 32) + lane;
      const CDec dec = cdec_make(nx, slot, o0, o1);
      if (pr.keepR & kXIndep) {
        // A-independent: units of 1,024 A-blocks, each at A = 0 and 1
        int rlast = -1;
#pragma unroll
        for (int r = 0; r < 7; r++)
          if (slot[r] == nx - 1) rlast = r;
        for (unsigned long long u = u0; u < u1; u++) {
          const unsigned long long first = u * kXBitsBlocks;
          const unsigned long long nb = (pr.nblocks - first < kXBitsBlocks) ? pr.nblocks - first : kXBitsBlocks;
          bad = cxbits_unit(u, pr.nblocks, nx, dec, rlast, pw, int(tl), int(cl), pr.keepF, pr.keepR, o0, o1, sm) ||
                bad;
          my_states += (256ull * nb) << xs;
          my_eval += 2ull * nb;
          if (__any_sync(kFull, bad)) break;
          if (__shfl_sync(kFull, lane == 0 ? *reinterpret_cast<volatile uint32_t*>(&R.rejected[p]) : 0u, 0)) {
          stopped = true;
          break;
        }
        }
      } else {
        for (unsigned long long u = u0; u < u1; u++) {
          const unsigned long long first = u * kBitsBlocks;
          const unsigned long long nb = (pr.nblocks - first < kBitsBlocks) ? pr.nblocks - first : kBitsBlocks;
          bad = cbits_unit(u, pr.nblocks, dec, pw, int(tl), int(cl), pr.keepF, pr.keepR, o0, o1, sm) || bad;
          my_states += (256ull * nb) << xs;
          my_eval += 256ull * nb;
          if (__any_sync(kFull, bad)) break;
          if ((u & 15ull) == 15ull &&
              __shfl_sync(kFull, lane == 0 ? *reinterpret_cast<volatile uint32_t*>(&R.rejected[p]) : 0u, 0))
            {
              stopped = true;
              break;
            }
        }
      }
    } else if constexpr (!XI) {
      // Unit = 4 A-blocks, bit-sliced (256 states of each block in 8 lanes).
      // The reference nests its loops as A, carry, first register, ...,
      // last register, SP (verifier.go:498-531,578-610); the block index
      // varies SP and the last register fastest, so a sweep the reference
      // abandons early is abandoned early here too.
      extern __shared__ uint32_t zsm[];
      uint32_t* sm = zsm + (threadIdx.x >> 5) * (kBitsWords * 32) + lane;
      for (unsigned long long u = u0; u < u1; u++) {
        const unsigned long long first = u * kBitsBlocks;
        const unsigned long long nb = (pr.nblocks - first < kBitsBlocks) ? pr.nblocks - first : kBitsBlocks;
        bad = bits_unit(u, pr.nblocks, bd, pw, int(tl), int(cl), pr.keepF, pr.keepR, sm) || bad;
        my_states += (256ull * nb) << xs;
        my_eval += 256ull * nb;
        if (__any_sync(kFull, bad)) break;
        if ((u & 15ull) == 15ull &&
            __shfl_sync(kFull, lane == 0 ? *reinterpret_cast<volatile uint32_t*>(&R.rejected[p]) : 0u, 0))
          {
            stopped = true;
            break;
          }
      }
    } else if constexpr (CLS == 2) {
      // Unit = 1,024 A-blocks, 32 per lane, each at A = 0 and A = 1.
      extern __shared__ uint32_t zsm[];
      uint32_t* sm = zsm + (threadIdx.x >> 5) * (kBitsWords * 32) + lane;
      int rlast = -1;  // the register of the last swept field (the fastest)
#pragma unroll
      for (int r = 0; r < 7; r++)
        if (slot[r] == nx - 1) rlast = r;
      for (unsigned long long u = u0; u < u1; u++) {
        const unsigned long long first = u * kXBitsBlocks;
        const unsigned long long nb = (pr.nblocks - first < kXBitsBlocks) ? pr.nblocks - first : kXBitsBlocks;
        bad = xbits_unit(u, pr.nblocks, spw, reduced, nx, fw, slot, rlast, pw, int(tl), int(cl), pr.keepF,
                         pr.keepR, sm) ||
              bad;
        my_states += (256ull * nb) << xs;
        my_eval += 2ull * nb;
        if (__any_sync(kFull, bad)) break;
        if (__shfl_sync(kFull, lane == 0 ? *reinterpret_cast<volatile uint32_t*>(&R.rejected[p]) : 0u, 0)) {
          stopped = true;
          break;
        }
      }
    } else {
      // Unit = 128 A-blocks, each evaluated at A = 0 and A = 1: state slot s
      // of the warp (s = (i*K + q)*32 + lane) takes block unit*128 + s/2 with
      // A = s & 1.
      for (unsigned long long u = u0; u < u1; u++) {
        const unsigned long long first = u * kUnitBlocks;
        const unsigned long long nb = (pr.nblocks - first < kUnitBlocks) ? pr.nblocks - first : kUnitBlocks;
        bad = xindep_unit<K>(first, nb, bd, pw, int(tl), int(cl), keep0, keep1) || bad;
        my_states += (256ull * nb) << xs;
        my_eval += 2ull * nb;
        if (__any_sync(kFull, bad)) break;
        if ((u & 3ull) == 3ull &&
            __shfl_sync(kFull, lane == 0 ? *reinterpret_cast<volatile uint32_t*>(&R.rejected[p]) : 0u, 0))
          {
            stopped = true;
            break;
          }
      }
    }
    const bool any_bad = __any_sync(kFull, bad);
    if (lane == 0) {
      if (any_bad) atomicExch(&R.rejected[p], 1u);
      else if (!stopped && R.wend)
        chunk_passed(R.rejected, R.wend, R.cdone, p,
                     uint32_t((p + 1 < npairs ? cbase[p + 1] : total) - cbase[p]));
    }
  }
  if (lane == 0 && my_states) {
    atomicAdd(R.states, my_states);
    atomicAdd(R.states + 1, my_eval);
  }
}
// Window heads settle their lane: the first pair of the window that passed
// wins; if none did, the lane moves past the window and the next window
// doubles (up to 2^max_spec).
__global__ void k_round_resolve(RoundBuf R, uint32_t npairs, QCOut q, Lanes L, uint32_t max_spec,
                                const uint32_t* __restrict__ dev_np) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (dev_np) npairs = *dev_np;
  if (p >= npairs) return;
  const uint32_t w = R.wlen[p];
  if (w == 0) return;
  const PairRec pr = R.pairs[p];
  const uint32_t idx = 2 * pr.target + ((pr.keepR & 0x80u) ? 1u : 0u);
  for (uint32_t j = 0; j < w; j++) {
    if (R.rejected[p + j] == 0) {
      L.win[idx] = R.pairs[p + j].cand;
      L.windiff[idx] = q.sdiff[R.pair_src[p + j]];
      L.next[idx] = (L.next[idx] + j) | kResolved;
      return;
    }
  }
  L.next[idx] += w;
  if (L.spec[idx] < max_spec) L.spec[idx] += 1;
}

__global__ void k_midcheck(DevTargets T, DevPool P, const uint32_t* __restrict__ surv,
                           const uint32_t* __restrict__ surv_target, uint32_t nsurv, uint8_t* __restrict__ pass) {
  const unsigned lane = lane_id();
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = gw; i < nsurv; i += nw) {
    const uint32_t t = surv_target[i], c = surv[i];
    const uint32_t tl = target_len(T, t), cl = pool_len(P, c);
    uint32_t pw = 0;
    if (lane < tl) pw = T.insn[(size_t)t * T.stride + lane];
    else if (lane < tl + cl) pw = P.insn[(size_t)c * P.stride + (lane - tl)];
    Z80S x = vec_state(int(lane)), y = x;
    run_lanes(x, pw, 0, int(tl));
    run_lanes(y, pw, int(tl), int(cl));
    const Keep keep = make_keep(~target_dead(T, t), ~target_dead_regs(T, t) & 0x3Fu, true);
    bool ok = __all_sync(kFull, eq_keep(x, y, keep));
    if (lane == 0) pass[i] = ok ? 1 : 0;
  }
}

__global__ void k_surv_targets(QCOut q, uint32_t n, uint32_t* __restrict__ st) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  uint32_t b = q.base[t], c = q.cnt_f[t] + q.cnt_m[t];
  for (uint32_t j = 0; j < c; j++) st[b + j] = t;
}

__global__ void k_rule_count_first(Lanes L, Lanes L2, uint32_t n, uint32_t* __restrict__ cnt, DevTargets T,
                                   unsigned long long* checked, uint32_t pool_enum,
                                   unsigned long long pool2_enum) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long ch = 0;
  if (t < n) {
    uint32_t c = 0;
    const bool masked = target_dead(T, t) != 0 || target_dead_regs(T, t) != 0;
    for (int kind = 0; kind < 2; kind++) {
      const uint32_t w1 = L.win[2 * t + kind];
      const uint32_t w2 = L2.win ? L2.win[2 * t + kind] : kNone;
      c += (w1 != kNone || w2 != kNone) ? 1u : 0u;
      // worker.go:134 counts every enumerated candidate up to and including
      // the winner (the pool index is the enumeration ordinal): all of the
      // shorter lengths, then the winner's own length
      if (kind == 0 || masked) {
        if (w1 != kNone) ch += (unsigned long long)w1 + 1ull;
        else if (L2.win) ch += pool_enum + ((w2 != kNone) ? (unsigned long long)w2 + 1ull : pool2_enum);
        else ch += pool_enum;
      }
    }
    cnt[t] = c;
  }
  for (int off = 16; off; off >>= 1) ch += __shfl_down_sync(kFull, ch, off);
  if (lane_id() == 0 && ch) atomicAdd(checked, ch);
}
__global__ void k_rule_write_first(Lanes L, Lanes L2, uint32_t n, const uint32_t* __restrict__ base,
                                   DevRule* __restrict__ out) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  uint32_t b = base[t];
  for (int kind = 0; kind < 2; kind++) {
    const uint32_t idx = 2 * t + kind;
    const uint32_t w1 = L.win[idx];
    const uint32_t w2 = L2.win ? L2.win[idx] : kNone;
    if (w1 == kNone && w2 == kNone) continue;
    DevRule r;
    r.target = t;
    r.cand = w1 != kNone ? w1 : w2;
    r.diff = kind ? (w1 != kNone ? L.windiff[idx] : L2.windiff[idx]) : uint16_t(0);
    r.kind = uint8_t(kind);
    r.clen = w1 != kNone ? 1 : 2;
    out[b++] = r;
  }
}

// All-hits: flag[i] = 1 when survivor i passed MidCheck and ExhaustiveCheck.
__global__ void k_rule_count_all(RoundBuf R, uint32_t npairs, uint32_t* __restrict__ flag) {
  uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npairs) return;
  if (R.rejected[p] == 0) flag[R.pair_src[p]] = 1u;
}

__global__ void k_rule_write_all(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ base,
                                 uint32_t nsurv, const uint32_t* __restrict__ surv,
                                 const uint16_t* __restrict__ sdiff, const uint32_t* __restrict__ surv_target,
                                 DevRule* __restrict__ out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsurv || !flag[i]) return;
  DevRule r;
  r.target = surv_target[i];
  r.cand = surv[i];
  r.diff = sdiff[i];
  r.kind = 2;
  r.clen = 1;
  out[base[i]] = r;
}

// Verifier tiers for explicit pairs (QuickCheck, MidCheck, FlagDiff); warp
// per pair, lane v = vector v.
__global__ void k_verify_small(const uint32_t* __restrict__ tgt, const uint8_t* __restrict__ tlens,
                               const uint32_t* __restrict__ cand, const uint8_t* __restrict__ clens,
                               uint32_t stride, uint32_t n, const uint8_t* __restrict__ dead,
                               uint32_t tiers, uint8_t* __restrict__ out, uint8_t* __restrict__ flagdiff) {
  const unsigned lane = lane_id();
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = gw; i < n; i += nw) {
    const uint32_t tl = tlens[i], cl = clens[i];
    uint32_t pw = 0;
    if (lane < tl) pw = tgt[(size_t)i * stride + lane];
    else if (lane < tl + cl) pw = cand[(size_t)i * stride + (lane - tl)];
    Z80S x = vec_state(int(lane)), y = x;
    run_lanes(x, pw, 0, int(tl));
    run_lanes(y, pw, int(tl), int(cl));
    const uint32_t dm = dead ? dead[i] : 0u;
    const Keep keep = make_keep(~dm, 0x3Fu, true);
    const bool eq = eq_keep(x, y, keep);
    // FlagDiff (verifier.go:658-673) over the 8 QuickCheck vectors
    const bool regs_eq = (x.a == y.a) && (x.b == y.b) && (x.c == y.c) && (x.d == y.d) &&
                         (x.e == y.e) && (x.h == y.h) && (x.l == y.l) && (x.sp == y.sp) && (x.m == y.m);
    const unsigned q8 = __ballot_sync(kFull, eq) & 0xFFu;
    const unsigned all32 = __ballot_sync(kFull, eq);
    const unsigned r8 = __ballot_sync(kFull, regs_eq) & 0xFFu;
    uint32_t fx = lane < 8 ? (x.f ^ y.f) : 0u;
    for (int off = 16; off; off >>= 1) fx |= __shfl_down_sync(kFull, fx, off);
    if (lane == 0) {
      uint8_t r = 0;
      if ((tiers & 1u) && q8 == 0xFFu) r |= 1;
      if ((tiers & 2u) && all32 == kFull) r |= 2;
      out[i] = r;
      if (flagdiff) flagdiff[i] = (r8 == 0xFFu) ? uint8_t(fx) : uint8_t(0);
    }
  }
}

// ------------------------------------------------- length-2 candidates
//
// The candidates of length 2 are the 4,531^2 odometer pairs of the 8-bit
// list (pair index = first * 4531 + second, the EnumerateSequences8 order),
// held as a pool whose QuickCheck outputs are precomputed like the length-1
// pool.  Instead of comparing every target with all 20.5M pairs, each pair
// is filed in a sorted index under a hash of its vector-0 output with F left
// out and the dead registers zeroed (one index per dead-register mask in
// use).  A target hashes its own vector-0 output the same way, finds its
// bucket by binary search, and QuickChecks only the bucket's pairs, which
// the index keeps in enumeration order.  Survivors go to fixed slots per
// (target, kind) lane; a lane whose slots are used up without a winner
// rescans its bucket from where it stopped.

// Bytes of the packed vector-0 word 0 / word 1 kept in the bucket key.
__device__ __forceinline__ uint32_t key_keep0(uint32_t dregs) {
  return 0xFFu | ((dregs & 1u) ? 0u : 0xFF0000u) | ((dregs & 2u) ? 0u : 0xFF000000u);
}
__device__ __forceinline__ uint32_t key_keep1(uint32_t dregs) {
  return ((dregs & 4u) ? 0u : 0xFFu) | ((dregs & 8u) ? 0u : 0xFF00u) | ((dregs & 16u) ? 0u : 0xFF0000u) |
         ((dregs & 32u) ? 0u : 0xFF000000u);
}
// 32-bit bucket hash of a masked output (splitmix64 finalizer).
__device__ __forceinline__ uint32_t bucket_hash(uint32_t w0, uint32_t w1, uint32_t w2) {
  unsigned long long h = ((unsigned long long)w0 << 32) | w1;
  h ^= (unsigned long long)w2 * 0x9E3779B97F4A7C15ull;
  h ^= h >> 30;
  h *= 0xBF58476D1CE4E5B9ull;
  h ^= h >> 27;
  h *= 0x94D049BB133111EBull;
  h ^= h >> 31;
  return uint32_t(h >> 32);
}

__global__ void k_pair_keys(DevPool P, uint32_t dregs, unsigned long long* __restrict__ keys) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= P.n) return;
  if (P.prune[q]) {
    keys[q] = ~0ull;  // sorts after every real entry
    return;
  }
  const uint4 o = P.qc[q];
  keys[q] = ((unsigned long long)bucket_hash(o.x & key_keep0(dregs), o.y & key_keep1(dregs), o.z) << 32) | q;
}

// Lanes of the length-2 pass: a (target, kind) lane takes part when the
// length-1 pass found no candidate for it, the target is long enough in
// bytes for a 2-instruction replacement, and (masked kind) the target has
// dead flags or registers.
__global__ void k_pair_lanes_init(DevTargets T, Lanes L1, QCOut q1, Lanes L2, PairScan ps) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long chk = 0;
  if (t < T.n) {
    const uint32_t tb = q1.meta[t].bytes;
    const bool masked = target_dead(T, t) != 0 || target_dead_regs(T, t) != 0;
    bool any = false;
    for (int kind = 0; kind < 2; kind++) {
      const uint32_t idx = 2 * t + kind;
      const bool need = L1.win[idx] == kNone && tb >= 3 && (kind == 0 || masked);
      L2.next[idx] = need ? 0u : kResolved;
      L2.spec[idx] = 0;
      L2.win[idx] = kNone;
      L2.windiff[idx] = 0;
      ps.cnt[idx] = 0;
      ps.resume[idx] = need ? 0u : kNone;
      any = any || need;
    }
    if (any) chk = ps.eligible[tb < 16 ? tb : 15];
  }
  for (int off = 16; off; off >>= 1) chk += __shfl_down_sync(kFull, chk, off);
  if (lane_id() == 0 && chk) atomicAdd(ps.checks, chk);
}

__device__ __forceinline__ uint32_t lower_bound_u64(const unsigned long long* a, uint32_t n, unsigned long long v) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    const uint32_t mid = lo + ((hi - lo) >> 1);
    if (a[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// QuickCheck bucket index of a candidate pool (at most 65,536 entries): one
// segment per dead-register mask m, keys m << 48 | bucket hash << 16 | index
// sorted, pruned candidates left out (their keys sort past the last
// segment); a top table per segment holds the first entry of each 4,096th of
// the hash range.
__global__ void k_qc_keys(DevPool P, uint32_t w2mask, unsigned long long* __restrict__ keys) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 64u * P.n) return;
  const uint32_t m = i / P.n, q = i - m * P.n;
  if (P.prune[q]) {
    keys[i] = ~0ull;
    return;
  }
  const uint4 o = P.qc[q];
  const uint32_t h = bucket_hash(o.x & key_keep0(m), o.y & key_keep1(m), o.z & w2mask);
  keys[i] = ((unsigned long long)m << 48) | ((unsigned long long)h << 16) | q;
}
__global__ void k_qc_top(const unsigned long long* __restrict__ keys, uint32_t nv, uint32_t* __restrict__ top) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 64u * (kQCTop + 1)) return;
  const uint32_t m = i / (kQCTop + 1), b = i - m * (kQCTop + 1);
  top[i] = b == kQCTop ? (m + 1) * nv
                       : m * nv + lower_bound_u64(keys + (size_t)m * nv, nv,
                                                  ((unsigned long long)m << 48) | ((unsigned long long)b << 36));
}

// QuickCheck through the bucket index: a target only meets the candidates
// whose vector-0 output agrees with its own on A, the live registers and
// word 2 (the flags are compared per candidate, under the dead flags), which
// is every candidate that can pass.  Entries of a bucket are in pool order,
// so survivors come out in enumeration order as in the full scan.
// Four targets per warp, eight lanes each: lane 8g + v runs target t0 + g on
// vector v, so one pass of the dispatch loop, the output shuffles and the
// bucket loop serve four targets (the buckets hold a candidate or two; a
// warp per target left three quarters of its lanes idle).  Lanes of a group
// that has no target (past the end) take part in the warp's collectives
// with nothing to do.
__device__ __forceinline__ void qc_target4(const DevTargets& T, uint32_t t, bool valid, QCTarget& g) {
  const unsigned lane = lane_id();
  const unsigned sub = lane & 7u;
  const uint32_t tl = valid ? target_len(T, t) : 0u;
  const uint32_t pw = sub < tl ? T.insn[(size_t)t * T.stride + sub] : 0u;
  uint32_t sz = 0, ts = 0, rd = 0;
  if (sub < tl) {
    const OpInfo oi = g_ops[pw & 0xFFFFu];
    sz = oi.size;
    ts = oi.tstates;
    rd = oi.reads;
  }
#pragma unroll
  for (int off = 2; off >= 1; off >>= 1) {
    sz += __shfl_down_sync(kFull, sz, off, 8);
    ts += __shfl_down_sync(kFull, ts, off, 8);
    rd |= __shfl_down_sync(kFull, rd, off, 8);
  }
  g.tl = tl;
  g.tb = __shfl_sync(kFull, sz, 0, 8);
  g.tts = __shfl_sync(kFull, ts, 0, 8);
  g.trd = __shfl_sync(kFull, rd, 0, 8);
  Z80S s = vec_state(int(sub));
  const uint32_t steps = __reduce_max_sync(kFull, tl);
#pragma unroll 1
  for (uint32_t i = 0; i < steps; i++) {
    const uint32_t w = __shfl_sync(kFull, pw, int(i), 8);
    if (i < tl) z_step(s, w & 0xFFFFu, w >> 16);
  }
  uint32_t w[3];
  z_pack(s, w);
#pragma unroll
  for (int v = 0; v < 8; v++) {
    g.tw[v][0] = __shfl_sync(kFull, w[0], v, 8);
    g.tw[v][1] = __shfl_sync(kFull, w[1], v, 8);
    g.tw[v][2] = __shfl_sync(kFull, w[2], v, 8);
  }
  const uint32_t dead = valid ? target_dead(T, t) & 0xFFu : 0u;
  const uint32_t dregs = valid ? target_dead_regs(T, t) & 0x3Fu : 0u;
  g.keep0 = 0xFFu | ((~dead & 0xFFu) << 8) | ((dregs & 1u) ? 0u : 0xFF0000u) | ((dregs & 2u) ? 0u : 0xFF000000u);
  g.keep1 = ((dregs & 4u) ? 0u : 0xFFu) | ((dregs & 8u) ? 0u : 0xFF00u) | ((dregs & 16u) ? 0u : 0xFF0000u) |
            ((dregs & 32u) ? 0u : 0xFF000000u);
}

// COLLECT: the collect pass; else the count pass, which with KEEP also keeps
// the survivors of targets with at most kQCSlots (single pass).
template <bool COLLECT, bool KEEP>
__global__ void __launch_bounds__(kBlock, 4) k_qc_bucket(DevTargets T, DevPool P, QCConfig cfg, QCIndex ix, QCOut o) {
  const unsigned lane = lane_id();
  const unsigned sub = lane & 7u, gshift = lane & ~7u;
  const unsigned group_lt = lanemask_lt() & (0xFFu << gshift);
  const uint32_t gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  unsigned long long my_checks = 0;
  for (uint32_t t0 = gw * 4u; t0 < T.n; t0 += nw * 4u) {
    const uint32_t t = t0 + (lane >> 3);
    const bool valid = t < T.n;
    uint32_t nf_total = 0, obase = 0;
    bool work = valid;
    if (COLLECT) {
      if (valid) {
        nf_total = o.cnt_f[t];
        const uint32_t tot = nf_total + o.cnt_m[t];
        // single pass: the count pass kept the survivors of targets with at
        // most kQCSlots of them
        work = o.tmp ? tot > kQCSlots : tot != 0;
        obase = o.base[t];
      }
      if (!__any_sync(kFull, work)) continue;
    }
    QCTarget g;
    qc_target4(T, t, valid, g);
    const uint32_t m = valid ? target_dead_regs(T, t) & 0x3Fu : 0u;
    const uint32_t h = bucket_hash(g.tw[0][0] & key_keep0(m), g.tw[0][1] & key_keep1(m), g.tw[0][2] & cfg.w2mask);
    uint32_t r0 = 0, r1 = 0;
    if (work) {
      const uint32_t* top = ix.top + m * (kQCTop + 1) + (h >> (32 - kQCTopBits));
      r0 = top[0];
      r1 = top[1];
    }
    const uint32_t iters = (__reduce_max_sync(kFull, r1 - r0) + 7u) / 8u;
    uint32_t nf = 0, nm = 0, lf = 0, lm = 0;
    uint32_t nk = 0;  // this group's survivors so far (count pass, single pass)
    uint32_t* const keep = KEEP ? o.tmp + (size_t)t * kQCSlots : nullptr;
    for (uint32_t k = 0; k < iters; k++) {
      const uint32_t i = r0 + 8u * k + sub;
      bool fp = false, mp = false;
      uint32_t diff = 0, c = 0;
      if (i < r1) {
        const unsigned long long key = ix.keys[i];
        c = uint32_t(key) & 0xFFFFu;
        if (uint32_t(key >> 16) == h && P.size[c] < g.tb)
          qc_candidate(P, P.qc[c], c, g, cfg.w2mask, cfg.all_hits != 0, fp, mp, diff);
      }
      if constexpr (!COLLECT) {
        lf += fp ? 1u : 0u;
        lm += mp ? 1u : 0u;
        if constexpr (KEEP) {
          const bool sv = fp || mp;
          const unsigned bs = __ballot_sync(kFull, sv);
          if (bs) {  // most steps find nothing
            const uint32_t rank = nk + __popc(bs & group_lt);
            if (sv && rank < kQCSlots) keep[rank] = c | (diff << 16) | (mp ? 0x80000000u : 0u);
            nk += __popc((bs >> gshift) & 0xFFu);
          }
        }
      } else {
        // this group's survivors of the step, in enumeration order
        const unsigned bf = __ballot_sync(kFull, fp), bm = __ballot_sync(kFull, mp);
        if (fp) {
          const uint32_t idx = obase + nf + __popc(bf & group_lt);
          o.surv[idx] = c;
          o.sdiff[idx] = uint16_t(diff);
        }
        if (mp) {
          const uint32_t idx = obase + nf_total + nm + __popc(bm & group_lt);
          o.surv[idx] = c;
          o.sdiff[idx] = uint16_t(diff);
        }
        nf += __popc((bf >> gshift) & 0xFFu);
        nm += __popc((bm >> gshift) & 0xFFu);
      }
    }
    if constexpr (!COLLECT) {
#pragma unroll
      for (int off = 4; off >= 1; off >>= 1) {
        lf += __shfl_xor_sync(kFull, lf, off);
        lm += __shfl_xor_sync(kFull, lm, off);
      }
      if (sub == 0 && valid) {
        my_checks += ix.elig_lt[g.tb < 255u ? g.tb : 255u];
        qc_count_out(o, t, g, lf, lm);
        if (KEEP && lf + lm > kQCSlots) atomicAdd(o.over, 1u);
      }
    }
  }
  if constexpr (!COLLECT) {
    for (int off = 16; off; off >>= 1) my_checks += __shfl_down_sync(kFull, my_checks, off);
    if (lane == 0 && my_checks) atomicAdd(o.checks, my_checks);
  }
}

// Thread per target: the survivors the single-pass count kept go to
// base[t] + (full ones in order, then masked ones in order), as the collect
// pass would have placed them.
__global__ void __launch_bounds__(256) k_qc_compact(QCOut o, uint32_t n) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const uint32_t nf = o.cnt_f[t], tot = nf + o.cnt_m[t];
  if (tot == 0 || tot > kQCSlots) return;
  const uint32_t* __restrict__ kept = o.tmp + (size_t)t * kQCSlots;
  uint32_t jf = o.base[t], jm = jf + nf;
  for (uint32_t j = 0; j < tot; j++) {
    const uint32_t e = kept[j];
    const uint32_t idx = (e >> 31) ? jm++ : jf++;
    o.surv[idx] = e & 0xFFFFu;
    o.sdiff[idx] = uint16_t((e >> 16) & 0x7FFFu);
  }
}

// Warp per target: (re)fills the slots of each lane whose slots are used up
// and whose bucket has pairs left.
__global__ void __launch_bounds__(kBlock) k_pair_scan(DevTargets T, DevPool P, QCOut q1, Lanes L2, PairScan ps,
                                                      const RoundCtl* __restrict__ gate) {
  if (gate && gate->np != 0) return;  // device-driven rounds: rescan only after an empty round
  const unsigned lane = lane_id();
  const uint32_t gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  for (uint32_t t = gw; t < T.n; t += nw) {
    bool need[2];
#pragma unroll
    for (int kind = 0; kind < 2; kind++) {
      const uint32_t idx = 2 * t + kind;
      const uint32_t nx = L2.next[idx];
      need[kind] = !(nx & kResolved) && nx >= ps.cnt[idx] && ps.resume[idx] != kNone;
    }
    if (!need[0] && !need[1]) continue;
    const uint32_t tl = target_len(T, t);
    const uint32_t pw = lane < tl ? T.insn[(size_t)t * T.stride + lane] : 0u;
    Z80S st = vec_state(int(lane & 7u));
    run_lanes(st, pw, 0, int(tl));
    uint32_t w[3];
    z_pack(st, w);
    uint32_t tw[8][3];
#pragma unroll
    for (int v = 0; v < 8; v++) {
      tw[v][0] = __shfl_sync(kFull, w[0], v);
      tw[v][1] = __shfl_sync(kFull, w[1], v);
      tw[v][2] = __shfl_sync(kFull, w[2], v);
    }
    const uint32_t tb = q1.meta[t].bytes;
    const uint32_t dead = target_dead(T, t) & 0xFFu;
    const uint32_t dregs = target_dead_regs(T, t) & 0x3Fu;
    for (int kind = 0; kind < 2; kind++) {
      if (!need[kind]) continue;
      const uint32_t idx = 2 * t + kind;
      const uint32_t m = kind ? dregs : 0u;
      // the index holding only pairs that can be shorter than the target
      const unsigned long long* ix = tb == 3 ? ps.idx_le2[m] : (tb == 4 ? ps.idx_le3[m] : ps.idx[m]);
      const uint32_t nv = tb == 3 ? ps.n_le2 : (tb == 4 ? ps.n_le3 : ps.n_valid);
      const uint32_t h = bucket_hash(tw[0][0] & key_keep0(m), tw[0][1] & key_keep1(m), tw[0][2]);
      uint32_t lo = 0, hi = 0;
      if (lane == 0) {
        lo = lower_bound_u64(ix, nv, (unsigned long long)h << 32);
        hi = (h == 0xFFFFFFFFu) ? nv : lower_bound_u64(ix, nv, (unsigned long long)(h + 1u) << 32);
      }
      lo = __shfl_sync(kFull, lo, 0);
      hi = __shfl_sync(kFull, hi, 0);
      // compared bytes: kind 0 everything; kind 1 without the dead flags and registers
      const uint32_t keep0 = kind ? (0xFFu | ((~dead & 0xFFu) << 8) | ((dregs & 1u) ? 0u : 0xFF0000u) |
                                     ((dregs & 2u) ? 0u : 0xFF000000u))
                                  : 0xFFFFFFFFu;
      const uint32_t keep1 = kind ? key_keep1(dregs) : 0xFFFFFFFFu;
      uint32_t pos = lo + ps.resume[idx];
      uint32_t found = 0;
      bool capped = false;
      while (pos < hi && !capped) {
        const uint32_t j = pos + lane;
        bool pass = false;
        uint32_t c = 0, diff = 0;
        if (j < hi) {
          c = uint32_t(ix[j]);
          if (P.size[c] < tb) {
            const uint4 o = P.qc[c];
            const uint32_t d0 = o.x ^ tw[0][0], d1 = o.y ^ tw[0][1], d2 = o.z ^ tw[0][2];
            if (((d0 & keep0) | (d1 & keep1) | d2) == 0) {
              bool full = (d0 | d1 | d2) == 0;
              uint32_t fd = (d0 >> 8) & 0xFFu, rdf = reg_diff(d0, d1);
              bool ok = true;
#pragma unroll
              for (int v = 1; v < 8; v++) {
                const uint4 ov = P.qc[(size_t)v * P.n + c];
                const uint32_t e0 = ov.x ^ tw[v][0], e1 = ov.y ^ tw[v][1], e2 = ov.z ^ tw[v][2];
                ok = ok && (((e0 & keep0) | (e1 & keep1) | e2) == 0);
                full = full && ((e0 | e1 | e2) == 0);
                fd |= (e0 >> 8) & 0xFFu;
                rdf |= reg_diff(e0, e1);
              }
              pass = ok && (kind ? !full : full);
              diff = fd | (rdf << 8);
            }
          }
        }
        const unsigned b = __ballot_sync(kFull, pass);
        const uint32_t room = kSlots2 - found;
        const uint32_t r = __popc(b & lanemask_lt());
        if (pass && r < room) {
          ps.surv[(size_t)idx * kSlots2 + found + r] = c;
          ps.sdiff[(size_t)idx * kSlots2 + found + r] = uint16_t(diff);
        }
        const uint32_t nb = __popc(b);
        if (nb > room) {
          // resume after the last survivor that fit
          uint32_t bb = b;
          for (uint32_t k = 0; k < room; k++) bb &= bb - 1;
          pos += uint32_t(__ffs(bb)) - 1u;
          found = kSlots2;
          capped = true;
        } else {
          found += nb;
          pos += 32;
          capped = found == kSlots2;
        }
      }
      if (lane == 0) {
        ps.cnt[idx] = found;
        L2.next[idx] = 0;
        ps.resume[idx] = pos >= hi ? kNone : pos - lo;
      }
    }
  }
}

// One pair per length-2 lane with an untried survivor; lanes with no slot
// left either end without a winner (bucket exhausted) or wait for a rescan.
// One round of the length-2 pass: windows over the lane's slots; a lane
// with its slots used up and its bucket not exhausted asks for a rescan.
__global__ void k_pair_round_build(DevTargets T, DevPool P, QCOut q1, Lanes L2, PairScan ps, RoundBuf R) {
  const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t w = 0, sbase = 0;
  if (idx < 2 * T.n) {
    const uint32_t nx = L2.next[idx];
    if (!(nx & kResolved)) {
      if (nx < ps.cnt[idx]) {
        w = min(1u << L2.spec[idx], ps.cnt[idx] - nx);
        sbase = idx * kSlots2 + nx;
      } else if (ps.resume[idx] == kNone) {
        L2.next[idx] = nx | kResolved;
      } else {
        atomicAdd(ps.refill, 1u);
      }
    }
  }
  if (!__any_sync(kFull, w != 0)) return;
  const uint32_t p0 = alloc_pairs(R.npairs, w);
  const uint32_t fit = p0 >= R.cap ? 0u : min(w, R.cap - p0);
  for (uint32_t j = 0; j < fit; j++)
    put_pair(R, p0 + j, T, P, q1, idx >> 1, idx & 1u, ps.surv[sbase + j], sbase + j,
             j == 0 ? uint8_t(fit) : uint8_t(0), p0 + fit);
}


unsigned grid_for(uint32_t n, unsigned block) { return (n + block - 1) / block; }

// Launch facts are properties of a device: its SM count, and per kernel the
// dynamic shared-memory limit (cudaFuncSetAttribute acts on the current
// device) and the resident blocks per SM.  They are cached per device, for
// the device current at the launch; devices past kMaxCachedDevices are
// queried on every launch.
constexpr int kMaxCachedDevices = 64;
std::atomic<int> g_num_sms[kMaxCachedDevices];

int current_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
  return dev;
}

// Resident blocks per SM of kernel f on the current device with `smem`
// bytes of dynamic shared memory, raising the kernel's shared-memory limit
// to smem first when it is above the default; cache[] keeps one answer per
// device.
template <class F>
int blocks_per_sm(std::atomic<int>* cache, F f, int block, size_t smem, size_t smem_limit) {
  const int dev = current_device();
  if (dev >= 0 && dev < kMaxCachedDevices) {
    const int c = cache[dev].load(std::memory_order_relaxed);
    if (c) return c;
  }
  if (smem_limit) cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_limit));
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, block, smem);
  if (per_sm < 1) per_sm = 1;
  if (dev >= 0 && dev < kMaxCachedDevices) cache[dev].store(per_sm, std::memory_order_relaxed);
  return per_sm;
}

}  // namespace

int dev_num_sms() {
  const int dev = current_device();
  if (dev >= 0 && dev < kMaxCachedDevices) {
    const int c = g_num_sms[dev].load(std::memory_order_relaxed);
    if (c) return c;
  }
  int n = 0;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  if (n <= 0) n = 1;
  if (dev >= 0 && dev < kMaxCachedDevices) g_num_sms[dev].store(n, std::memory_order_relaxed);
  return n;
}

}  // namespace z80b

// Host helpers that need the tables (kept out of the anonymous namespace).
#include "z80_tables.h"

namespace z80b {

void dev_upload_tables(cudaStream_t s) {
  cudaMemcpyToSymbolAsync(g_ops, op_table(), sizeof(OpInfo) * kNumOps, 0, cudaMemcpyHostToDevice, s);
  cudaMemcpyToSymbolAsync(g_vec, mid_vectors(), sizeof(uint32_t) * 32 * 3, 0, cudaMemcpyHostToDevice, s);
  cudaMemcpyToSymbolAsync(c_rep, rep_values(), 32, 0, cudaMemcpyHostToDevice, s);
  cudaMemcpyToSymbolAsync(c_repsp, rep_sp(), 32, 0, cudaMemcpyHostToDevice, s);
  cudaMemcpyToSymbolAsync(g_rep, rep_values(), 32, 0, cudaMemcpyHostToDevice, s);
  cudaMemcpyToSymbolAsync(g_repsp, rep_sp(), 32, 0, cudaMemcpyHostToDevice, s);
  cudaMemcpyToSymbolAsync(g_aclass, op_aclass(), kNumOps, 0, cudaMemcpyHostToDevice, s);
  {
    cudaMemcpyToSymbolAsync(g_dep, op_deps(), sizeof(uint32_t) * kNumOps * kDepFields, 0, cudaMemcpyHostToDevice, s);
    cudaMemcpyToSymbolAsync(g_keepa, op_keeps_a(), kNumOps, 0, cudaMemcpyHostToDevice, s);
    cudaMemcpyToSymbolAsync(g_keeps, op_keeps(), sizeof(uint16_t) * kNumOps, 0, cudaMemcpyHostToDevice, s);
    const CompactTables& C = compact_tables();
    cudaMemcpyToSymbolAsync(g_cren, C.ren, sizeof C.ren, 0, cudaMemcpyHostToDevice, s);
    cudaMemcpyToSymbolAsync(g_corig, C.orig, sizeof C.orig, 0, cudaMemcpyHostToDevice, s);
    cudaMemcpyToSymbolAsync(g_cid, C.id_of_set, sizeof C.id_of_set, 0, cudaMemcpyHostToDevice, s);
    cudaMemcpyToSymbolAsync(g_opregs, C.opregs, sizeof C.opregs, 0, cudaMemcpyHostToDevice, s);
    const WideTables& W = wide_tables();
    cudaMemcpyToSymbolAsync(g_wren, W.ren, sizeof W.ren, 0, cudaMemcpyHostToDevice, s);
    cudaMemcpyToSymbolAsync(g_worig, W.orig, sizeof W.orig, 0, cudaMemcpyHostToDevice, s);
    cudaMemcpyToSymbolAsync(g_wid, W.id_of_set, sizeof W.id_of_set, 0, cudaMemcpyHostToDevice, s);
  }
}

void launch_pool_outputs(const uint32_t* insn, uint32_t n, uint32_t len, uint4* qc, uint4* mid,
                         cudaStream_t s) {
  if (!n) return;
  unsigned grid = std::min<unsigned>(grid_for(n, 4), unsigned(dev_num_sms() * 16));
  k_pool_outputs<<<grid, 128, 0, s>>>(insn, n, len, qc, mid);
}
void launch_exec(const uint32_t* in, const uint32_t* seqs, const uint8_t* lens, uint32_t len,
                 uint32_t stride, uint32_t n, uint32_t* out, cudaStream_t s) {
  if (!n) return;
  unsigned grid = std::min<unsigned>(grid_for(n, 4), unsigned(dev_num_sms() * 16));
  k_exec<<<grid, 128, 0, s>>>(in, seqs, lens, len, stride, n, out);
}
void launch_fingerprints(const uint32_t* seqs, uint32_t n, uint32_t len, uint8_t* out, cudaStream_t s) {
  if (!n) return;
  unsigned grid = std::min<unsigned>(grid_for(n, 4), unsigned(dev_num_sms() * 16));
  k_fingerprints<<<grid, 128, 0, s>>>(seqs, n, len, out);
}
void launch_fp_query(const DevPool& P, const uint32_t* fp, uint32_t dead, uint32_t* hits,
                     uint32_t* nhits, uint32_t cap, cudaStream_t s) {
  if (!P.n) return;
  k_fp_query<<<grid_for(P.n, 256), 256, 0, s>>>(P, fp, dead, hits, nhits, cap);
}
void launch_qc_scan(const DevTargets& T, const DevPool& P, const QCConfig& cfg, const QCOut& o,
                    bool collect, cudaStream_t s) {
  if (!T.n) return;
  size_t smem = cfg.use_smem ? (size_t)P.n * 17 + 16 : 0;
  // occupancy depends on smem (the pool's size), so it is cached per device
  // only for the limit; the answer for this launch is computed each time
  static std::atomic<int> limit_set[2][kMaxCachedDevices];
  const int dev = current_device();
  const bool cache_ok = dev >= 0 && dev < kMaxCachedDevices;
  if (!cache_ok || !limit_set[collect][dev].load(std::memory_order_relaxed)) {
    if (collect) cudaFuncSetAttribute(k_qc_scan<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    else cudaFuncSetAttribute(k_qc_scan<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (cache_ok) limit_set[collect][dev].store(1, std::memory_order_relaxed);
  }
  int per_sm = 0;
  if (collect)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_qc_scan<true>, kBlock, smem);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_qc_scan<false>, kBlock, smem);
  if (per_sm < 1) per_sm = 1;
  unsigned need = grid_for(T.n, kBlock / 32);
  unsigned grid = unsigned(dev_num_sms() * per_sm);
  if (grid > need) grid = need;
  if (collect) k_qc_scan<true><<<grid, kBlock, smem, s>>>(T, P, cfg, o);
  else k_qc_scan<false><<<grid, kBlock, smem, s>>>(T, P, cfg, o);
}
void launch_qc_keys(const DevPool& P, uint32_t w2mask, unsigned long long* keys, cudaStream_t s) {
  const uint32_t n = 64u * P.n;
  if (n) k_qc_keys<<<grid_for(n, 256), 256, 0, s>>>(P, w2mask, keys);
}
void launch_qc_top(const unsigned long long* keys, uint32_t nv, uint32_t* top, cudaStream_t s) {
  const uint32_t n = 64u * (kQCTop + 1);
  k_qc_top<<<grid_for(n, 256), 256, 0, s>>>(keys, nv, top);
}
void launch_qc_compact(const QCOut& q, uint32_t n, cudaStream_t s) {
  if (!n) return;
  k_qc_compact<<<grid_for(n, 256), 256, 0, s>>>(q, n);
}

void launch_qc_bucket(const DevTargets& T, const DevPool& P, const QCConfig& cfg, const QCIndex& ix,
                      const QCOut& o, bool collect, cudaStream_t s) {
  if (!T.n) return;
  static std::atomic<int> occ[3][kMaxCachedDevices];
  const bool keep = !collect && o.tmp;
  const int per_sm = collect ? blocks_per_sm(occ[1], k_qc_bucket<true, false>, kBlock, 0, 0)
                             : (keep ? blocks_per_sm(occ[2], k_qc_bucket<false, true>, kBlock, 0, 0)
                                     : blocks_per_sm(occ[0], k_qc_bucket<false, false>, kBlock, 0, 0));
  unsigned need = grid_for((T.n + 3u) / 4u, kBlock / 32);  // four targets per warp
  unsigned grid = unsigned(dev_num_sms() * per_sm);
  if (grid > need) grid = need;
  if (collect) k_qc_bucket<true, false><<<grid, kBlock, 0, s>>>(T, P, cfg, ix, o);
  else if (keep) k_qc_bucket<false, true><<<grid, kBlock, 0, s>>>(T, P, cfg, ix, o);
  else k_qc_bucket<false, false><<<grid, kBlock, 0, s>>>(T, P, cfg, ix, o);
}
void launch_round_build(const DevTargets& T, const DevPool& P, const QCOut& q, const Lanes& L,
                        const RoundBuf& R, cudaStream_t s) {
  if (!T.n) return;
  k_round_build<<<grid_for(T.n, 256), 256, 0, s>>>(T, P, q, L, R);
}
void launch_pairs_from_survivors(const DevTargets& T, const DevPool& P, const QCOut& q,
                                 const uint8_t* midpass, uint32_t nsurv, const uint32_t* surv_target,
                                 const RoundBuf& R, cudaStream_t s) {
  if (!nsurv) return;
  k_pairs_from_survivors<<<grid_for(nsurv, 256), 256, 0, s>>>(T, P, q, midpass, nsurv, surv_target, R);
}
// Shared memory of a sweep kernel (bit-sliced classes): the candidate's
// output planes, one column of words per lane.
constexpr int exhaustive_smem(int cls) {
  return cls == 1 ? 0
                  : kBlock * (cls == 3 ? kCompactWords : (cls == 4 ? kWideWords : (cls == 5 ? kRegWords : kBitsWords))) * 4;
}
// Resident blocks per SM of a sweep kernel on the current device (its
// shared-memory limit raised first), cached per device.
template <int K, int CLS>
int exhaustive_blocks_per_sm() {
  constexpr int smem = exhaustive_smem(CLS);
  static std::atomic<int> occ[kMaxCachedDevices];
  return blocks_per_sm(occ, k_exhaustive<K, CLS>, kBlock, smem, smem);
}
template <int K, int CLS>
void launch_exhaustive_k(const DevTargets& T, const DevPool& P, const RoundBuf& R, uint32_t npairs,
                         unsigned long long total, cudaStream_t s) {
  constexpr int smem = exhaustive_smem(CLS);
  const int per_sm = exhaustive_blocks_per_sm<K, CLS>();
  // resident blocks, or more when the chunks exceed kChunksPerWarp per warp
  const unsigned long long wpb = kBlock / 32;
  unsigned long long need = (total + wpb - 1) / wpb;
  unsigned long long grid = (unsigned long long)dev_num_sms() * per_sm;
  if (grid > need) grid = need;
  const unsigned long long cover = (total + wpb * kChunksPerWarp - 1) / (wpb * kChunksPerWarp);
  if (grid < cover) grid = cover;
  if (grid > 0x7FFFFFFFull) grid = 0x7FFFFFFFull;
  k_exhaustive<K, CLS><<<unsigned(grid), kBlock, smem, s>>>(T, P, R, npairs, total, nullptr, nullptr,
                                                               kChunksPerWarp);
}

// The same kernel on a persistent grid (resident blocks on every SM) whose
// blocks take chunks until the class's device-side total is spent.
template <int K, int CLS>
void launch_exhaustive_dev_k(const DevTargets& T, const DevPool& P, const RoundBuf& R, const unsigned long long* total,
                             const uint32_t* np, cudaStream_t s) {
  constexpr int smem = exhaustive_smem(CLS);
  const int per_sm = exhaustive_blocks_per_sm<K, CLS>();
  const unsigned grid = unsigned(dev_num_sms() * per_sm);
  k_exhaustive<K, CLS><<<grid, kBlock, smem, s>>>(T, P, R, 0u, 0ull, total, np, 0x7FFFFFFF);
}

int launch_exhaustive(const DevTargets& T, const DevPool& P, const RoundBuf& R, uint32_t npairs,
                      unsigned long long total_b, unsigned long long total_x, unsigned long long total_c,
                      unsigned long long total_w, unsigned long long total_r, int k, cudaStream_t s,
                      uint32_t* kernels) {
  if (!npairs) return 0;
  int n = 0;
  uint32_t mask = 0;
  if (total_r) {
    launch_exhaustive_k<1, 5>(T, P, R, npairs, total_r, s);
    mask |= kSweepRegs;
    n++;
  }
  if (total_w) {
    launch_exhaustive_k<1, 4>(T, P, R, npairs, total_w, s);
    mask |= kSweepWide;
    n++;
  }
  if (total_c) {
    launch_exhaustive_k<1, 3>(T, P, R, npairs, total_c, s);
    mask |= kSweepCompact;
    n++;
  }
  if (total_b) {
    launch_exhaustive_k<1, 0>(T, P, R, npairs, total_b, s);
    mask |= kSweepBits;
    n++;
  }
  if (total_x) {
    if (R.xunit == kXBitsBlocks) {
      launch_exhaustive_k<1, 2>(T, P, R, npairs, total_x, s);
      mask |= kSweepXBits;
    } else {
      switch (k) {
        case 1: launch_exhaustive_k<1, 1>(T, P, R, npairs, total_x, s); mask |= kSweepScalarK1; break;
        case 2: launch_exhaustive_k<2, 1>(T, P, R, npairs, total_x, s); mask |= kSweepScalarK1 << 1; break;
        case 8: launch_exhaustive_k<8, 1>(T, P, R, npairs, total_x, s); mask |= kSweepScalarK1 << 3; break;
        default: launch_exhaustive_k<4, 1>(T, P, R, npairs, total_x, s); mask |= kSweepScalarK1 << 2; break;
      }
    }
    n++;
  }
  if (kernels) *kernels |= mask;
  return n;
}
void launch_round_resolve(const RoundBuf& R, uint32_t npairs, const QCOut& q, const Lanes& L, uint32_t max_spec,
                          cudaStream_t s) {
  if (!npairs) return;
  k_round_resolve<<<grid_for(npairs, 256), 256, 0, s>>>(R, npairs, q, L, max_spec, nullptr);
}

// The round's chunk prefixes on the device, in three launches: every block
// of k_round_scan_sum sums its contiguous segment of each class's chunk
// counts (coalesced tiles), k_round_scan_write rescans its segment from the
// sum of the blocks before it, and k_round_scan_ctl takes the totals, clears
// the dispensers, keeps the loop's counters and sets its condition.  The
// first two only read RoundCtl; the third alone writes it.
constexpr int kRScanThreads = 256;
static_assert(kRScanThreads == kRScanBlocks, "one block sum per thread in the offset reduction");

__device__ __forceinline__ bool rscan_on(const RoundBuf& R, int c) { return !((c == 2 && !R.compact) || (c >= 3 && !R.wide)); }
__device__ __forceinline__ const unsigned long long* rscan_in(const RoundBuf& R, int c) {
  return c == 0 ? R.nchunks : (c == 1 ? R.nchunks_x : (c == 2 ? R.nchunks_c : (c == 3 ? R.nchunks_w : R.nchunks_r)));
}
__device__ __forceinline__ unsigned long long* rscan_out(const RoundBuf& R, int c) {
  return c == 0 ? R.cbase : (c == 1 ? R.cbase_x : (c == 2 ? R.cbase_c : (c == 3 ? R.cbase_w : R.cbase_r)));
}
// The pairs to scan: the build's count, or 0 once the loop is past its bound.
__device__ __forceinline__ uint32_t rscan_np(const RoundBuf& R, const RoundCtl* ctl) {
  const uint32_t np = min(*R.npairs, R.cap);
  return ctl->iters + 1 >= kMaxRoundIters ? 0u : np;
}
// Block-wide sum, the result in every thread (red: kRScanThreads / 32 slots).
__device__ __forceinline__ unsigned long long rscan_block_sum(unsigned long long v, unsigned long long* red) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  __syncthreads();  // red is free (an earlier call has been read)
  if (lane_id() == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  unsigned long long t = 0;
#pragma unroll
  for (int w = 0; w < kRScanThreads / 32; w++) t += red[w];
  return t;
}

__global__ void __launch_bounds__(kRScanThreads) k_round_scan_sum(RoundBuf R, RoundCtl* __restrict__ ctl) {
  __shared__ unsigned long long red[kRScanThreads / 32];
  const uint32_t np = rscan_np(R, ctl);
  if (np == 0) return;
  const uint32_t per = (np + kRScanBlocks - 1) / kRScanBlocks;
  const uint32_t lo = uint32_t(min((unsigned long long)blockIdx.x * per, (unsigned long long)np));
  const uint32_t hi = lo + min(per, np - lo);
  for (int c = 0; c < 5; c++) {
    if (!rscan_on(R, c)) continue;  // the same for every block
    const unsigned long long* __restrict__ in = rscan_in(R, c);
    unsigned long long v = 0;
    for (uint32_t i = lo + threadIdx.x; i < hi; i += kRScanThreads) v += in[i];
    v = rscan_block_sum(v, red);
    if (threadIdx.x == 0) ctl->bsum[c][blockIdx.x] = v;  // 0 for an empty segment
  }
}

__global__ void __launch_bounds__(kRScanThreads) k_round_scan_write(RoundBuf R, const RoundCtl* __restrict__ ctl) {
  __shared__ unsigned long long red[kRScanThreads / 32];
  const uint32_t np = rscan_np(R, ctl);
  if (np == 0) return;
  const uint32_t per = (np + kRScanBlocks - 1) / kRScanBlocks;
  const uint32_t lo = uint32_t(min((unsigned long long)blockIdx.x * per, (unsigned long long)np));
  const uint32_t hi = lo + min(per, np - lo);
  const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
  for (int c = 0; c < 5; c++) {
    if (!rscan_on(R, c)) continue;
    const unsigned long long* __restrict__ in = rscan_in(R, c);
    unsigned long long* __restrict__ out = rscan_out(R, c);
    // chunks of the blocks before this one
    unsigned long long run = rscan_block_sum(threadIdx.x < blockIdx.x ? ctl->bsum[c][threadIdx.x] : 0ull, red);
    for (uint32_t base = lo; base < hi; base += kRScanThreads) {
      const uint32_t i = base + threadIdx.x;
      const unsigned long long v = i < hi ? in[i] : 0ull;
      // inclusive warp scan, then the warps' totals
      unsigned long long x = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(kFull, x, o);
        if (lane >= unsigned(o)) x += y;
      }
      __syncthreads();  // red is free
      if (lane == 31) red[warp] = x;
      __syncthreads();
      unsigned long long before = 0, tile = 0;
#pragma unroll
      for (int w = 0; w < kRScanThreads / 32; w++) {
        before += unsigned(w) < warp ? red[w] : 0ull;
        tile += red[w];
      }
      if (i < hi) out[i] = run + before + x - v;
      run += tile;
    }
  }
}

__global__ void k_round_scan_ctl(RoundBuf R, RoundCtl* __restrict__ ctl, const uint32_t* __restrict__ refill,
                                 cudaGraphConditionalHandle loop) {
  const unsigned lane = lane_id();
  const uint32_t np = min(*R.npairs, R.cap);
  const bool over = ctl->iters + 1 >= kMaxRoundIters;
  const bool empty = np == 0 || over;
  unsigned long long tot[5];
#pragma unroll
  for (int c = 0; c < 5; c++) {
    unsigned long long v = 0;
    if (!empty && rscan_on(R, c))
      for (int b = lane; b < kRScanBlocks; b += 32) v += ctl->bsum[c][b];
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    tot[c] = v;
  }
  if (lane != 0) return;
  ctl->iters += 1;
  if (over) {
    // the loop has run far past any legitimate number of rounds: end it,
    // sweep nothing more, and let the host report the error
    ctl->overrun = 1;
    cudaGraphSetConditional(loop, 0);
  }
  ctl->np = over ? 0u : np;
  if (!empty) {
    ctl->rounds += 1;
    ctl->pairs += np;
  }
  R.counter[0] = R.counter[1] = R.counter[2] = R.counter[3] = R.counter[4] = 0;
#pragma unroll
  for (int c = 0; c < 5; c++) ctl->totals[c] = tot[c];
  if (empty && (!refill || *refill == 0)) cudaGraphSetConditional(loop, 0);
}

void launch_round_scan(const RoundBuf& R, RoundCtl* ctl, const uint32_t* refill, cudaGraphConditionalHandle loop,
                       cudaStream_t s) {
  k_round_scan_sum<<<kRScanBlocks, kRScanThreads, 0, s>>>(R, ctl);
  k_round_scan_write<<<kRScanBlocks, kRScanThreads, 0, s>>>(R, ctl);
  k_round_scan_ctl<<<1, 32, 0, s>>>(R, ctl, refill, loop);
}

template <int K, int CLS>
void warm_exhaustive_k() {
  (void)exhaustive_blocks_per_sm<K, CLS>();
}
void warm_exhaustive_dev(const RoundBuf& R, int k) {
  (void)dev_num_sms();
  if (R.wide) {
    warm_exhaustive_k<1, 4>();
    warm_exhaustive_k<1, 5>();
  }
  if (R.compact) warm_exhaustive_k<1, 3>();
  warm_exhaustive_k<1, 0>();
  if (R.xunit == kXBitsBlocks) warm_exhaustive_k<1, 2>();
  else if (k == 1) warm_exhaustive_k<1, 1>();
  else if (k == 2) warm_exhaustive_k<2, 1>();
  else if (k == 8) warm_exhaustive_k<8, 1>();
  else warm_exhaustive_k<4, 1>();
}

int launch_exhaustive_dev(const DevTargets& T, const DevPool& P, const RoundBuf& R, const RoundCtl* ctl, int k,
                          const cudaStream_t* ss) {
  int n = 0;
  if (R.wide) {
    launch_exhaustive_dev_k<1, 5>(T, P, R, &ctl->totals[4], &ctl->np, ss[0]);
    launch_exhaustive_dev_k<1, 4>(T, P, R, &ctl->totals[3], &ctl->np, ss[1]);
    n += 2;
  }
  if (R.compact) {
    launch_exhaustive_dev_k<1, 3>(T, P, R, &ctl->totals[2], &ctl->np, ss[2]);
    n++;
  }
  launch_exhaustive_dev_k<1, 0>(T, P, R, &ctl->totals[0], &ctl->np, ss[3]);
  const cudaStream_t sx = ss[4];
  if (R.xunit == kXBitsBlocks) {
    launch_exhaustive_dev_k<1, 2>(T, P, R, &ctl->totals[1], &ctl->np, sx);
  } else {
    switch (k) {
      case 1: launch_exhaustive_dev_k<1, 1>(T, P, R, &ctl->totals[1], &ctl->np, sx); break;
      case 2: launch_exhaustive_dev_k<2, 1>(T, P, R, &ctl->totals[1], &ctl->np, sx); break;
      case 8: launch_exhaustive_dev_k<8, 1>(T, P, R, &ctl->totals[1], &ctl->np, sx); break;
      default: launch_exhaustive_dev_k<4, 1>(T, P, R, &ctl->totals[1], &ctl->np, sx); break;
    }
  }
  return n + 2;
}

void launch_round_resolve_dev(const RoundBuf& R, const RoundCtl* ctl, const QCOut& q, const Lanes& L,
                              uint32_t max_spec, cudaStream_t s) {
  k_round_resolve<<<grid_for(R.cap, 256), 256, 0, s>>>(R, R.cap, q, L, max_spec, &ctl->np);
}

void launch_midcheck(const DevTargets& T, const DevPool& P, const uint32_t* surv,
                     const uint32_t* surv_target, uint32_t nsurv, uint8_t* pass, cudaStream_t s) {
  if (!nsurv) return;
  unsigned long long need = (unsigned long long)nsurv * 32;
  unsigned grid = unsigned(need / 256 + 1);
  unsigned cap = unsigned(dev_num_sms() * 8);
  if (grid > cap) grid = cap;
  k_midcheck<<<grid, 256, 0, s>>>(T, P, surv, surv_target, nsurv, pass);
}
void launch_surv_targets(const QCOut& q, uint32_t n, uint32_t* st, cudaStream_t s) {
  if (!n) return;
  k_surv_targets<<<grid_for(n, 256), 256, 0, s>>>(q, n, st);
}
void launch_rule_count_first(const Lanes& L, const Lanes& L2, uint32_t n, uint32_t* cnt, const DevTargets& T,
                             unsigned long long* checked, uint32_t pool_enum, unsigned long long pool2_enum,
                             cudaStream_t s) {
  if (!n) return;
  k_rule_count_first<<<grid_for(n, 256), 256, 0, s>>>(L, L2, n, cnt, T, checked, pool_enum, pool2_enum);
}
void launch_rule_write_first(const Lanes& L, const Lanes& L2, uint32_t n, const uint32_t* base, DevRule* out,
                             cudaStream_t s) {
  if (!n) return;
  k_rule_write_first<<<grid_for(n, 256), 256, 0, s>>>(L, L2, n, base, out);
}
void launch_rule_count_all(const RoundBuf& R, uint32_t npairs, uint32_t* flag, cudaStream_t s) {
  if (!npairs) return;
  k_rule_count_all<<<grid_for(npairs, 256), 256, 0, s>>>(R, npairs, flag);
}
void launch_rule_write_all(const uint32_t* flag, const uint32_t* base, uint32_t nsurv,
                           const uint32_t* surv, const uint16_t* sdiff, const uint32_t* surv_target,
                           DevRule* out, cudaStream_t s) {
  if (!nsurv) return;
  k_rule_write_all<<<grid_for(nsurv, 256), 256, 0, s>>>(flag, base, nsurv, surv, sdiff, surv_target, out);
}
void launch_verify_small(const uint32_t* tgt, const uint8_t* tlens, const uint32_t* cand,
                         const uint8_t* clens, uint32_t stride, uint32_t n, const uint8_t* dead,
                         uint32_t tiers, uint8_t* out, uint8_t* flagdiff, cudaStream_t s) {
  if (!n) return;
  unsigned grid = unsigned(((unsigned long long)n * 32 + 255) / 256);
  unsigned cap = unsigned(dev_num_sms() * 8);
  if (grid > cap) grid = cap;
  k_verify_small<<<grid, 256, 0, s>>>(tgt, tlens, cand, clens, stride, n, dead, tiers, out, flagdiff);
}

void launch_pair_keys(const DevPool& P, uint32_t dregs, unsigned long long* keys, cudaStream_t s) {
  if (!P.n) return;
  k_pair_keys<<<grid_for(P.n, 256), 256, 0, s>>>(P, dregs, keys);
}
void launch_pair_lanes_init(const DevTargets& T, const Lanes& L1, const QCOut& q1, const Lanes& L2,
                            const PairScan& ps, cudaStream_t s) {
  if (!T.n) return;
  k_pair_lanes_init<<<grid_for(T.n, 256), 256, 0, s>>>(T, L1, q1, L2, ps);
}
void launch_pair_scan(const DevTargets& T, const DevPool& P, const QCOut& q1, const Lanes& L2, const PairScan& ps,
                      cudaStream_t s) {
  if (!T.n) return;
  unsigned grid = std::min<unsigned>(grid_for(T.n, kBlock / 32), unsigned(dev_num_sms() * 8));
  k_pair_scan<<<grid, kBlock, 0, s>>>(T, P, q1, L2, ps, nullptr);
}
void launch_pair_scan_gated(const DevTargets& T, const DevPool& P, const QCOut& q1, const Lanes& L2,
                            const PairScan& ps, const RoundCtl* ctl, cudaStream_t s) {
  if (!T.n) return;
  unsigned grid = std::min<unsigned>(grid_for(T.n, kBlock / 32), unsigned(dev_num_sms() * 8));
  k_pair_scan<<<grid, kBlock, 0, s>>>(T, P, q1, L2, ps, ctl);
}
void launch_pair_round_build(const DevTargets& T, const DevPool& P, const QCOut& q1, const Lanes& L2,
                             const PairScan& ps, const RoundBuf& R, cudaStream_t s) {
  if (!T.n) return;
  k_pair_round_build<<<grid_for(2 * T.n, 256), 256, 0, s>>>(T, P, q1, L2, ps, R);
}


}  // namespace z80b
