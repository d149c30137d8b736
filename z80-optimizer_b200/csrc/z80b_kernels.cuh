// z80b_kernels.cuh -- kernel declarations and launch parameters.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "z80b_device.cuh"

namespace z80b {

// Surviving (target, candidate) pairs of the QuickCheck scan.
struct QCOut {
  uint32_t* cnt_f;   // [n] full-equivalence survivors per target
  uint32_t* cnt_m;   // [n] masked-only survivors per target
  uint32_t* cnt_all; // [n] cnt_f + cnt_m (scan input)
  const uint32_t* base;  // [n] exclusive prefix of cnt_f + cnt_m (collect pass)
  uint32_t* surv;    // survivor pool indices
  uint16_t* sdiff;   // FlagDiff (low byte) | differing registers << 8
  TargetMeta* meta;  // [n]
  unsigned long long* checks;  // eligible pairs evaluated (count pass)
  // Single-pass QuickCheck (bucket index only; null: count and collect
  // passes): the count pass also keeps the survivors of each target that has
  // at most kQCSlots of them, in enumeration order, as candidate | diff << 16
  // | masked << 31 in tmp[t * kQCSlots ...], and counts the targets with more
  // in *over; k_qc_compact moves the kept ones to their places and the
  // collect pass runs for the others alone.
  uint32_t* tmp;
  uint32_t* over;
};
constexpr uint32_t kQCSlots = 8;

struct QCConfig {
  uint32_t w2mask;   // 0xFFFFFFFF: compare SP and M; 0x0000FFFF: fingerprint (SP only)
  int all_hits;      // 1: pkg/gpu semantics (one list: masked-QC passes)
  int use_smem;      // pool QC0 staged in shared memory
};

// QuickCheck bucket index of a candidate pool (pools of at most 65,536
// candidates): 64 segments (one per dead-register mask) of sorted keys
// m << 48 | hash << 16 | index over the unpruned candidates, a top table of
// kQCTop + 1 offsets per segment, and the unpruned candidates shorter than b
// bytes (the count of QuickCheck units a target of b bytes evaluates).
constexpr uint32_t kQCTopBits = 12, kQCTop = 1u << kQCTopBits;
constexpr uint32_t kQCIndexMax = 65536;
struct QCIndex {
  const unsigned long long* keys;  // [64 * n_valid]
  const uint32_t* top;             // [64 * (kQCTop + 1)]
  const uint32_t* elig_lt;         // [256]
};

// Per-(target, kind) progress of the first-found rounds.
struct Lanes {
  uint32_t* next;    // [2n] survivor index to try next; bit31 = resolved
  uint32_t* win;     // [2n] winning pool index or kNone
  uint16_t* windiff; // [2n] sdiff of the winner
  uint8_t* spec;     // [2n] log2 of the lane's survivor window in the next round
};

// A-independent sweeps: 128 A-blocks per unit in the scalar kernel, 1,024
// (32 per lane, 32 states per lane word) in the bit-sliced one.
constexpr uint32_t kXScalarBlocks = 128, kXBitsBlocks = 1024;

// Survivor windows: a lane whose survivors keep failing ExhaustiveCheck
// takes 1, 2, 4, ... of its next survivors (in enumeration order) into one
// round, up to these caps; the first one that passes wins, as if they had
// been tried one per round.
constexpr uint32_t kMaxSpec1 = 6;  // length-1 pass: windows up to 64
constexpr uint32_t kMaxSpec2 = 5;  // length-2 pass: windows up to 32 (the lane's slots)

struct RoundBuf {
  PairRec* pairs;
  uint32_t* pair_src;              // index of the (target, kind) lane or survivor
  // Two sweep kernels share a round: one runs the bit-sliced pairs (outputs
  // depend on A), the other the A-independent ones; each class has its own
  // chunk numbering (pairs of the other class count zero chunks in it).
  unsigned long long* nchunks;     // per pair (scan input), bit-sliced class
  unsigned long long* cbase;       // exclusive prefix of nchunks
  unsigned long long* nchunks_x;   // per pair, A-independent class
  unsigned long long* cbase_x;     // exclusive prefix of nchunks_x
  unsigned long long* nchunks_c;   // per pair, compact class (with compact set; else unused)
  unsigned long long* cbase_c;     // exclusive prefix of nchunks_c
  uint32_t compact;                // A-dependent pairs whose registers fit the compact state get
                                   // their own class and kernel
  unsigned long long* nchunks_w;   // per pair, wide compact class (with wide set; else unused)
  unsigned long long* cbase_w;     // exclusive prefix of nchunks_w
  unsigned long long* nchunks_r;   // per pair, register-state class (with wide set; else unused)
  unsigned long long* cbase_r;     // exclusive prefix of nchunks_r
  uint32_t wide;                   // pairs whose registers fit the wide compact state (and not
                                   // the compact one) get their own class and kernel, and so do
                                   // the rest that name neither SP nor the memory byte
                                   // (register-state class)
  uint32_t* rejected;              // per pair
  uint8_t* wlen;                   // per pair: survivors in the window it heads (0: not a head)
  // First-found windows (null for independent pairs): per pair the end
  // (exclusive) of its survivor window, and the chunks of its sweep that
  // finished without a mismatch.  A pair whose every chunk finished so
  // passed; the pairs after it in its window can no longer win, and their
  // sweeps are cancelled (rejected = 2).
  uint32_t* wend;
  uint32_t* cdone;
  uint32_t cap;                    // pair slots of the buffers
  uint32_t* npairs;                // device counter
  unsigned long long* counter;     // chunk dispensers: [0] bit-sliced, [1] A-independent, [2] compact,
                                   // [3] wide compact, [4] register-state class
  unsigned long long* states;      // [2]: states of the reference's sweeps covered, states evaluated
  uint32_t chunk_blocks;           // A-blocks per work chunk
  uint32_t xunit;                  // A-blocks per unit of an A-independent sweep: kXBitsBlocks
                                   // (bit-sliced kernel), else (0 too) the scalar kernel's 128
};

// Length-2 candidate pass (pair pool): bucket indexes and per-lane slots.
constexpr uint32_t kSlots2 = 32;  // survivors held per (target, kind) lane
struct PairScan {
  const unsigned long long* const* idx;  // [64] sorted bucket keys per dead-register mask
  uint32_t n_valid;                      // entries of each index (the unpruned pairs)
  // The same indexes over the unpruned pairs of at most 2 and at most 3
  // bytes ([64] each, in the same order): a target of 3 or 4 bytes can only
  // take those, and its bucket in the full index is nearly all longer pairs.
  const unsigned long long* const* idx_le2;
  const unsigned long long* const* idx_le3;
  uint32_t n_le2, n_le3;
  uint32_t* cnt;                         // [2n] survivors in the lane's slots
  uint32_t* resume;                      // [2n] bucket offset to rescan from; kNone: exhausted
  uint32_t* surv;                        // [2n * kSlots2] pair-pool indices
  uint16_t* sdiff;                       // [2n * kSlots2]
  uint32_t* refill;                      // lanes waiting for a rescan (round build)
  const unsigned long long* eligible;    // [16] unpruned pairs shorter than b bytes
  unsigned long long* checks;            // QuickCheck units (eligible pairs per target)
};

struct DevRule {
  uint32_t target;
  uint32_t cand;
  uint16_t diff;   // flag diff | reg diff << 8
  uint8_t kind;    // 0 full, 1 masked, 2 all-hits
  uint8_t clen;    // candidate length: 1 (pool index) or 2 (pair-pool index)
};

// Moves the survivors the count pass kept (targets with 1..kQCSlots) to
// their places after base[t]: the full ones first, then the masked ones,
// each in enumeration order.
void launch_qc_compact(const QCOut& q, uint32_t n, cudaStream_t s);
void dev_upload_tables(cudaStream_t s);
int dev_num_sms();

void launch_pool_outputs(const uint32_t* insn, uint32_t n, uint32_t len, uint4* qc, uint4* mid,
                         cudaStream_t s);
void launch_exec(const uint32_t* in_states, const uint32_t* seqs, const uint8_t* lens, uint32_t len,
                 uint32_t stride, uint32_t n, uint32_t* out_states, cudaStream_t s);
void launch_fingerprints(const uint32_t* seqs, uint32_t n, uint32_t len, uint8_t* out, cudaStream_t s);
void launch_qc_scan(const DevTargets& T, const DevPool& P, const QCConfig& cfg, const QCOut& o,
                    bool collect, cudaStream_t s);
void launch_fp_query(const DevPool& P, const uint32_t* fp3x8, uint32_t dead, uint32_t* hits,
                     uint32_t* nhits, uint32_t cap, cudaStream_t s);
void launch_qc_keys(const DevPool& P, uint32_t w2mask, unsigned long long* keys, cudaStream_t s);
void launch_qc_top(const unsigned long long* keys, uint32_t nv, uint32_t* top, cudaStream_t s);
void launch_qc_bucket(const DevTargets& T, const DevPool& P, const QCConfig& cfg, const QCIndex& ix,
                      const QCOut& o, bool collect, cudaStream_t s);
void launch_round_build(const DevTargets& T, const DevPool& P, const QCOut& q, const Lanes& L,
                        const RoundBuf& R, cudaStream_t s);
void launch_pairs_from_survivors(const DevTargets& T, const DevPool& P, const QCOut& q,
                                 const uint8_t* midpass, uint32_t nsurv, const uint32_t* surv_target,
                                 const RoundBuf& R, cudaStream_t s);
// k = states per lane per dispatch: 1, 2, 4 or 8.
// Launches the sweep kernel of each class that has chunks (total_b
// bit-sliced, total_x A-independent, total_c compact); returns the number of
// launches and ORs the launched instantiations into *kernels (may be NULL):
// kSweep* bits.
constexpr uint32_t kSweepBits = 1u, kSweepXBits = 2u, kSweepCompact = 4u;
constexpr uint32_t kSweepScalarK1 = 8u;  // scalar A-independent kernel, K = 1, 2, 4, 8: bits 3..6
constexpr uint32_t kSweepWide = 128u, kSweepRegs = 256u;
int launch_exhaustive(const DevTargets& T, const DevPool& P, const RoundBuf& R, uint32_t npairs,
                      unsigned long long total_b, unsigned long long total_x, unsigned long long total_c,
                      unsigned long long total_w, unsigned long long total_r, int k, cudaStream_t s,
                      uint32_t* kernels = nullptr);
void launch_round_resolve(const RoundBuf& R, uint32_t npairs, const QCOut& q, const Lanes& L, uint32_t max_spec,
                          cudaStream_t s);

// ---- device-driven rounds (one CUDA graph, a WHILE node over the round body)
// The round's pair count and chunk totals stay on the device: the round
// scan (three launches) takes the count the build left in R.npairs, scans
// the chunk counts of the five classes (per-block segment sums in bsum, then
// each segment from its blocks' offset), clears the dispensers and ends the
// loop (sets the graph's condition to 0) when the round is empty and no lane
// waits for a rescan.
constexpr int kRScanBlocks = 256;
struct RoundCtl {
  unsigned long long totals[5];  // chunks of the current round: bit-sliced, A-independent, compact, wide,
                                 // register state
  unsigned long long pairs;      // pairs swept, all rounds
  uint32_t rounds;               // rounds with pairs
  uint32_t iters;                // loop iterations (rounds, rescans, the last empty one)
  uint32_t np;                   // pairs of the current round
  uint32_t overrun;              // set when the loop stopped at kMaxRoundIters (an error)
  unsigned long long bsum[5][kRScanBlocks];  // the current round's chunks per class and scan block
};
// Bound on the iterations of one device-driven loop: a loop that has not
// ended by then stops and reports an error instead of running on.
constexpr uint32_t kMaxRoundIters = 1u << 20;
void launch_round_scan(const RoundBuf& R, RoundCtl* ctl, const uint32_t* refill, cudaGraphConditionalHandle loop,
                       cudaStream_t s);
// The sweep kernels of the configured classes on persistent grids, the
// chunk totals and pair count read from ctl; returns the launches per round.
// ss[0..4]: the streams of the register-state, wide, compact, bit-sliced
// and A-independent classes (the classes share no chunk, pair or
// dispenser, so their launches may run side by side: one class's blocks
// take the SMs that another's finished blocks leave).
int launch_exhaustive_dev(const DevTargets& T, const DevPool& P, const RoundBuf& R, const RoundCtl* ctl, int k,
                          const cudaStream_t* ss);
// Sets up (outside any stream capture) the launch facts of the kernels
// launch_exhaustive_dev will launch for R and k.
void warm_exhaustive_dev(const RoundBuf& R, int k);
// k_round_resolve over the pair slots, the pair count read from ctl.
void launch_round_resolve_dev(const RoundBuf& R, const RoundCtl* ctl, const QCOut& q, const Lanes& L,
                              uint32_t max_spec, cudaStream_t s);
// k_pair_scan that does its work only when the current round is empty (the
// rescan step of the length-2 pass).
void launch_pair_scan_gated(const DevTargets& T, const DevPool& P, const QCOut& q1, const Lanes& L2,
                            const PairScan& ps, const RoundCtl* ctl, cudaStream_t s);
void launch_midcheck(const DevTargets& T, const DevPool& P, const uint32_t* surv,
                     const uint32_t* surv_target, uint32_t nsurv, uint8_t* pass, cudaStream_t s);
void launch_surv_targets(const QCOut& q, uint32_t n, uint32_t* surv_target, cudaStream_t s);
// L2: the lanes of the length-2 candidate pass (all pointers null when the
// job stops at length 1); pool2_enum: the enumerated length-2 sequences.
void launch_rule_count_first(const Lanes& L, const Lanes& L2, uint32_t n, uint32_t* cnt, const DevTargets& T,
                             unsigned long long* checked, uint32_t pool_enum, unsigned long long pool2_enum,
                             cudaStream_t s);
void launch_rule_write_first(const Lanes& L, const Lanes& L2, uint32_t n, const uint32_t* base, DevRule* out,
                             cudaStream_t s);
void launch_rule_write_all(const uint32_t* flag, const uint32_t* base, uint32_t nsurv,
                           const uint32_t* surv, const uint16_t* sdiff, const uint32_t* surv_target,
                           DevRule* out, cudaStream_t s);
void launch_rule_count_all(const RoundBuf& R, uint32_t npairs, uint32_t* flag, cudaStream_t s);
void launch_pair_keys(const DevPool& P, uint32_t dregs, unsigned long long* keys, cudaStream_t s);
void launch_pair_lanes_init(const DevTargets& T, const Lanes& L1, const QCOut& q1, const Lanes& L2,
                            const PairScan& ps, cudaStream_t s);
void launch_pair_scan(const DevTargets& T, const DevPool& P, const QCOut& q1, const Lanes& L2, const PairScan& ps,
                      cudaStream_t s);
void launch_pair_round_build(const DevTargets& T, const DevPool& P, const QCOut& q1, const Lanes& L2,
                             const PairScan& ps, const RoundBuf& R, cudaStream_t s);
void launch_verify_small(const uint32_t* tgt, const uint8_t* tlens, const uint32_t* cand,
                         const uint8_t* clens, uint32_t stride, uint32_t n, const uint8_t* dead,
                         uint32_t tiers, uint8_t* out, uint8_t* flagdiff, cudaStream_t s);

}  // namespace z80b
