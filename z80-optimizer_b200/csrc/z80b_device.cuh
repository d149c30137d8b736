// z80b_device.cuh -- device-side data layout shared by the kernels.
#pragma once
#include <cstdint>

#include "z80_exec.cuh"

namespace z80b {

// Max instructions per sequence handled by the kernels (targets up to 4,
// candidates up to 3).
constexpr int kMaxSeq = 4;
constexpr uint32_t kNone = 0xFFFFFFFFu;

// Candidate table resident in HBM.  Outputs are stored vector-major so a warp
// scanning consecutive candidates on one vector issues coalesced 16-byte
// loads: out[v * n + c] = {A|F<<8|B<<16|C<<24, D|E<<8|H<<16|L<<24, SP|M<<16, 0}.
struct DevPool {
  const uint32_t* insn;    // n * stride packed instructions
  const uint4* qc;         // 8 * n
  const uint4* mid;        // 32 * n (may be null)
  const uint8_t* size;     // encoded bytes of the whole sequence
  const uint8_t* prune;    // ShouldPrune(candidate)
  const uint16_t* reads;   // regsRead(candidate)
  const uint8_t* lens;     // per-candidate length or null (len)
  uint32_t n, len, stride;
};

__device__ __forceinline__ uint32_t pool_len(const DevPool& P, uint32_t c) {
  return P.lens ? P.lens[c] : P.len;
}

// A batch of targets.
struct DevTargets {
  const uint32_t* insn;     // n * stride
  const uint8_t* len;       // per-target length or null (fixed_len)
  const uint8_t* dead;      // per-target dead-flag mask or null (global_dead)
  const uint8_t* dead_regs; // per-target dead-register mask (bit0..5 = B,C,D,E,H,L) or null
  uint32_t n, stride, fixed_len;
  uint32_t global_dead;
};

// Per-target metadata written by the QuickCheck count pass.
struct TargetMeta {
  uint16_t tstates;
  uint8_t bytes;
  uint8_t len;
  uint16_t reads;
  uint16_t pad;
};

// One ExhaustiveCheck work unit: pair (target, candidate) of a round.
struct PairRec {
  unsigned long long nblocks;  // A-blocks (256 states each) in the sweep
  uint32_t target;
  uint32_t cand;       // pool index
  uint16_t reads;      // union of regsRead
  uint8_t keepF;       // ~deadFlags
  uint8_t keepR;       // bits 0..5: register compared (B,C,D,E,H,L); bit 7: masked pass
  uint8_t cmap;        // compact sweep: 1 + the register-set entry of its tables; 0: full state
  // Swept registers left out because no compared output of either program
  // depends on them (reads holds the ones swept): bit 7 the reference's
  // sweep of this pair is a reduced one (32 values per register), bits 0..5
  // log2 of the reference states each evaluated state stands for.
  uint8_t sweepf;
};

__device__ __forceinline__ uint32_t target_len(const DevTargets& T, uint32_t t) {
  return T.len ? T.len[t] : T.fixed_len;
}
__device__ __forceinline__ uint32_t target_dead(const DevTargets& T, uint32_t t) {
  return T.dead ? T.dead[t] : T.global_dead;
}
__device__ __forceinline__ uint32_t target_dead_regs(const DevTargets& T, uint32_t t) {
  return T.dead_regs ? T.dead_regs[t] : 0u;
}

}  // namespace z80b
