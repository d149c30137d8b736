// z80b_mulopt.cuh -- constant-multiply search (cmd/mulopt) on the device.
//
// One enumeration per sequence length serves every constant K at once: a
// sequence that maps x = 1 to k is a candidate for K = k only, so instead
// of one odometer per K (cmd/mulopt/main.go:186-229) the device walks the
// N^L sequences of length L once and files each sequence that passes the
// all-256-inputs test under its own K.  Per K and length the winner is the
// minimum of (T-states, odometer index), which is the reference's rule
// (shortest length, then `c < bestCost` in odometer order).
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

namespace z80b {
namespace mul {

// Instruction pools (numbers shared with the C ABI).
enum PoolId : int { kPoolGo = 0, kPoolWide = 1, kPoolFast = 2, kPoolCuda = 3, kNumPools = 4 };

struct PoolInfo {
  int n;                 // instructions in the pool
  int max_len;           // longest length whose odometer index fits the 48-bit key
  const char* const* names;
  const uint8_t* tstates;
};
const PoolInfo& pool_info(int pool);

struct SearchArgs {
  int pool;
  uint8_t b, c, f;       // initial B, C, F (A', F' and the shadows start at 0)
  int min_len, max_len;
  uint32_t want[8];      // bit k: constant k is searched (k = 2..255)
};

struct LenStats {
  unsigned long long filter_nodes;  // warp-level nodes whose leaves passed the x=2/x=255 filter
  unsigned long long full_checks;   // all-256 tests run
  unsigned long long full_pass;     // tests passed
};

// Key of a passing sequence: tstates << 48 | odometer index.
constexpr int kKeyShift = 48;
constexpr unsigned long long kNoKey = ~0ull;

// Launches the search of one length L on `stream`.  best[k] (256 entries,
// pre-set to kNoKey) receives the minimum key per constant; `st` (device)
// accumulates the counters.  Returns the CUDA error of the launch.
cudaError_t launch_length(const SearchArgs& a, int len, unsigned long long* best, LenStats* st,
                          int sms, cudaStream_t stream);

}  // namespace mul
}  // namespace z80b
