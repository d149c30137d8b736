// Constant-multiply model of the oracle (test infrastructure only).
#pragma once
#include <cstdint>
#include <vector>

namespace orc {

// Pool identifiers (the library's C ABI uses the same numbers).
//   kMulPoolReference  cmd/mulopt/main.go's 14 ops (all state zero but A)
//   kMulPoolWide       the 21-op pool of the constant-multiply workload
//   kMulPoolFast       cuda/z80_mulopt_fast.cu's 14 ops
//   kMulPoolCuda       cuda/z80_mulopt.cu's 21 ops
enum MulPoolId { kMulPoolReference = 0, kMulPoolWide = 1, kMulPoolFast = 2, kMulPoolCuda = 3 };

// The 21-op pool of the constant-multiply workload (pkg/cpu semantics).
constexpr int kMulPoolSize = 21;
constexpr uint16_t kExAF = 0xFFFF;  // EX AF,AF' marker (not a pkg/cpu opcode)
extern const uint16_t kMulPool[kMulPoolSize];
extern const char* const kMulNames[kMulPoolSize];


struct MulInit {
  uint8_t b, c, f;
};
struct MulResult {
  int k = 0, length = 0, tstates = 0;
  std::vector<int> ops;
};

int MulPoolSize(int pool);
const char* MulOpName(int pool, int i);
int MulOpTStates(int i);
uint8_t MulRun(const int* seq, int n, uint8_t x, const MulInit& init);
bool MulTest(const int* seq, int n, uint8_t k, const MulInit& init);
bool MulFindOptimal(uint8_t k, int minLen, int maxLen, const MulInit& init, MulResult* out);

// Pool-generic forms (pool = kMulPoolReference or kMulPoolWide).
int MulOpTStatesPool(int pool, int i);
uint8_t MulRunPool(int pool, const int* seq, int n, uint8_t x, const MulInit& init);
bool MulTestPool(int pool, const int* seq, int n, uint8_t k, const MulInit& init);
bool MulFindOptimalPool(int pool, uint8_t k, int minLen, int maxLen, const MulInit& init, MulResult* out);

}  // namespace orc
