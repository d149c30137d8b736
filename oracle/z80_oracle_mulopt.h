// Constant-multiply model of the oracle (test infrastructure only).
#pragma once
#include <cstdint>
#include <vector>

namespace orc {

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

int MulOpTStates(int i);
uint8_t MulRun(const int* seq, int n, uint8_t x, const MulInit& init);
bool MulTest(const int* seq, int n, uint8_t k, const MulInit& init);
bool MulFindOptimal(uint8_t k, int minLen, int maxLen, const MulInit& init, MulResult* out);

}  // namespace orc
