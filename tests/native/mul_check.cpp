// Host-side comparison of the constant-multiply instruction model of the
// search kernels (z80b_mul_ops.cuh compiled as plain C++, four inputs per
// word) with the oracle's MulRunPool, on random sequences over every pool and
// every input x.  Built and run by tests/test_mulopt_host.py; exits non-zero
// on the first mismatch.
#include <cstdio>
#include <random>
#include <vector>

#include "../../oracle/z80_oracle.h"
#include "../../oracle/z80_oracle_mulopt.h"
#include "../../z80-optimizer_b200/csrc/z80b_mul_ops.cuh"

using namespace z80b::mul::ops;

template <class P>
static int check_pool(int pool, std::mt19937_64& rng, long long* checked) {
  if (P::N != orc::MulPoolSize(pool)) {
    std::printf("pool %d: size %d vs oracle %d\n", pool, P::N, orc::MulPoolSize(pool));
    return 1;
  }
  for (int i = 0; i < P::N; i++)
    if (int(cost_of<P>(i)) != orc::MulOpTStatesPool(pool, i)) {
      std::printf("pool %d op %d: %u T-states vs oracle %d\n", pool, i, cost_of<P>(i),
                  orc::MulOpTStatesPool(pool, i));
      return 1;
    }
  for (int t = 0; t < 20000; t++) {
    const int len = 1 + int(rng() % 7);
    std::vector<int> seq(static_cast<size_t>(len));
    for (auto& o : seq) o = int(rng() % P::N);
    const uint8_t b = uint8_t(rng()), c = uint8_t(rng()), f = uint8_t(rng());
    const orc::MulInit init{b, c, f};
    for (int x0 = 0; x0 < 256; x0 += 4) {
      S4 s{};
      s.a = uint32_t(x0) | uint32_t(x0 + 1) << 8 | uint32_t(x0 + 2) << 16 | uint32_t(x0 + 3) << 24;
      s.b = b * 0x01010101u;
      s.c = (pool == orc::kMulPoolWide ? c : 0) * 0x01010101u;
      s.cf = (f & 1u) * 0x01010101u;
      for (int o : seq) apply_at<P>(o, s);
      for (int j = 0; j < 4; j++) {
        const uint8_t want = orc::MulRunPool(pool, seq.data(), len, uint8_t(x0 + j), init);
        const uint8_t got = uint8_t(s.a >> (8 * j));
        ++*checked;
        if (want != got) {
          std::printf("MISMATCH pool %d x=%d b=%02X c=%02X f=%02X seq=", pool, x0 + j, b, c, f);
          for (int o : seq) std::printf("%d,", o);
          std::printf(" oracle %02X model %02X\n", want, got);
          return 1;
        }
      }
    }
  }
  return 0;
}

int main() {
  orc::Init();
  std::mt19937_64 rng(2024);
  long long checked = 0;
  if (check_pool<PGo>(orc::kMulPoolReference, rng, &checked) || check_pool<PWide>(orc::kMulPoolWide, rng, &checked) ||
      check_pool<PFast>(orc::kMulPoolFast, rng, &checked) || check_pool<PCuda>(orc::kMulPoolCuda, rng, &checked))
    return 1;
  std::printf("OK %lld\n", checked);
  return 0;
}
