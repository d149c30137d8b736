// Checks of the ranged target enumeration of the host API
// (search::EnumerateTargets): whole ranges against the library's full
// enumeration, split ranges and batch sizes, the length-2 sample against
// Floyd's algorithm over the unpruned indices, and length-3 ranges against
// the CPU oracle's pruner.  Needs no device.  Built and run by
// tests/test_export.py.
#include <algorithm>
#include <cstdio>
#include <random>
#include <set>

#include "../../oracle/z80_oracle.h"
#include "search_api.h"

using namespace z80opt;

static int fails = 0;
#define CHECK(c)                                       \
  do {                                                 \
    if (!(c)) {                                        \
      std::printf("FAIL line %d: %s\n", __LINE__, #c); \
      fails++;                                         \
    }                                                  \
  } while (0)

static std::vector<uint32_t> collect(int len, int a, int b, uint64_t sample, uint64_t seed, uint64_t batch,
                                     std::vector<uint64_t>* sizes = nullptr) {
  std::vector<uint32_t> all;
  search::EnumerateTargets(len, a, b, sample, seed, batch, [&](const std::vector<uint32_t>& w, uint64_t n) {
    if (w.size() != n * uint64_t(len)) fails++;
    all.insert(all.end(), w.begin(), w.end());
    if (sizes) sizes->push_back(n);
  });
  return all;
}

int main() {
  orc::Init();
  std::vector<uint32_t> pool(4531);
  pool.resize(z80b_pool8(pool.data(), uint32_t(pool.size())));
  const uint32_t P = uint32_t(pool.size());
  // length 2, whole range = the library's enumeration
  const uint64_t total = z80b_enumerate(pool.data(), P, 2, nullptr, 0);
  std::vector<uint32_t> ref(total * 2);
  z80b_enumerate(pool.data(), P, 2, ref.data(), total);
  CHECK(collect(2, 0, -1, 0, 0, 1u << 22) == ref);
  // split ranges and odd batch sizes give the same sequence
  std::vector<uint64_t> sizes;
  std::vector<uint32_t> a = collect(2, 0, 1000, 0, 0, 777777, &sizes);
  const std::vector<uint32_t> b = collect(2, 1000, int(P) + 50, 0, 0, 1u << 20);
  a.insert(a.end(), b.begin(), b.end());
  CHECK(a == ref);
  for (size_t i = 0; i + 1 < sizes.size(); i++) CHECK(sizes[i] == 777777);
  CHECK(collect(2, 300, 300, 0, 0, 10).empty());
  // length-2 sample: Floyd's algorithm over the unpruned indices, index order
  {
    const uint64_t sample = 5000, seed = 9;
    std::mt19937_64 rng(seed);
    std::vector<uint64_t> pick;
    std::vector<uint8_t> taken(total, 0);
    for (uint64_t j = total - sample; j < total; j++) {
      uint64_t t = std::uniform_int_distribution<uint64_t>(0, j)(rng);
      if (taken[t]) t = j;
      taken[t] = 1;
      pick.push_back(t);
    }
    std::sort(pick.begin(), pick.end());
    std::vector<uint32_t> want;
    for (uint64_t t : pick) want.insert(want.end(), ref.begin() + long(2 * t), ref.begin() + long(2 * t + 2));
    CHECK(collect(2, 0, -1, sample, seed, 1000) == want);
  }
  // length 3, one first instruction: the oracle's unpruned sequences, in order
  {
    const auto& I = orc::Instructions8();
    const int f = 2000;
    std::vector<uint32_t> want;
    orc::Instruction s[3];
    s[0] = I[size_t(f)];
    for (uint32_t j = 0; j < P; j++)
      for (uint32_t k = 0; k < P; k++) {
        s[1] = I[j];
        s[2] = I[k];
        if (!orc::ShouldPrune(s, 3))
          for (auto& x : s) want.push_back(uint32_t(x.op) | uint32_t(x.imm) << 16);
      }
    CHECK(collect(3, f, f + 1, 0, 0, 1u << 22) == want);
    // a sample of that range: distinct, in order, unpruned, repeatable
    const std::vector<uint32_t> smp = collect(3, f, f + 1, 3000, 4, 512);
    CHECK(smp.size() == 3 * 3000);
    CHECK(smp == collect(3, f, f + 1, 3000, 4, 1u << 20));
    std::set<std::vector<uint32_t>> seen;
    size_t pos = 0;
    for (size_t i = 0; i < smp.size(); i += 3) {
      std::vector<uint32_t> t(smp.begin() + long(i), smp.begin() + long(i + 3));
      seen.insert(t);
      auto it = std::search(want.begin() + long(pos), want.end(), t.begin(), t.end());
      while (it != want.end() && (it - want.begin()) % 3 != 0) it = std::search(it + 1, want.end(), t.begin(), t.end());
      CHECK(it != want.end());
      if (it != want.end()) pos = size_t(it - want.begin()) + 3;
    }
    CHECK(seen.size() == 3000);
  }
  // length 1: the unpruned instructions of the range; a sample as large as
  // the range is the whole range
  {
    const uint64_t t1 = z80b_enumerate(pool.data(), P, 1, nullptr, 0);
    std::vector<uint32_t> r1(t1);
    z80b_enumerate(pool.data(), P, 1, r1.data(), t1);
    CHECK(collect(1, 0, -1, 0, 0, 100) == r1);
    CHECK(collect(1, 0, -1, t1 + 5, 3, 100) == r1);
    std::vector<uint32_t> part;
    for (uint32_t w : r1)
      for (uint32_t i = 10; i < 20; i++)
        if (pool[i] == w) part.push_back(w);
    CHECK(collect(1, 10, 20, 0, 0, 3) == part);
  }
  // a length-2 sample of a sub-range comes from that range only, in order,
  // without repeats
  {
    const std::vector<uint32_t> sub = collect(2, 40, 45, 0, 0, 1u << 20);
    const std::vector<uint32_t> smp = collect(2, 40, 45, 700, 8, 64);
    CHECK(smp.size() == 1400);
    size_t pos = 0;
    bool ordered = true;
    for (size_t i = 0; i < smp.size(); i += 2) {
      while (pos < sub.size() && !(sub[pos] == smp[i] && sub[pos + 1] == smp[i + 1])) pos += 2;
      if (pos >= sub.size()) ordered = false;
      pos += 2;
    }
    CHECK(ordered);
  }
  // bad arguments
  bool threw = false;
  try {
    collect(4, 0, 1, 0, 0, 10);
  } catch (const Error&) {
    threw = true;
  }
  CHECK(threw);
  threw = false;
  try {
    collect(3, 0, 1, 20000000, 0, 10);
  } catch (const Error&) {
    threw = true;
  }
  CHECK(threw);
  if (fails) return 1;
  std::printf("OK\n");
  return 0;
}
