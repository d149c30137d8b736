// z80b_mulopt.cu -- constant-multiply search kernels (cmd/mulopt on the
// device; see z80b_mulopt.cuh for the search rule).
//
// The instruction model (four inputs per word) is z80b_mul_ops.cuh.
//
// Layout of the walk: four inputs x travel together as the four bytes of
// one 32-bit word per register (byte 0: x = 1, byte 1: x = 2, byte 2:
// x = 255, byte 3: x = 127), with the carry in bit 0 of each byte, so one
// instruction of a sequence costs a few 32-bit integer operations for four
// inputs.  A warp takes 32 consecutive odometer prefixes (one per lane) and
// walks the same suffix tree in lock step, so every lane dispatches the same
// instruction at the same time; the last level is unrolled per pool.  A leaf
// is filtered by one shared-memory lookup: with k = A at x = 1, the table
// row of k holds the A that x = 2, 255, 127 must give (2k, -k, 127k) when k
// is a wanted constant, and an impossible value otherwise, so constants
// already solved at a shorter length (and k = 0, 1) cost nothing further.
// The table has one copy per lane (row k, column lane), so the lookups of a
// warp never share a bank.  Survivors get the whole warp: it runs the
// sequence on all 256 inputs (8 per lane).
#include <cuda_runtime.h>

#include "z80b_mul_ops.cuh"
#include "z80b_mulopt.cuh"

namespace z80b {
namespace mul {
namespace {

constexpr unsigned FULL = 0xFFFFFFFFu;
using namespace ops;

struct Params {
  int len, plen;                 // sequence length, prefix length (L = plen + D)
  unsigned long long n_prefix;   // N^plen
  unsigned long long nd;         // N^D
  uint32_t b, c, f;
  uint32_t want[8];
  unsigned long long* best;      // [256]
  LenStats* st;
};

struct Walk {
  uint32_t pidx;                 // this lane's prefix (odometer digits 0..plen-1)
  uint32_t pcost;
  bool active;
  const uint32_t* tab;           // shared expected-A table, this lane's column
  const Params* p;
  unsigned long long n_slow, n_full, n_pass;  // warp-level counters (lane 0 adds them)
};

__device__ __forceinline__ S4 initial_state(const Params& p) {
  S4 s;
  s.a = 0x7FFF0201u;  // x = 1, 2, 255, 127
  s.b = (p.b & 0xFFu) * M1;
  s.c = (p.c & 0xFFu) * M1;
  s.cf = (p.f & 1u) * M1;
  s.as = s.bs = s.cs = s.cfs = 0;
  return s;
}

// The whole sequence (prefix digits of pidx, suffix digits of sidx) on all
// 256 inputs, 8 per lane; true on every lane iff A = x*k for every x.
template <class P, int D>
__device__ bool full_check(const Params& p, uint32_t pidx, uint32_t sidx, uint32_t k) {
  const int lane = threadIdx.x & 31;
  int dg[16];
  uint32_t v = pidx;
  for (int i = p.plen - 1; i >= 0; i--) {
    dg[i] = int(v % P::N);
    v /= P::N;
  }
  v = sidx;
  for (int i = p.plen + D - 1; i >= p.plen; i--) {
    dg[i] = int(v % P::N);
    v /= P::N;
  }
  S4 s0 = initial_state(p), s1 = s0;
  const uint32_t x0 = 8u * lane;
  s0.a = (x0 | ((x0 + 1) << 8) | ((x0 + 2) << 16) | ((x0 + 3) << 24));
  s1.a = s0.a + 0x04040404u;
  for (int i = 0; i < p.len; i++) {
    apply_at<P>(dg[i], s0);
    apply_at<P>(dg[i], s1);
  }
  uint32_t e0 = 0, e1 = 0;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    e0 |= (((x0 + j) * k) & 0xFFu) << (8 * j);
    e1 |= (((x0 + 4 + j) * k) & 0xFFu) << (8 * j);
  }
  return __all_sync(FULL, s0.a == e0 && s1.a == e1);
}

// Rare path: some lane of the warp has a leaf under this parent that passes
// the table filter.  Re-derives the N leaves and runs the full test on each
// passing leaf whose key beats the best so far, one at a time.
template <class P, int D>
__device__ __noinline__ void slow_parent(const S4& s, uint32_t sidx_parent, uint32_t scost_parent, Walk& w) {
  const Params& p = *w.p;
  const int lane = threadIdx.x & 31;
  if (lane == 0) w.n_slow++;
  for (int i = 0; i < P::N; i++) {
    S4 t = s;
    apply_at<P>(i, t);
    const uint32_t a = t.a;
    const uint32_t k = a & 0xFFu;
    const uint32_t sidx = sidx_parent * P::N + uint32_t(i);
    bool q = w.active && (a >> 8) == w.tab[k << 5];
    unsigned long long key = 0;
    if (q) {
      const unsigned long long cost = w.pcost + scost_parent + cost_of<P>(i);
      key = (cost << kKeyShift) | (uint64_t(w.pidx) * p.nd + sidx);
      q = key < *(volatile unsigned long long*)&p.best[k];
    }
    unsigned m = __ballot_sync(FULL, q);
    while (m) {
      const int j = __ffs(m) - 1;
      m &= m - 1;
      const uint32_t kj = __shfl_sync(FULL, k, j);
      const uint32_t pj = __shfl_sync(FULL, w.pidx, j);
      const unsigned long long keyj = __shfl_sync(FULL, key, j);
      if (lane == 0) w.n_full++;
      if (full_check<P, D>(p, pj, sidx, kj) && lane == 0) {
        w.n_pass++;
        atomicMin(&p.best[kj], keyj);
      }
    }
  }
}

template <class P, int I>
__device__ __forceinline__ void leaves(const S4& s, const uint32_t* tab, bool& hit) {
  if constexpr (I < P::N) {
    S4 t = s;
    apply<P::kind[I]>(t);
    hit |= (t.a >> 8) == tab[(t.a & 0xFFu) << 5];
    leaves<P, I + 1>(s, tab, hit);
  }
}

template <class P, int LVL, int D>
__device__ __forceinline__ void walk(const S4& s, uint32_t sidx, uint32_t scost, Walk& w) {
  if constexpr (LVL == D - 1) {
    bool hit = false;
    leaves<P, 0>(s, w.tab, hit);
    if (__any_sync(FULL, w.active && hit)) slow_parent<P, D>(s, sidx, scost, w);
  } else {
#pragma unroll 1
    for (int i = 0; i < P::N; i++) {
      S4 t = s;
      apply_at<P>(i, t);
      walk<P, LVL + 1, D>(t, sidx * P::N + uint32_t(i), scost + cost_of<P>(i), w);
    }
  }
}

template <class P, int D>
__global__ void __launch_bounds__(256) k_mul_length(Params p) {
  // Row k: the A of x = 2, 255, 127 (bytes 0..2) for a wanted k >= 2, else
  // all ones (no A >> 8 equals it); 32 copies of each row, one per lane.
  __shared__ uint32_t expect[256 * 32];
  for (int i = threadIdx.x; i < 256 * 32; i += blockDim.x) {
    const uint32_t k = uint32_t(i) >> 5;
    const bool wanted = k >= 2u && ((p.want[k >> 5] >> (k & 31u)) & 1u);
    expect[i] = wanted ? (((2u * k) & 0xFFu) | (((0u - k) & 0xFFu) << 8) | (((127u * k) & 0xFFu) << 16))
                       : 0xFFFFFFFFu;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const unsigned long long groups = (p.n_prefix + 31) / 32;
  const unsigned long long warps = (unsigned long long)gridDim.x * (blockDim.x / 32);
  Walk w;
  w.tab = expect + lane;
  w.p = &p;
  w.n_slow = w.n_full = w.n_pass = 0;
  for (unsigned long long g = (unsigned long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; g < groups;
       g += warps) {
    const unsigned long long pi = g * 32 + lane;
    w.active = pi < p.n_prefix;
    w.pidx = w.active ? uint32_t(pi) : 0u;
    // Prefix state: digit by digit, each pool instruction applied (warp-
    // uniformly) to the lanes whose digit it is.
    S4 s = initial_state(p);
    uint32_t pcost = 0;
    uint32_t pw = 1;
    for (int i = 1; i < p.plen; i++) pw *= P::N;
    for (int d = 0; d < p.plen; d++) {
      const int dgt = int((w.pidx / pw) % P::N);
      pw /= P::N;
      for (int i = 0; i < P::N; i++) {
        if (__any_sync(FULL, dgt == i)) {
          S4 t = s;
          apply_at<P>(i, t);
          if (dgt == i) s = t;
        }
      }
      pcost += cost_of<P>(dgt);
    }
    w.pcost = pcost;
    walk<P, 0, D>(s, 0u, 0u, w);
  }
  if (lane == 0 && (w.n_slow | w.n_full | w.n_pass)) {
    atomicAdd(&p.st->filter_nodes, w.n_slow);
    atomicAdd(&p.st->full_checks, w.n_full);
    atomicAdd(&p.st->full_pass, w.n_pass);
  }
}

template <class P>
cudaError_t launch_pool(const Params& prm, int D, int sms, cudaStream_t stream) {
  auto pick = [&](auto kernel) -> cudaError_t {
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    const unsigned long long groups = (prm.n_prefix + 31) / 32;
    unsigned long long blocks = (unsigned long long)sms * per_sm;
    const unsigned long long need = (groups + 7) / 8;
    if (need < blocks) blocks = need;
    if (blocks < 1) blocks = 1;
    kernel<<<unsigned(blocks), 256, 0, stream>>>(prm);
    return cudaGetLastError();
  };
  switch (D) {
    case 1: return pick(k_mul_length<P, 1>);
    case 2: return pick(k_mul_length<P, 2>);
    case 3: return pick(k_mul_length<P, 3>);
    case 4: return pick(k_mul_length<P, 4>);
    default: return pick(k_mul_length<P, 5>);
  }
}

const char* const kNamesGo[] = {"ADD A,A", "ADD A,B", "SUB B",   "LD B,A",  "SLA A",   "SRL A", "EX AF,AF'",
                                "EXX",     "ADC A,B", "ADC A,A", "SBC A,B", "SBC A,A", "OR A",  "NEG"};
const uint8_t kTGo[] = {4, 4, 4, 4, 8, 8, 4, 4, 4, 4, 4, 4, 4, 8};
const char* const kNamesWide[] = {"ADD A,A", "ADD A,B", "SUB B", "LD B,A", "SLA A",     "SRL A",  "RLA",
                                  "RRA",     "RLCA",    "RRCA",  "NEG",    "CPL",       "OR A",   "SCF",
                                  "CCF",     "EX AF,AF'", "LD C,A", "ADD A,C", "SUB C", "LD A,B", "LD A,C"};
const uint8_t kTWide[] = {4, 4, 4, 4, 8, 8, 4, 4, 4, 4, 8, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4};
const char* const kNamesFast[] = {"ADD A,A", "ADD A,B", "SUB B", "LD B,A", "ADC A,B", "ADC A,A", "SBC A,B",
                                  "SBC A,A", "SRL A",   "RLA",   "RRA",    "RLCA",    "RRCA",    "NEG"};
const uint8_t kTFast[] = {4, 4, 4, 4, 4, 4, 4, 4, 8, 4, 4, 4, 4, 8};
const char* const kNamesCuda[] = {"ADD A,A", "ADD A,B", "SUB B", "LD B,A", "ADC A,B", "ADC A,A", "SBC A,B",
                                  "SBC A,A", "SLA A",   "SRA A", "SRL A",  "RLA",     "RRA",     "RLCA",
                                  "RRCA",    "RLC A",   "RRC A", "OR A",   "NEG",     "SCF",     "EX AF,AF'"};
const uint8_t kTCuda[] = {4, 4, 4, 4, 4, 4, 4, 4, 8, 8, 8, 4, 4, 4, 4, 8, 8, 4, 8, 4, 4};

// Longest length whose odometer index N^L stays below 2^48.
constexpr int max_len_for(int n) {
  int l = 0;
  unsigned long long v = 1;
  while (v * n < (1ull << kKeyShift)) {
    v *= n;
    l++;
  }
  return l;
}

const PoolInfo kInfo[kNumPools] = {{14, max_len_for(14), kNamesGo, kTGo},
                                   {21, max_len_for(21), kNamesWide, kTWide},
                                   {14, max_len_for(14), kNamesFast, kTFast},
                                   {21, max_len_for(21), kNamesCuda, kTCuda}};

// Split of length L into a prefix walked per lane and a suffix of D levels:
// at least ~1M prefixes when L allows (load balance over all SMs), D <= 5.
void split(int n, int len, int* plen, int* d) {
  int pt = 0;
  unsigned long long v = 1;
  while (v < (1ull << 20)) {
    v *= n;
    pt++;
  }
  int p = len - 1 < pt ? len - 1 : pt;
  int dd = len - p;
  if (dd > 5) {
    dd = 5;
    p = len - 5;
  }
  *plen = p;
  *d = dd;
}

}  // namespace

const PoolInfo& pool_info(int pool) { return kInfo[pool]; }

cudaError_t launch_length(const SearchArgs& a, int len, unsigned long long* best, LenStats* st, int sms,
                          cudaStream_t stream) {
  const PoolInfo& pi = kInfo[a.pool];
  Params p{};
  p.len = len;
  int D = 1;
  split(pi.n, len, &p.plen, &D);
  p.n_prefix = 1;
  for (int i = 0; i < p.plen; i++) p.n_prefix *= pi.n;
  p.nd = 1;
  for (int i = 0; i < D; i++) p.nd *= pi.n;
  p.b = a.b;
  p.c = a.c;
  p.f = a.f;
  for (int i = 0; i < 8; i++) p.want[i] = a.want[i];
  p.best = best;
  p.st = st;
  switch (a.pool) {
    case kPoolGo: return launch_pool<PGo>(p, D, sms, stream);
    case kPoolWide: return launch_pool<PWide>(p, D, sms, stream);
    case kPoolFast: return launch_pool<PFast>(p, D, sms, stream);
    default: return launch_pool<PCuda>(p, D, sms, stream);
  }
}

}  // namespace mul
}  // namespace z80b
