// z80b_noalloc.cu -- ExhaustiveCheck for callers that cannot allocate.
//
// Some callers of this library cannot call cudaMalloc.  A process whose
// device memory is budgeted by another component (a serving framework that
// pre-reserves the GPU and fails foreign allocations), code on a latency
// path that must not pay for an allocation or the device-wide
// synchronization cudaFree implies, or a plugin host whose rules forbid
// allocator calls.  z80b_exhaustive_noalloc serves them: it needs no context
// and performs no allocation, neither on the device nor on the host heap.
// Its device scratch is the file-scope array below, kNoAllocBytes in size,
// which every GPU that loads the library holds until the process exits; its
// host staging is static as well.  The caller passes host arrays for the
// pairs and for the results.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/z80b200.h"
#include "z80_tables.h"
#include "z80b_kernels.cuh"

namespace z80b {
namespace {

constexpr uint32_t kMaxPairs = Z80B_NOALLOC_MAX_PAIRS;
constexpr uint32_t kStride = 4;  // words per sequence inside the scratch

// Device scratch layout (byte offsets, each 256-aligned).
constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffTgt = 0;
constexpr size_t kOffCand = align256(kOffTgt + 4ull * kStride * kMaxPairs);
constexpr size_t kOffTLen = align256(kOffCand + 4ull * kStride * kMaxPairs);
constexpr size_t kOffCLen = align256(kOffTLen + kMaxPairs);
constexpr size_t kOffDead = align256(kOffCLen + kMaxPairs);
constexpr size_t kOffPairs = align256(kOffDead + kMaxPairs);
constexpr size_t kOffCbase = align256(kOffPairs + sizeof(PairRec) * kMaxPairs);
constexpr size_t kOffCbaseX = align256(kOffCbase + 8ull * kMaxPairs);
constexpr size_t kOffRej = align256(kOffCbaseX + 8ull * kMaxPairs);
constexpr size_t kOffCounter = align256(kOffRej + 4ull * kMaxPairs);
constexpr size_t kOffStates = kOffCounter + 16;
constexpr size_t kNoAllocBytes = align256(kOffStates + 16);
static_assert(kNoAllocBytes <= 320 * 1024, "the scratch stays modest");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Host staging, also static; g_mu serializes calls so they share it safely.
std::mutex g_mu;
uint32_t h_tgt[kStride * kMaxPairs], h_cand[kStride * kMaxPairs], h_rej[kMaxPairs];
PairRec h_pairs[kMaxPairs];
unsigned long long h_cbase[kMaxPairs], h_cbase_x[kMaxPairs];  // chunk prefixes: bit-sliced / A-independent pairs

constexpr int kMaxDevices = 64;
unsigned char* g_dev_ptr[kMaxDevices] = {};  // device address of the scratch on each device

// Once per device, with that device current: the device address of the
// scratch array (in host code its name is only a host-side stand-in) and the
// constant tables of the sweep kernel.  Caller holds g_mu.
int setup_device(int device, cudaStream_t s, unsigned char** out) {
  if (!g_dev_ptr[device]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return Z80B_ECUDA;
    dev_upload_tables(s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return Z80B_ECUDA;
    g_dev_ptr[device] = static_cast<unsigned char*>(p);
  }
  *out = g_dev_ptr[device];
  return Z80B_OK;
}

// The device part of z80b_exhaustive_noalloc, with `device` current and the
// host staging (h_tgt, h_cand, h_pairs, chunk prefixes) filled; g_mu held.
int run_on_device(int device, uint32_t n, const uint8_t* tlens, const uint8_t* clens, const uint8_t* dead,
                  unsigned long long total, unsigned long long total_x, cudaStream_t s, uint8_t* pass) {
  unsigned char* base = nullptr;
  int r = setup_device(device, s, &base);
  if (r != Z80B_OK) return r;

  // The scratch keeps whatever the previous call left in it: the rejection
  // flags and the work counters, which must start at zero, are cleared here.
  // Calls in one process are serialized by g_mu and return only after their
  // stream has finished, so their GPU work never overlaps; work enqueued by
  // any other route that touched this array (e.g. a captured graph replayed
  // later) would race with a call on it.
  bool ok = cudaMemcpyAsync(base + kOffTgt, h_tgt, 4ull * kStride * n, cudaMemcpyHostToDevice, s) == cudaSuccess &&
            cudaMemcpyAsync(base + kOffCand, h_cand, 4ull * kStride * n, cudaMemcpyHostToDevice, s) == cudaSuccess &&
            cudaMemcpyAsync(base + kOffTLen, tlens, n, cudaMemcpyHostToDevice, s) == cudaSuccess &&
            cudaMemcpyAsync(base + kOffCLen, clens, n, cudaMemcpyHostToDevice, s) == cudaSuccess &&
            cudaMemcpyAsync(base + kOffPairs, h_pairs, sizeof(PairRec) * n, cudaMemcpyHostToDevice, s) == cudaSuccess &&
            cudaMemcpyAsync(base + kOffCbase, h_cbase, 8ull * n, cudaMemcpyHostToDevice, s) == cudaSuccess &&
            cudaMemcpyAsync(base + kOffCbaseX, h_cbase_x, 8ull * n, cudaMemcpyHostToDevice, s) == cudaSuccess &&
            cudaMemsetAsync(base + kOffRej, 0, 4ull * n, s) == cudaSuccess &&
            cudaMemsetAsync(base + kOffCounter, 0, 32, s) == cudaSuccess;
  if (dead) ok = ok && cudaMemcpyAsync(base + kOffDead, dead, n, cudaMemcpyHostToDevice, s) == cudaSuccess;
  else ok = ok && cudaMemsetAsync(base + kOffDead, 0, n, s) == cudaSuccess;
  if (!ok) return Z80B_ECUDA;

  DevTargets T{};
  T.insn = reinterpret_cast<const uint32_t*>(base + kOffTgt);
  T.len = base + kOffTLen;
  T.dead = base + kOffDead;
  T.n = n;
  T.stride = kStride;
  DevPool P{};
  P.insn = reinterpret_cast<const uint32_t*>(base + kOffCand);
  P.lens = base + kOffCLen;
  P.n = n;
  P.stride = kStride;
  RoundBuf R{};
  R.pairs = reinterpret_cast<PairRec*>(base + kOffPairs);
  R.cbase = reinterpret_cast<unsigned long long*>(base + kOffCbase);
  R.cbase_x = reinterpret_cast<unsigned long long*>(base + kOffCbaseX);
  R.rejected = reinterpret_cast<uint32_t*>(base + kOffRej);
  R.counter = reinterpret_cast<unsigned long long*>(base + kOffCounter);
  R.states = reinterpret_cast<unsigned long long*>(base + kOffStates);
  R.chunk_blocks = 32;
  launch_exhaustive(T, P, R, n, total, total_x, 0, 0, 0, 4, s);
  if (cudaGetLastError() != cudaSuccess) return Z80B_ECUDA;
  if (cudaMemcpyAsync(h_rej, base + kOffRej, 4ull * n, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return Z80B_ECUDA;
  for (uint32_t i = 0; i < n; i++) pass[i] = h_rej[i] ? 0 : 1;
  return Z80B_OK;
}

}  // namespace
}  // namespace z80b

using namespace z80b;

extern "C" int z80b_exhaustive_noalloc(int device, const uint32_t* tgt, const uint8_t* tlens, const uint32_t* cand,
                                       const uint8_t* clens, uint32_t stride, uint32_t n, const uint8_t* dead,
                                       uint8_t* pass, void* stream) {
  if (n > kMaxPairs) return Z80B_ECAPACITY;
  if (n == 0) return Z80B_OK;
  if (!tgt || !tlens || !cand || !clens || !pass || stride < 1 || stride > kStride) return Z80B_EINVAL;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return Z80B_ENODEV;
  if (device < 0 || device >= ndev || device >= kMaxDevices) return Z80B_EINVAL;
  std::lock_guard<std::mutex> lock(g_mu);
  // Sequences repacked to the scratch stride; per pair the sweep shape
  // (pkg/search/verifier.go:159-171,428-476) and the chunk prefix.
  std::memset(h_tgt, 0, 4ull * kStride * n);
  std::memset(h_cand, 0, 4ull * kStride * n);
  unsigned long long total = 0, total_x = 0;
  for (uint32_t i = 0; i < n; i++) {
    const uint32_t tl = tlens[i], cl = clens[i];
    if (tl < 1 || tl > kStride || tl > stride || cl < 1 || cl > 3 || cl > stride) return Z80B_EINVAL;
    for (uint32_t k = 0; k < tl; k++) {
      const uint32_t w = tgt[size_t(i) * stride + k];
      if (insn_op(w) >= kNumOps) return Z80B_EINVAL;
      h_tgt[size_t(i) * kStride + k] = w;
    }
    for (uint32_t k = 0; k < cl; k++) {
      const uint32_t w = cand[size_t(i) * stride + k];
      if (insn_op(w) >= kNumOps) return Z80B_EINVAL;
      h_cand[size_t(i) * kStride + k] = w;
    }
    const uint16_t rd =
        uint16_t(seq_reads(&h_tgt[size_t(i) * kStride], int(tl)) | seq_reads(&h_cand[size_t(i) * kStride], int(cl)));
    PairRec& p = h_pairs[i];
    std::memset(&p, 0, sizeof p);
    p.target = i;
    p.cand = i;
    p.reads = rd;
    p.nblocks = sweep_for(rd).states / 256;
    p.keepF = uint8_t(~(dead ? dead[i] : 0u));
    p.keepR = 0x3F;
    // sweep units (see the sweep kernel): 128 A-blocks for A-independent
    // pairs, 4 A-blocks (bit-sliced) for the others
    unsigned long long units = (p.nblocks + 3) / 4;
    if (seq_aflow(&h_tgt[size_t(i) * kStride], int(tl)) && seq_aflow(&h_cand[size_t(i) * kStride], int(cl))) {
      p.keepR |= 0x40;
      units = (p.nblocks + 127) / 128;
    }
    unsigned long long ch = (units + 31) / 32;
    if (ch > (1ull << 20)) ch = 1ull << 20;
    h_cbase[i] = total;
    h_cbase_x[i] = total_x;
    if (p.keepR & 0x40) total_x += ch;
    else total += ch;
  }
  // The work runs with `device` current; the caller's current device is
  // put back on every return path below.
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return Z80B_ECUDA;
  if (prev != device && cudaSetDevice(device) != cudaSuccess) return Z80B_ECUDA;
  const int r = run_on_device(device, n, tlens, clens, dead, total, total_x, static_cast<cudaStream_t>(stream),
                              pass);
  if (prev != device && cudaSetDevice(prev) != cudaSuccess && r == Z80B_OK) return Z80B_ECUDA;
  return r;
}
