// z80b_engine.cu -- context, pipeline orchestration and the C ABI of
// libz80b200.so (declared in include/z80b200.h).
//
// The batched pipeline of one job (first-found semantics, pkg/search
// worker.go:124-265):
//   1. QuickCheck count pass   (k_qc_scan<false>)  survivors per target
//   2. exclusive scan          -> contiguous per-target survivor ranges
//   3. QuickCheck collect pass (k_qc_scan<true>)   survivors in enumeration order
//   4. rounds: each unresolved (target, pass) lane offers its next survivor;
//      ExhaustiveCheck of all offered pairs at once; a passing pair resolves
//      its lane (first passing survivor in enumeration order = the
//      reference's first found), a failing one advances it.
//   5. rule compaction in target order.
// The all-hits pipeline (pkg/gpu/search.go:80-199) replaces 4 by MidCheck on
// every survivor and one ExhaustiveCheck pass over the MidCheck survivors.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#if defined(__SSE2__)
#include <emmintrin.h>
#endif

#include "../../include/z80b200.h"
#include "z80_tables.h"
#include "z80b_kernels.cuh"
#include "z80b_engine.h"
#include "z80b_mulopt.cuh"

using namespace z80b;

namespace {

struct DBuf {
  void* p = nullptr;
  size_t bytes = 0;
  ~DBuf() {
    if (p) cudaFree(p);
  }
  cudaError_t ensure(size_t b) {
    if (b <= bytes && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    size_t want = std::max<size_t>(b, 256);
    cudaError_t e = cudaMalloc(&p, want);
    if (e == cudaSuccess) bytes = want;
    return e;
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

// Pinned host memory (device-to-host copies run as DMA at full speed).
struct HBuf {
  void* p = nullptr;
  size_t bytes = 0;
  ~HBuf() {
    if (p) cudaFreeHost(p);
  }
  cudaError_t ensure(size_t b) {
    if (b <= bytes && p) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    size_t want = std::max<size_t>(b, 4096);
    cudaError_t e = cudaHostAlloc(&p, want, cudaHostAllocDefault);
    if (e == cudaSuccess) bytes = want;
    return e;
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

struct PoolBufs {
  DBuf insn, qc, mid, size, prune, reads, lens;
  // QuickCheck bucket index (pools of at most kQCIndexMax candidates)
  DBuf qkeys, qkeys_tmp, qtop, qelig, qsort_tmp;
  int qstate = 0;          // 0 not built, 1 built, -1 pool too large
  uint32_t qw2 = 0;        // word-2 mask the index hashes
  DevPool dev{};
  std::vector<uint32_t> host_insn;
  std::vector<uint8_t> host_lens;
  uint32_t n = 0, len = 0;
  bool loaded = false;
};

struct Reporter;

// What a pipeline run needs to know about its job beyond the device arrays.
struct PipeOpts {
  uint32_t mode = Z80B_MODE_FIRST;
  uint32_t max_cand = 1;        // longest candidate (1 or 2 instructions)
  uint64_t dreg_masks = 1;      // bit m: dead-register mask m occurs in a masked pass (bit 0 always)
  bool no_exhaustive = false;   // all-hits mode: MidCheck survivors are the rules (Z80B_JOB_NO_EXHAUSTIVE)
  Reporter* rep = nullptr;      // per-target answers as they become final (first-found mode)
  // Targets uploaded in chunks on the copy stream (z80b_search on large
  // jobs): chunk k holds targets [up_hi[k-1], up_hi[k]) and is complete at
  // the context's up_ev[k]; the QuickCheck count runs chunk by chunk behind
  // the copies.  0: the targets are on the device before the pipeline starts.
  int up_chunks = 0;
  const uint32_t* up_hi = nullptr;
};
constexpr int kUpChunks = 4;
constexpr uint32_t kUpChunkMin = 1u << 16;  // targets; smaller jobs upload in one copy

// The 4,531^2 pair pool, its QuickCheck outputs and its bucket indexes (one
// per dead-register mask, built on first use).  Read-only once built, so all
// contexts of a device share one copy; mu serializes the builds.
struct PairShared {
  std::mutex mu;
  PoolBufs pool;
  uint32_t valid = 0;                          // unpruned pairs
  std::vector<unsigned long long> eligible;    // [16] unpruned pairs shorter than b bytes
  DBuf idx[64];
  bool ok[64] = {};
  DBuf ptrs, eligible_dev, keys_tmp, sort_tmp;
  // the indexes restricted to unpruned pairs of at most 2 / 3 bytes
  uint32_t n_le[2] = {0, 0};
  DBuf idx_le[2][64];
  DBuf ptrs_le[2], sel_tmp, sel_count;
};

std::mutex g_pairs_mu;
std::map<int, std::weak_ptr<PairShared>> g_pairs;

std::shared_ptr<PairShared> pair_shared(int device) {
  std::lock_guard<std::mutex> lk(g_pairs_mu);
  std::shared_ptr<PairShared> p = g_pairs[device].lock();
  if (!p) {
    p = std::make_shared<PairShared>();
    g_pairs[device] = p;
  }
  return p;
}

struct Staged {
  PipeOpts opts;
  std::vector<uint32_t> targets;
  std::vector<uint8_t> lens, dead, dregs;
  z80b_job job{};
  bool valid = false;
  DBuf d_targets, d_lens, d_dead, d_dregs;
  int up_chunks = 0;            // the last upload's chunks (PipeOpts::up_chunks)
  uint32_t up_hi[kUpChunks] = {};
};

}  // namespace

// An instantiated round loop (see rounds_on_device) and the launch
// arguments it was captured with; a run with other arguments captures anew.
struct RoundGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<unsigned char> key;
  RoundGraph() = default;
  RoundGraph(const RoundGraph&) = delete;
  RoundGraph& operator=(const RoundGraph&) = delete;
  ~RoundGraph() { reset(); }
  void reset() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
    key.clear();
  }
};

struct z80b_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[4] = {};
  std::vector<cudaEvent_t> kev;  // per-kernel timing events (pairs)
  std::vector<int> kev_cat;      // category of each pair: 0 qc, 1 exhaustive
  size_t kev_used = 0;
  std::string err;
  PoolBufs pool8;    // the 4,531 8-bit instructions (first-found candidates)
  PoolBufs loaded;   // z80b_load_candidates
  PoolBufs firstop;  // EnumerateFirstOp pool for all-hits jobs
  Staged staged;
  // pipeline scratch
  DBuf cnt_f, cnt_m, cnt_all, base, meta, surv, sdiff, checks;
  DBuf qc_tmp, qc_over;       // single-pass QuickCheck: kept survivors, targets with more
  DBuf next, win, windiff, spec, spec2, wlen, wend, cdone;
  DBuf pairs, pair_src, nchunks, cbase, nchunks_x, cbase_x, nchunks_c, cbase_c, nchunks_w, cbase_w, nchunks_r,
      cbase_r, rejected, npairs, counter, states;
  DBuf rcnt, rbase, rules, checked, surv_target, midpass, flag;
  HBuf h_rules;               // pinned staging of the device rules read back
  DBuf cub_tmp;
  DBuf hits, nhits, fpq;
  DBuf v_tgt, v_cand, v_tl, v_cl, v_dead, v_out, v_fd, v_in, v_outs;
  DBuf mul_best, mul_stats;   // constant-multiply search: best key per K, counters
  // length-2 candidates: the pair pool and its indexes, shared by the
  // contexts of a device; the per-lane pass state is per context
  std::shared_ptr<PairShared> pairpool;
  DBuf next2, win2, windiff2, cnt2, resume2, surv2, sdiff2, refill2;
  uint64_t n_rules_dev = 0;
  uint32_t launches = 0;
  int exh_k = 4;              // ExhaustiveCheck states per lane per dispatch (z80b_set_option)
  int chunk_blocks = 32;      // A-blocks per ExhaustiveCheck work chunk
  int priority = 0;           // Z80B_OPT_STREAM_PRIORITY
  int qc_index = 1;           // Z80B_OPT_QC_INDEX
  int xbits = 1;              // Z80B_OPT_XINDEP_BITS
  int compact = 1;            // Z80B_OPT_COMPACT_SWEEP
  int wide = 1;               // Z80B_OPT_WIDE_SWEEP
  uint32_t sweep_kernels = 0; // kSweep* bits of the sweep kernels launched since the last reset
  int graph_rounds = 1;       // Z80B_OPT_GRAPH_ROUNDS
  int concurrent_sweeps = 1;  // Z80B_OPT_CONCURRENT_SWEEPS
  int qc_single = 1;          // Z80B_OPT_QC_SINGLE_PASS
  // capture-time streams and events of the device rounds' parallel sweep
  // branches (created with the first graph that uses them)
  cudaStream_t side[4] = {};
  cudaEvent_t fork_ev = nullptr, join_ev[4] = {};
  // chunked target uploads: the copy stream, one event per chunk and one
  // that orders the copies after the context stream's earlier work
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t up_ev[kUpChunks + 1] = {};
  DBuf roundctl;              // RoundCtl of the device-driven rounds
  RoundGraph rg1, rg2;        // instantiated round loops: length-1 and length-2 candidate passes
};

namespace {

// Stage tracing to stderr when Z80B_TRACE is set (timestamps from the
// first traced event).
void trace(const char* fmt, ...) {
  static const bool on = std::getenv("Z80B_TRACE") != nullptr;
  if (!on) return;
  static const auto t0 = std::chrono::steady_clock::now();
  double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  std::fprintf(stderr, "[z80b %9.4fs] %s\n", dt, buf);
  std::fflush(stderr);
}

int fail(z80b_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

#define CK(call)                                                                       \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(ctx, e_ == cudaErrorMemoryAllocation ? Z80B_ENOMEM : Z80B_ECUDA,     \
                  "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

#define CKR(expr)              \
  do {                         \
    int r_ = (expr);           \
    if (r_ != Z80B_OK) return r_; \
  } while (0)

int check_launch(z80b_ctx* ctx, const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(ctx, Z80B_ECUDA, "%s launch: %s", what, cudaGetErrorString(e));
  ctx->launches++;
  return Z80B_OK;
}

// Exclusive prefix sum (CUB) of n items.
template <class T>
int scan(z80b_ctx* ctx, const T* in, T* out, uint32_t n) {
  if (!n) return Z80B_OK;
  size_t tmp = 0;
  CK(cub::DeviceScan::ExclusiveSum(nullptr, tmp, in, out, n, ctx->stream));
  CK(ctx->cub_tmp.ensure(tmp));
  CK(cub::DeviceScan::ExclusiveSum(ctx->cub_tmp.p, tmp, in, out, n, ctx->stream));
  ctx->launches += 2;  // tile-state init + scan kernel
  return Z80B_OK;
}

template <class T>
int fetch(z80b_ctx* ctx, T* host, const T* dev, size_t n = 1) {
  CK(cudaMemcpyAsync(host, dev, sizeof(T) * n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return Z80B_OK;
}

// Uploads a candidate list and computes its QuickCheck (and optionally
// MidCheck) outputs on the device.
int build_pool(z80b_ctx* ctx, PoolBufs& P, const uint32_t* insn, uint32_t n, uint32_t len,
               const uint8_t* lens, bool with_mid) {
  P.loaded = false;
  P.qstate = 0;  // a QuickCheck index of the previous contents is stale
  P.n = n;
  P.len = len;
  P.host_insn.assign(insn, insn + (size_t)n * len);
  P.host_lens.clear();
  if (lens) P.host_lens.assign(lens, lens + n);
  std::vector<uint8_t> size(n), prune(n);
  std::vector<uint16_t> reads(n);
  auto fill = [&](uint32_t lo, uint32_t hi) {
    for (uint32_t i = lo; i < hi; i++) {
      const uint32_t* s = insn + (size_t)i * len;
      int l = lens ? lens[i] : int(len);
      size[i] = uint8_t(seq_bytes(s, l));
      prune[i] = should_prune(s, l) ? 1 : 0;
      reads[i] = seq_reads(s, l);
    }
  };
  const uint32_t nth = n > (1u << 16) ? std::max(1u, std::min(32u, std::thread::hardware_concurrency())) : 1u;
  std::vector<std::thread> th;
  for (uint32_t k = 0; k < nth; k++)
    th.emplace_back(fill, uint32_t(uint64_t(n) * k / nth), uint32_t(uint64_t(n) * (k + 1) / nth));
  for (auto& t : th) t.join();
  CK(P.insn.ensure(sizeof(uint32_t) * n * len));
  CK(P.qc.ensure(sizeof(uint4) * 8 * n));
  if (with_mid) CK(P.mid.ensure(sizeof(uint4) * 32 * n));
  CK(P.size.ensure(n));
  CK(P.prune.ensure(n));
  CK(P.reads.ensure(sizeof(uint16_t) * n));
  if (lens) CK(P.lens.ensure(n));
  CK(cudaMemcpyAsync(P.insn.p, insn, sizeof(uint32_t) * n * len, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(P.size.p, size.data(), n, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(P.prune.p, prune.data(), n, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(P.reads.p, reads.data(), sizeof(uint16_t) * n, cudaMemcpyHostToDevice, ctx->stream));
  if (lens) CK(cudaMemcpyAsync(P.lens.p, lens, n, cudaMemcpyHostToDevice, ctx->stream));
  if (lens) {
    // variable-length pools run through k_exec-style outputs: lengths are
    // honoured by padding with NOP-free zero words is not possible, so the
    // pool kernel requires a fixed length
    return fail(ctx, Z80B_EINVAL, "candidate pools need a fixed sequence length");
  }
  trace("pool: %u candidates uploaded", n);
  launch_pool_outputs(P.insn.as<uint32_t>(), n, len, P.qc.as<uint4>(), with_mid ? P.mid.as<uint4>() : nullptr,
                      ctx->stream);
  CKR(check_launch(ctx, "pool_outputs"));
  trace("pool: kernel launched");
  CK(cudaStreamSynchronize(ctx->stream));
  trace("pool: outputs ready");
  P.dev = DevPool{};
  P.dev.insn = P.insn.as<uint32_t>();
  P.dev.qc = P.qc.as<uint4>();
  P.dev.mid = with_mid ? P.mid.as<uint4>() : nullptr;
  P.dev.size = P.size.as<uint8_t>();
  P.dev.prune = P.prune.as<uint8_t>();
  P.dev.reads = P.reads.as<uint16_t>();
  P.dev.lens = nullptr;
  P.dev.n = n;
  P.dev.len = len;
  P.dev.stride = len;
  P.loaded = true;
  return Z80B_OK;
}

int ensure_firstop(z80b_ctx* ctx) {
  if (ctx->firstop.loaded) return Z80B_OK;
  std::vector<uint32_t> v = first_op_pool();
  return build_pool(ctx, ctx->firstop, v.data(), uint32_t(v.size()), 1, nullptr, false);
}

bool valid_seq(const uint32_t* s, int n) {
  for (int i = 0; i < n; i++)
    if (insn_op(s[i]) >= kNumOps) return false;
  return true;
}

// The length-2 candidate pool: every odometer pair of the 8-bit list
// (pair index = first * 4531 + second, EnumerateSequences8(2) order), with
// its QuickCheck outputs, built once per context.
int ensure_pairpool(z80b_ctx* ctx) {
  if (!ctx->pairpool) ctx->pairpool = pair_shared(ctx->device);
  PairShared& S = *ctx->pairpool;
  std::lock_guard<std::mutex> lk(S.mu);
  if (S.pool.loaded) return Z80B_OK;
  const auto& p8 = pool8();
  const uint32_t n1 = uint32_t(p8.size());
  const uint32_t n = n1 * n1;
  std::vector<uint32_t> insn(size_t(n) * 2);
  for (uint32_t a = 0; a < n1; a++)
    for (uint32_t b = 0; b < n1; b++) {
      insn[(size_t(a) * n1 + b) * 2] = p8[a];
      insn[(size_t(a) * n1 + b) * 2 + 1] = p8[b];
    }
  trace("pair pool: %u pairs", n);
  CKR(build_pool(ctx, S.pool, insn.data(), n, 2, nullptr, false));
  // unpruned pairs by encoded size, for the eligible-pair count per target
  std::vector<uint8_t> size(n), prune(n);
  CK(cudaMemcpy(size.data(), S.pool.size.p, n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(prune.data(), S.pool.prune.p, n, cudaMemcpyDeviceToHost));
  std::vector<unsigned long long> by_size(17, 0);
  uint32_t valid = 0;
  for (uint32_t q = 0; q < n; q++)
    if (!prune[q]) {
      valid++;
      by_size[std::min<uint32_t>(size[q], 16)]++;
    }
  S.valid = valid;
  S.n_le[0] = uint32_t(by_size[0] + by_size[1] + by_size[2]);
  S.n_le[1] = uint32_t(S.n_le[0] + by_size[3]);
  S.eligible.assign(16, 0);
  for (int b = 1; b < 16; b++) S.eligible[size_t(b)] = S.eligible[size_t(b - 1)] + by_size[size_t(b - 1)];
  CK(S.eligible_dev.ensure(16 * sizeof(unsigned long long)));
  CK(cudaMemcpy(S.eligible_dev.p, S.eligible.data(), 16 * sizeof(unsigned long long), cudaMemcpyHostToDevice));
  CK(S.ptrs.ensure(64 * sizeof(void*)));
  CK(cudaMemset(S.ptrs.p, 0, 64 * sizeof(void*)));
  for (int k = 0; k < 2; k++) {
    CK(S.ptrs_le[k].ensure(64 * sizeof(void*)));
    CK(cudaMemset(S.ptrs_le[k].p, 0, 64 * sizeof(void*)));
  }
  trace("pair pool ready: %u unpruned (%u of at most 2 bytes, %u of at most 3)", valid, S.n_le[0], S.n_le[1]);
  return Z80B_OK;
}

// Selects index entries of unpruned pairs of at most max_size bytes (pruned
// pairs' keys are all ones).
struct ShortPair {
  const uint8_t* size;
  uint8_t max_size;
  __device__ bool operator()(const unsigned long long& key) const {
    return key != ~0ull && size[uint32_t(key)] <= max_size;
  }
};

// Bucket index of the pair pool for one dead-register mask: the pairs'
// (hash of the masked vector-0 output, pair index) keys, sorted.
int ensure_pair_index(z80b_ctx* ctx, uint32_t m) {
  PairShared& S = *ctx->pairpool;
  std::lock_guard<std::mutex> lk(S.mu);
  if (S.ok[m]) return Z80B_OK;
  const DevPool& P = S.pool.dev;
  const size_t n = P.n;
  CK(S.keys_tmp.ensure(n * 8));
  CK(S.idx[m].ensure(n * 8));
  launch_pair_keys(P, m, S.keys_tmp.as<unsigned long long>(), ctx->stream);
  CKR(check_launch(ctx, "pair_keys"));
  size_t tmp = 0;
  CK(cub::DeviceRadixSort::SortKeys(nullptr, tmp, S.keys_tmp.as<unsigned long long>(),
                                    S.idx[m].as<unsigned long long>(), int(n), 0, 64, ctx->stream));
  CK(S.sort_tmp.ensure(tmp));
  CK(cub::DeviceRadixSort::SortKeys(S.sort_tmp.p, tmp, S.keys_tmp.as<unsigned long long>(),
                                    S.idx[m].as<unsigned long long>(), int(n), 0, 64, ctx->stream));
  ctx->launches += 2;
  void* ptr = S.idx[m].p;
  CK(cudaMemcpyAsync(S.ptrs.as<void*>() + m, &ptr, sizeof ptr, cudaMemcpyHostToDevice, ctx->stream));
  // the short-pair indexes: the entries of pairs of at most 2 / 3 bytes, in
  // the full index's order (a stable selection)
  CK(S.sel_count.ensure(sizeof(int)));
  for (int k = 0; k < 2; k++) {
    CK(S.idx_le[k][m].ensure(8ull * std::max<uint32_t>(S.n_le[k], 1)));
    const ShortPair pred{P.size, uint8_t(2 + k)};
    size_t stmp = 0;
    CK(cub::DeviceSelect::If(nullptr, stmp, S.idx[m].as<unsigned long long>(), S.idx_le[k][m].as<unsigned long long>(),
                             S.sel_count.as<int>(), int(n), pred, ctx->stream));
    CK(S.sel_tmp.ensure(stmp));
    CK(cub::DeviceSelect::If(S.sel_tmp.p, stmp, S.idx[m].as<unsigned long long>(),
                             S.idx_le[k][m].as<unsigned long long>(), S.sel_count.as<int>(), int(n), pred,
                             ctx->stream));
    ctx->launches += 1;
    int got = 0;
    CK(cudaMemcpyAsync(&got, S.sel_count.p, sizeof got, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (uint32_t(got) != S.n_le[k])
      return fail(ctx, Z80B_ECUDA, "short-pair index holds %d entries, expected %u", got, S.n_le[k]);
    void* q = S.idx_le[k][m].p;
    CK(cudaMemcpyAsync(S.ptrs_le[k].as<void*>() + m, &q, sizeof q, cudaMemcpyHostToDevice, ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  S.ok[m] = true;
  trace("pair index for dead-register mask %02X built", m);
  return Z80B_OK;
}

// QuickCheck bucket index of a pool: every candidate's (dead-register mask,
// hash of its masked vector-0 output, index) key for all 64 masks in one
// sort, the per-mask top tables, and the eligible-candidate counts by
// target size.  Pools above kQCIndexMax candidates keep the full scan.
int ensure_qc_index(z80b_ctx* ctx, PoolBufs& P, uint32_t w2mask) {
  if (P.qstate == -1) return Z80B_OK;
  if (P.qstate == 1 && P.qw2 == w2mask) return Z80B_OK;
  const uint32_t n = P.dev.n;
  if (n == 0 || n > kQCIndexMax) {
    P.qstate = -1;
    return Z80B_OK;
  }
  cudaStream_t s = ctx->stream;
  std::vector<uint8_t> size(n), prune(n);
  CK(cudaMemcpyAsync(size.data(), P.size.p, n, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(prune.data(), P.prune.p, n, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  std::vector<uint32_t> by_size(257, 0), elig(256, 0);
  uint32_t nv = 0;
  for (uint32_t q = 0; q < n; q++)
    if (!prune[q]) {
      nv++;
      by_size[size[q]]++;
    }
  for (int b = 1; b < 256; b++) elig[size_t(b)] = elig[size_t(b - 1)] + by_size[size_t(b - 1)];
  const size_t nk = 64ull * n;
  CK(P.qkeys_tmp.ensure(nk * 8));
  CK(P.qkeys.ensure(nk * 8));
  CK(P.qtop.ensure(64ull * (kQCTop + 1) * 4));
  CK(P.qelig.ensure(256 * 4));
  launch_qc_keys(P.dev, w2mask, P.qkeys_tmp.as<unsigned long long>(), s);
  CKR(check_launch(ctx, "qc_keys"));
  size_t tmp = 0;
  CK(cub::DeviceRadixSort::SortKeys(nullptr, tmp, P.qkeys_tmp.as<unsigned long long>(),
                                    P.qkeys.as<unsigned long long>(), int(nk), 0, 64, s));
  CK(P.qsort_tmp.ensure(tmp));
  CK(cub::DeviceRadixSort::SortKeys(P.qsort_tmp.p, tmp, P.qkeys_tmp.as<unsigned long long>(),
                                    P.qkeys.as<unsigned long long>(), int(nk), 0, 64, s));
  launch_qc_top(P.qkeys.as<unsigned long long>(), nv, P.qtop.as<uint32_t>(), s);
  CKR(check_launch(ctx, "qc_top"));
  CK(cudaMemcpyAsync(P.qelig.p, elig.data(), 256 * 4, cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));
  ctx->launches += 3;
  P.qstate = 1;
  P.qw2 = w2mask;
  trace("QuickCheck index: %u candidates, %u unpruned, 64 masks", n, nv);
  return Z80B_OK;
}

// Runs fn(lo, hi) over [0, n) split into contiguous parts on up to 16 host
// threads (in the calling thread alone below 2^15 items).
template <class F>
void host_parallel(size_t n, F fn) {
  constexpr size_t kMinPart = size_t(1) << 14;
  size_t parts = std::min<size_t>(16, std::max(1u, std::thread::hardware_concurrency()));
  parts = std::min(parts, n / kMinPart);
  if (parts <= 1) {
    fn(size_t(0), n);
    return;
  }
  std::vector<std::thread> th;
  for (size_t k = 1; k < parts; k++) th.emplace_back(fn, n * k / parts, n * (k + 1) / parts);
  fn(size_t(0), n / parts);
  for (auto& t : th) t.join();
}

int validate_job(z80b_ctx* ctx, const z80b_job* job) {
  if (!job) return fail(ctx, Z80B_EINVAL, "job is null");
  if (job->n_targets && !job->targets) return fail(ctx, Z80B_EINVAL, "targets is null");
  if (job->target_stride < 1 || job->target_stride > 64) return fail(ctx, Z80B_EINVAL, "bad target_stride");
  if (job->mode != Z80B_MODE_FIRST && job->mode != Z80B_MODE_ALL) return fail(ctx, Z80B_EINVAL, "bad mode");
  if (job->path != Z80B_PATH_BATCHED && job->path != Z80B_PATH_PLAIN) return fail(ctx, Z80B_EINVAL, "bad path");
  if (job->max_cand_len < 1 || job->max_cand_len > 2)
    return fail(ctx, Z80B_EINVAL, "max_cand_len must be 1 or 2");
  if (job->max_cand_len == 2 && job->mode != Z80B_MODE_FIRST)
    return fail(ctx, Z80B_EINVAL, "length-2 candidates need Z80B_MODE_FIRST");
  if (job->flags & ~Z80B_JOB_NO_EXHAUSTIVE) return fail(ctx, Z80B_EINVAL, "unknown job flags %#x", job->flags);
  if ((job->flags & Z80B_JOB_NO_EXHAUSTIVE) && job->mode != Z80B_MODE_ALL)
    return fail(ctx, Z80B_EINVAL, "Z80B_JOB_NO_EXHAUSTIVE needs Z80B_MODE_ALL");
  if (job->global_dead_flags > 0xFF) return fail(ctx, Z80B_EINVAL, "dead flags > 0xFF");
  return Z80B_OK;
}

// The targets themselves (lengths, opcodes, dead-register masks).  Runs after
// validate_job, while the targets' upload is in flight; nothing reads the
// device copy before this returns Z80B_OK.
int validate_targets(z80b_ctx* ctx, const z80b_job* job) {
  // the first bad target (the reported one is the lowest index, as a
  // serial scan would find); the scan runs on several host threads
  std::atomic<uint64_t> first_bad{~0ull};
  host_parallel(job->n_targets, [&](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; i++) {
      const uint32_t l = job->target_lens ? job->target_lens[i] : job->target_len;
      const bool ok = l >= 1 && l <= uint32_t(kMaxSeq) && l <= job->target_stride &&
                      valid_seq(job->targets + i * job->target_stride, int(l)) &&
                      !(job->dead_regs && (job->dead_regs[i] & ~0x3Fu));
      if (!ok) {
        uint64_t cur = first_bad.load();
        while (i < cur && !first_bad.compare_exchange_weak(cur, i)) {
        }
        return;
      }
    }
  });
  if (first_bad.load() != ~0ull) {
    const uint32_t i = uint32_t(first_bad.load());
    const uint32_t l = job->target_lens ? job->target_lens[i] : job->target_len;
    if (l < 1 || l > uint32_t(kMaxSeq) || l > job->target_stride)
      return fail(ctx, Z80B_EINVAL, "target %u: length %u outside 1..%d", i, l, kMaxSeq);
    if (!valid_seq(job->targets + (size_t)i * job->target_stride, int(l)))
      return fail(ctx, Z80B_EINVAL, "target %u: opcode > 454", i);
    return fail(ctx, Z80B_EINVAL, "target %u: dead_regs uses bits above B..L", i);
  }
  return Z80B_OK;
}

// Brackets one kernel launch with a pair of events on the context stream.
int kbegin(z80b_ctx* ctx, int cat) {
  if (ctx->kev_used + 2 > ctx->kev.size()) {
    for (int i = 0; i < 64; i++) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return -1;
      ctx->kev.push_back(e);
    }
  }
  int i = int(ctx->kev_used);
  ctx->kev_used += 2;
  ctx->kev_cat.resize(ctx->kev_used / 2);
  ctx->kev_cat[size_t(i / 2)] = cat;
  cudaEventRecord(ctx->kev[size_t(i)], ctx->stream);
  return i;
}
void kend(z80b_ctx* ctx, int i) {
  if (i >= 0) cudaEventRecord(ctx->kev[size_t(i) + 1], ctx->stream);
}
void ksum(z80b_ctx* ctx, double* qc, double* exh) {
  for (size_t p = 0; p < ctx->kev_used / 2; p++) {
    float f = 0;
    cudaEventSynchronize(ctx->kev[2 * p + 1]);
    cudaEventElapsedTime(&f, ctx->kev[2 * p], ctx->kev[2 * p + 1]);
    if (ctx->kev_cat[p] == 0) *qc += f;
    else *exh += f;
  }
  ctx->kev_used = 0;
}

struct Timer {
  z80b_ctx* ctx;
  int a, b;
  void start() { cudaEventRecord(ctx->ev[a], ctx->stream); }
  void stop() { cudaEventRecord(ctx->ev[b], ctx->stream); }
  double ms() {
    float f = 0;
    cudaEventSynchronize(ctx->ev[b]);
    cudaEventElapsedTime(&f, ctx->ev[a], ctx->ev[b]);
    return f;
  }
};

void to_rules(z80b_ctx* ctx, const DevRule* dr, size_t ndr, const uint32_t* targets, const uint8_t* tlens,
              uint32_t tlen, uint32_t stride, uint32_t mode, uint32_t tindex_offset, z80b_rule* out);

// Hands each target's rules to a callback as soon as both of its
// (target, kind) lanes are final: a lane is final once it has a winner, or
// it is resolved without one and no longer candidates remain to try.  The
// pipeline calls update() after every ExhaustiveCheck round; each call
// copies the lane arrays (a few words per target) to the host.
struct Reporter {
  z80b_rule_cb cb = nullptr;
  void* user = nullptr;
  const uint32_t* targets = nullptr;
  const uint8_t* tlens = nullptr;
  uint32_t tlen = 0, stride = 0;
  std::vector<uint8_t> done;
  std::vector<uint32_t> n1, w1, n2, w2;
  std::vector<uint16_t> d1, d2;

  int update(z80b_ctx* ctx, uint32_t n, const Lanes& L, const Lanes& L2, uint32_t max_cand, bool phase2,
             bool last);
};

// ExhaustiveCheck of the np pairs of a round: chunk prefixes of both pair
// classes, then the sweep kernel of each class that has chunks.
int sweep_round(z80b_ctx* ctx, const DevTargets& T, const DevPool& P, const RoundBuf& R, uint32_t np) {
  cudaStream_t s = ctx->stream;
  CKR(scan(ctx, R.nchunks, R.cbase, np));
  CKR(scan(ctx, R.nchunks_x, R.cbase_x, np));
  if (R.compact) CKR(scan(ctx, R.nchunks_c, R.cbase_c, np));
  if (R.wide) {
    CKR(scan(ctx, R.nchunks_w, R.cbase_w, np));
    CKR(scan(ctx, R.nchunks_r, R.cbase_r, np));
  }
  unsigned long long last[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  CK(cudaMemcpyAsync(&last[0], R.cbase + (np - 1), 8, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&last[1], R.nchunks + (np - 1), 8, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&last[2], R.cbase_x + (np - 1), 8, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&last[3], R.nchunks_x + (np - 1), 8, cudaMemcpyDeviceToHost, s));
  if (R.compact) {
    CK(cudaMemcpyAsync(&last[4], R.cbase_c + (np - 1), 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&last[5], R.nchunks_c + (np - 1), 8, cudaMemcpyDeviceToHost, s));
  }
  if (R.wide) {
    CK(cudaMemcpyAsync(&last[6], R.cbase_w + (np - 1), 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&last[7], R.nchunks_w + (np - 1), 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&last[8], R.cbase_r + (np - 1), 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&last[9], R.nchunks_r + (np - 1), 8, cudaMemcpyDeviceToHost, s));
  }
  CK(cudaStreamSynchronize(s));
  CK(cudaMemsetAsync(R.counter, 0, 40, s));
  trace("sweep: %u pairs, %llu + %llu + %llu + %llu + %llu chunks", np, last[0] + last[1], last[2] + last[3],
        last[4] + last[5], last[6] + last[7], last[8] + last[9]);
  int ke = kbegin(ctx, 1);
  const int nl = launch_exhaustive(T, P, R, np, last[0] + last[1], last[2] + last[3], last[4] + last[5],
                                   last[6] + last[7], last[8] + last[9], ctx->exh_k, s, &ctx->sweep_kernels);
  kend(ctx, ke);
  CKR(check_launch(ctx, "exhaustive"));
  if (nl > 1) ctx->launches += uint32_t(nl - 1);
  return Z80B_OK;
}

template <class V>
void key_put(std::vector<unsigned char>& k, const V& v) {
  const unsigned char* b = reinterpret_cast<const unsigned char*>(&v);
  k.insert(k.end(), b, b + sizeof v);
}

// The rounds of one first-found pass driven by the device: one CUDA graph
// whose WHILE node repeats the round body -- clear the pair counter (and the
// rescan counter), build the round's pairs, scan their chunk counts and set
// the loop condition (k_round_scan), [rescan the length-2 buckets of lanes
// whose slots ran out, only after an empty round], the sweep kernels of
// every class on persistent grids, resolve -- until a round is empty with no
// rescan pending.  The same work and order as the host loop of
// run_pipeline, without a host round trip per round.  The graph is
// captured once per set of launch arguments and replayed.
int rounds_on_device(z80b_ctx* ctx, RoundGraph& g, const DevTargets& T, const DevPool& P, const QCOut& q,
                     const Lanes& L, const RoundBuf& R, uint32_t max_spec, const PairScan* ps, const QCOut* qres,
                     uint32_t* rounds, uint64_t* pairs) {
  cudaStream_t s = ctx->stream;
  CK(ctx->roundctl.ensure(sizeof(RoundCtl)));
  RoundCtl* ctl = ctx->roundctl.as<RoundCtl>();
  std::vector<unsigned char> key;
  key_put(key, T);
  key_put(key, P);
  key_put(key, q);
  key_put(key, L);
  key_put(key, R);
  key_put(key, max_spec);
  key_put(key, ctx->exh_k);
  key_put(key, ctl);
  if (ps) {
    key_put(key, *ps);
    key_put(key, *qres);
  }
  key_put(key, ctx->concurrent_sweeps);
  if (!g.exec || g.key != key) {
    g.reset();
    warm_exhaustive_dev(R, ctx->exh_k);
    if (ctx->concurrent_sweeps && !ctx->side[0]) {
      CK(cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming));
      for (int i = 0; i < 4; i++) {
        CK(cudaStreamCreateWithFlags(&ctx->side[i], cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&ctx->join_ev[i], cudaEventDisableTiming));
      }
    }
    CK(cudaGraphCreate(&g.graph, 0));
    cudaGraphConditionalHandle loop;
    CK(cudaGraphConditionalHandleCreate(&loop, g.graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = loop;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g.graph, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CK(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(R.npairs, 0, 4, s);
    if (ps) {
      cudaMemsetAsync(ps->refill, 0, 4, s);
      launch_pair_round_build(T, P, q, L, *ps, R, s);
      launch_round_scan(R, ctl, ps->refill, loop, s);
      launch_pair_scan_gated(T, P, q, L, *ps, ctl, s);
    } else {
      launch_round_build(T, P, q, L, R, s);
      launch_round_scan(R, ctl, nullptr, loop, s);
    }
    {
      // the classes' sweeps on parallel branches of the body graph
      cudaStream_t ss[5] = {s, s, s, s, s};
      if (ctx->concurrent_sweeps) {
        cudaEventRecord(ctx->fork_ev, s);
        for (int i = 0; i < 4; i++) {
          cudaStreamWaitEvent(ctx->side[i], ctx->fork_ev, 0);
          ss[i + 1] = ctx->side[i];
        }
      }
      launch_exhaustive_dev(T, P, R, ctl, ctx->exh_k, ss);
      if (ctx->concurrent_sweeps)
        for (int i = 0; i < 4; i++) {
          cudaEventRecord(ctx->join_ev[i], ctx->side[i]);
          cudaStreamWaitEvent(s, ctx->join_ev[i], 0);
        }
    }
    launch_round_resolve_dev(R, ctl, ps ? *qres : q, L, max_spec, s);
    cudaGraph_t captured = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(s, &captured);
    if (ce != cudaSuccess) {
      g.reset();
      cudaGetLastError();
      CK(ce);
    }
    CK(cudaGraphInstantiate(&g.exec, g.graph, 0));
    g.key = key;
    trace("round loop captured (%s pass)", ps ? "length-2" : "length-1");
  }
  // build, scan (3), [rescan], sweeps, resolve
  const int per_iter = (ps ? 5 : 4) + 1 + 2 + (R.compact ? 1 : 0) + (R.wide ? 2 : 0);
  CK(cudaMemsetAsync(ctl, 0, sizeof(RoundCtl), s));
  int ke = kbegin(ctx, 1);
  CK(cudaGraphLaunch(g.exec, s));
  kend(ctx, ke);
  CKR(check_launch(ctx, "round loop"));
  RoundCtl h{};
  CK(cudaMemcpyAsync(&h, ctl, offsetof(RoundCtl, bsum), cudaMemcpyDeviceToHost, s));  // the counters
  CK(cudaStreamSynchronize(s));
  if (h.overrun) return fail(ctx, Z80B_ETIMEOUT, "device round loop did not end within %u iterations", kMaxRoundIters);
  *rounds += h.rounds;
  *pairs += h.pairs;
  ctx->launches += h.iters * uint32_t(per_iter);
  uint32_t mask = (R.compact ? kSweepCompact : 0u) | (R.wide ? kSweepWide | kSweepRegs : 0u) | kSweepBits;
  if (R.xunit == kXBitsBlocks) mask |= kSweepXBits;
  else mask |= kSweepScalarK1 << (ctx->exh_k == 1 ? 0 : ctx->exh_k == 2 ? 1 : ctx->exh_k == 8 ? 3 : 2);
  ctx->sweep_kernels |= mask;
  trace("device rounds: %u rounds, %u iterations, %llu pairs", h.rounds, h.iters, (unsigned long long)h.pairs);
  return Z80B_OK;
}

// Runs the pipeline on device-resident targets.  Rules stay in ctx->rules
// (DevRule), count in *nr.
int run_pipeline(z80b_ctx* ctx, const DevTargets& T, const PipeOpts& opts, z80b_stats* st, uint64_t* nr) {
  const uint32_t mode = opts.mode;
  const uint32_t n = T.n;
  cudaStream_t s = ctx->stream;
  PoolBufs* pool = &ctx->pool8;
  QCConfig cfg{0xFFFFFFFFu, 0, 1};
  if (mode == Z80B_MODE_ALL) {
    if (ctx->loaded.loaded) pool = &ctx->loaded;
    else {
      CKR(ensure_firstop(ctx));
      pool = &ctx->firstop;
    }
    cfg.w2mask = 0x0000FFFFu;  // 80-byte fingerprint: SP but not M
    cfg.all_hits = 1;
  }
  cfg.use_smem = pool->dev.n <= 6144 ? 1 : 0;
  const DevPool& P = pool->dev;
  *nr = 0;
  if (n == 0) return Z80B_OK;

  CK(ctx->cnt_f.ensure(4ull * n));
  CK(ctx->cnt_m.ensure(4ull * n));
  CK(ctx->cnt_all.ensure(4ull * n));
  CK(ctx->base.ensure(4ull * n));
  CK(ctx->meta.ensure(sizeof(TargetMeta) * n));
  CK(ctx->checks.ensure(8));
  CK(ctx->checked.ensure(8));
  CK(ctx->states.ensure(16));
  CK(ctx->npairs.ensure(4));
  CK(ctx->counter.ensure(40));
  CK(cudaMemsetAsync(ctx->checks.p, 0, 8, s));
  CK(cudaMemsetAsync(ctx->checked.p, 0, 8, s));
  CK(cudaMemsetAsync(ctx->states.p, 0, 16, s));

  QCIndex qix{};
  bool use_ix = false;
  if (ctx->qc_index) {
    CKR(ensure_qc_index(ctx, *pool, cfg.w2mask));
    if (pool->qstate == 1) {
      use_ix = true;
      qix.keys = pool->qkeys.as<unsigned long long>();
      qix.top = pool->qtop.as<uint32_t>();
      qix.elig_lt = pool->qelig.as<uint32_t>();
    }
  }
  trace("pipeline: %u targets, mode %u, pool %u", n, mode, P.n);
  QCOut q{};
  q.cnt_f = ctx->cnt_f.as<uint32_t>();
  q.cnt_m = ctx->cnt_m.as<uint32_t>();
  q.cnt_all = ctx->cnt_all.as<uint32_t>();
  q.meta = ctx->meta.as<TargetMeta>();
  q.checks = ctx->checks.as<unsigned long long>();
  if (use_ix && ctx->qc_single) {
    // single pass: the count pass keeps the survivors of targets with few
    CK(ctx->qc_tmp.ensure(4ull * kQCSlots * n));
    CK(ctx->qc_over.ensure(4));
    CK(cudaMemsetAsync(ctx->qc_over.p, 0, 4, s));
    q.tmp = ctx->qc_tmp.as<uint32_t>();
    q.over = ctx->qc_over.as<uint32_t>();
  }
  // the count over targets [lo, hi) (every per-target array offset by lo)
  auto qc_count = [&](uint32_t lo, uint32_t hi) {
    DevTargets Tc = T;
    QCOut qc = q;
    if (lo) {
      Tc.insn += (size_t)lo * T.stride;
      if (Tc.len) Tc.len += lo;
      if (Tc.dead) Tc.dead += lo;
      if (Tc.dead_regs) Tc.dead_regs += lo;
      qc.cnt_f += lo;
      qc.cnt_m += lo;
      qc.cnt_all += lo;
      qc.meta += lo;
      if (qc.tmp) qc.tmp += (size_t)lo * kQCSlots;
    }
    Tc.n = hi - lo;
    if (use_ix) launch_qc_bucket(Tc, P, cfg, qix, qc, false, s);
    else launch_qc_scan(Tc, P, cfg, qc, false, s);
    return check_launch(ctx, "qc_count");
  };
  // chunked upload: the first chunk is on the device before the clock starts
  if (opts.up_chunks) CK(cudaStreamWaitEvent(s, ctx->up_ev[0], 0));
  Timer tall{ctx, 0, 1};
  ctx->kev_used = 0;
  tall.start();
  int kq = kbegin(ctx, 0);
  if (opts.up_chunks) {
    uint32_t lo = 0;
    for (int k = 0; k < opts.up_chunks; k++) {
      const uint32_t hi = opts.up_hi[k];
      if (k) CK(cudaStreamWaitEvent(s, ctx->up_ev[k], 0));
      if (hi > lo) CKR(qc_count(lo, hi));
      lo = hi;
    }
  } else {
    CKR(qc_count(0, n));
  }
  kend(ctx, kq);
  CKR(scan(ctx, ctx->cnt_all.as<uint32_t>(), ctx->base.as<uint32_t>(), n));
  uint32_t last[4] = {0, 0, 0, 0};
  CK(cudaMemcpyAsync(&last[0], ctx->base.as<uint32_t>() + (n - 1), 4, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&last[1], ctx->cnt_f.as<uint32_t>() + (n - 1), 4, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&last[2], ctx->cnt_m.as<uint32_t>() + (n - 1), 4, cudaMemcpyDeviceToHost, s));
  if (q.over) CK(cudaMemcpyAsync(&last[3], q.over, 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  const uint64_t nsurv = uint64_t(last[0]) + last[1] + last[2];
  trace("qc count done: %llu survivors", (unsigned long long)nsurv);
  if (nsurv > 0xFFFFFFF0ull) return fail(ctx, Z80B_ECAPACITY, "too many QuickCheck survivors (%llu)", (unsigned long long)nsurv);
  CK(ctx->surv.ensure(4ull * std::max<uint64_t>(nsurv, 1)));
  CK(ctx->sdiff.ensure(2ull * std::max<uint64_t>(nsurv, 1)));
  q.base = ctx->base.as<uint32_t>();
  q.surv = ctx->surv.as<uint32_t>();
  q.sdiff = ctx->sdiff.as<uint16_t>();
  if (nsurv && q.tmp) {
    int kc = kbegin(ctx, 0);
    launch_qc_compact(q, n, s);
    kend(ctx, kc);
    CKR(check_launch(ctx, "qc_compact"));
  }
  if (nsurv && (!q.tmp || last[3])) {
    // every target (two passes), or those with more survivors than the
    // count pass kept
    int kc = kbegin(ctx, 0);
    if (use_ix) launch_qc_bucket(T, P, cfg, qix, q, true, s);
    else launch_qc_scan(T, P, cfg, q, true, s);
    kend(ctx, kc);
    CKR(check_launch(ctx, "qc_collect"));
  }

  RoundBuf R{};
  uint32_t rounds = 0;
  uint64_t exh_pairs = 0, mid_surv = 0;
  if (mode == Z80B_MODE_FIRST) {
    CK(ctx->next.ensure(8ull * n));
    CK(ctx->win.ensure(8ull * n));
    CK(ctx->windiff.ensure(4ull * n));
    // pair slots per round: every lane once, and room for survivor windows
    const uint64_t cap = std::max<uint64_t>(2ull * n, std::min<uint64_t>(128ull * n, 1ull << 20));
    CK(ctx->pairs.ensure(sizeof(PairRec) * cap));
    CK(ctx->pair_src.ensure(4 * cap));
    CK(ctx->nchunks.ensure(8 * cap));
    CK(ctx->cbase.ensure(8 * cap));
    CK(ctx->nchunks_x.ensure(8 * cap));
    CK(ctx->cbase_x.ensure(8 * cap));
    if (ctx->compact) {
      CK(ctx->nchunks_c.ensure(8 * cap));
      CK(ctx->cbase_c.ensure(8 * cap));
    }
    if (ctx->wide) {
      CK(ctx->nchunks_w.ensure(8 * cap));
      CK(ctx->cbase_w.ensure(8 * cap));
      CK(ctx->nchunks_r.ensure(8 * cap));
      CK(ctx->cbase_r.ensure(8 * cap));
    }
    CK(ctx->rejected.ensure(4 * cap));
    CK(ctx->wlen.ensure(cap));
    CK(ctx->wend.ensure(4 * cap));
    CK(ctx->cdone.ensure(4 * cap));
    CK(ctx->spec.ensure(2ull * n));
    CK(cudaMemsetAsync(ctx->spec.p, 0, 2ull * n, s));
    CK(cudaMemsetAsync(ctx->next.p, 0, 8ull * n, s));
    CK(cudaMemsetAsync(ctx->win.p, 0xFF, 8ull * n, s));
    Lanes L{ctx->next.as<uint32_t>(), ctx->win.as<uint32_t>(), ctx->windiff.as<uint16_t>(), ctx->spec.as<uint8_t>()};
    R.pairs = ctx->pairs.as<PairRec>();
    R.pair_src = ctx->pair_src.as<uint32_t>();
    R.nchunks = ctx->nchunks.as<unsigned long long>();
    R.cbase = ctx->cbase.as<unsigned long long>();
    R.nchunks_x = ctx->nchunks_x.as<unsigned long long>();
    R.cbase_x = ctx->cbase_x.as<unsigned long long>();
    R.rejected = ctx->rejected.as<uint32_t>();
    R.wlen = ctx->wlen.as<uint8_t>();
    R.wend = ctx->wend.as<uint32_t>();
    R.cdone = ctx->cdone.as<uint32_t>();
    R.cap = uint32_t(cap);
    R.npairs = ctx->npairs.as<uint32_t>();
    R.counter = ctx->counter.as<unsigned long long>();
    R.states = ctx->states.as<unsigned long long>();
    R.chunk_blocks = uint32_t(ctx->chunk_blocks);
    R.xunit = ctx->xbits ? kXBitsBlocks : kXScalarBlocks;
    R.compact = mode == Z80B_MODE_FIRST && ctx->compact ? 1u : 0u;
    R.nchunks_c = R.compact ? ctx->nchunks_c.as<unsigned long long>() : nullptr;
    R.cbase_c = R.compact ? ctx->cbase_c.as<unsigned long long>() : nullptr;
    R.wide = mode == Z80B_MODE_FIRST && ctx->wide ? 1u : 0u;
    R.nchunks_w = R.wide ? ctx->nchunks_w.as<unsigned long long>() : nullptr;
    R.cbase_w = R.wide ? ctx->cbase_w.as<unsigned long long>() : nullptr;
    R.nchunks_r = R.wide ? ctx->nchunks_r.as<unsigned long long>() : nullptr;
    R.cbase_r = R.wide ? ctx->cbase_r.as<unsigned long long>() : nullptr;
    // rounds on the device (one graph) unless the caller takes answers
    // round by round (streaming callbacks)
    const bool dev_rounds = ctx->graph_rounds && !opts.rep;
    if (nsurv && dev_rounds) {
      CKR(rounds_on_device(ctx, ctx->rg1, T, P, q, L, R, kMaxSpec1, nullptr, nullptr, &rounds, &exh_pairs));
    } else if (nsurv) {
      for (;;) {
        CK(cudaMemsetAsync(R.npairs, 0, 4, s));
        launch_round_build(T, P, q, L, R, s);
        CKR(check_launch(ctx, "round_build"));
        uint32_t np = 0;
        CKR(fetch(ctx, &np, R.npairs));
        np = std::min(np, R.cap);
        trace("round %u: %u pairs", rounds, np);
        if (np == 0) break;
        rounds++;
        exh_pairs += np;
        CKR(sweep_round(ctx, T, P, R, np));
        launch_round_resolve(R, np, q, L, kMaxSpec1, s);
        CKR(check_launch(ctx, "round_resolve"));
        if (opts.rep) CKR(opts.rep->update(ctx, n, L, Lanes{}, opts.max_cand, false, false));
      }
    }
    Lanes L2{};
    unsigned long long pool2_enum = 0;
    if (opts.max_cand >= 2) {
      // Length-2 candidates for the lanes the length-1 pass left without a
      // winner (worker.go:131-184: candLen 2 after candLen 1).
      CKR(ensure_pairpool(ctx));
      const PairShared& PS = *ctx->pairpool;
      const DevPool& P2 = PS.pool.dev;
      pool2_enum = (unsigned long long)P2.n;
      for (uint32_t m = 0; m < 64; m++)
        if ((opts.dreg_masks >> m) & 1u) CKR(ensure_pair_index(ctx, m));
      CK(ctx->next2.ensure(8ull * n));
      CK(ctx->win2.ensure(8ull * n));
      CK(ctx->windiff2.ensure(4ull * n));
      CK(ctx->cnt2.ensure(8ull * n));
      CK(ctx->resume2.ensure(8ull * n));
      CK(ctx->surv2.ensure(8ull * n * kSlots2));
      CK(ctx->sdiff2.ensure(4ull * n * kSlots2));
      CK(ctx->refill2.ensure(4));
      CK(ctx->spec2.ensure(2ull * n));
      L2 = Lanes{ctx->next2.as<uint32_t>(), ctx->win2.as<uint32_t>(), ctx->windiff2.as<uint16_t>(),
                 ctx->spec2.as<uint8_t>()};
      PairScan ps{};
      ps.idx = reinterpret_cast<const unsigned long long* const*>(PS.ptrs.p);
      ps.n_valid = PS.valid;
      ps.idx_le2 = reinterpret_cast<const unsigned long long* const*>(PS.ptrs_le[0].p);
      ps.idx_le3 = reinterpret_cast<const unsigned long long* const*>(PS.ptrs_le[1].p);
      ps.n_le2 = PS.n_le[0];
      ps.n_le3 = PS.n_le[1];
      ps.cnt = ctx->cnt2.as<uint32_t>();
      ps.resume = ctx->resume2.as<uint32_t>();
      ps.surv = ctx->surv2.as<uint32_t>();
      ps.sdiff = ctx->sdiff2.as<uint16_t>();
      ps.refill = ctx->refill2.as<uint32_t>();
      ps.eligible = PS.eligible_dev.as<unsigned long long>();
      ps.checks = ctx->checks.as<unsigned long long>();
      QCOut q2 = q;
      q2.sdiff = ps.sdiff;
      launch_pair_lanes_init(T, L, q, L2, ps, s);
      CKR(check_launch(ctx, "pair_lanes_init"));
      int kq2 = kbegin(ctx, 0);
      launch_pair_scan(T, P2, q, L2, ps, s);
      kend(ctx, kq2);
      CKR(check_launch(ctx, "pair_scan"));
      if (dev_rounds)
        CKR(rounds_on_device(ctx, ctx->rg2, T, P2, q, L2, R, kMaxSpec2, &ps, &q2, &rounds, &exh_pairs));
      for (; !dev_rounds;) {
        CK(cudaMemsetAsync(R.npairs, 0, 4, s));
        CK(cudaMemsetAsync(ps.refill, 0, 4, s));
        launch_pair_round_build(T, P2, q, L2, ps, R, s);
        CKR(check_launch(ctx, "pair_round_build"));
        uint32_t np = 0, nref = 0;
        CK(cudaMemcpyAsync(&np, R.npairs, 4, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(&nref, ps.refill, 4, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        np = std::min(np, R.cap);
        trace("length-2 round %u: %u pairs, %u lanes to rescan", rounds, np, nref);
        if (np == 0) {
          if (nref == 0) break;
          int kr = kbegin(ctx, 0);
          launch_pair_scan(T, P2, q, L2, ps, s);
          kend(ctx, kr);
          CKR(check_launch(ctx, "pair_scan"));
          continue;
        }
        rounds++;
        exh_pairs += np;
        CKR(sweep_round(ctx, T, P2, R, np));
        launch_round_resolve(R, np, q2, L2, kMaxSpec2, s);
        CKR(check_launch(ctx, "round_resolve"));
        if (opts.rep) CKR(opts.rep->update(ctx, n, L, L2, opts.max_cand, true, false));
      }
    }
    if (opts.rep) CKR(opts.rep->update(ctx, n, L, L2, opts.max_cand, opts.max_cand >= 2, true));
    CK(ctx->rcnt.ensure(4ull * n));
    CK(ctx->rbase.ensure(4ull * n));
    launch_rule_count_first(L, L2, n, ctx->rcnt.as<uint32_t>(), T, ctx->checked.as<unsigned long long>(),
                            uint32_t(pool8().size()), pool2_enum, s);
    CKR(check_launch(ctx, "rule_count"));
    CKR(scan(ctx, ctx->rcnt.as<uint32_t>(), ctx->rbase.as<uint32_t>(), n));
    uint32_t lb = 0, lc = 0;
    CK(cudaMemcpyAsync(&lb, ctx->rbase.as<uint32_t>() + (n - 1), 4, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&lc, ctx->rcnt.as<uint32_t>() + (n - 1), 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    *nr = uint64_t(lb) + lc;
    CK(ctx->rules.ensure(sizeof(DevRule) * std::max<uint64_t>(*nr, 1)));
    launch_rule_write_first(L, L2, n, ctx->rbase.as<uint32_t>(), ctx->rules.as<DevRule>(), s);
    CKR(check_launch(ctx, "rule_write"));
  } else {
    // all-hits: MidCheck on every survivor, one ExhaustiveCheck pass
    const uint32_t S = uint32_t(nsurv);
    CK(ctx->surv_target.ensure(4ull * std::max<uint32_t>(S, 1)));
    CK(ctx->midpass.ensure(std::max<uint32_t>(S, 1)));
    CK(ctx->flag.ensure(4ull * std::max<uint32_t>(S, 1)));
    CK(ctx->rbase.ensure(4ull * std::max<uint32_t>(S, 1)));
    CK(ctx->pairs.ensure(sizeof(PairRec) * std::max<uint32_t>(S, 1)));
    CK(ctx->pair_src.ensure(4ull * std::max<uint32_t>(S, 1)));
    CK(ctx->nchunks.ensure(8ull * std::max<uint32_t>(S, 1)));
    CK(ctx->cbase.ensure(8ull * std::max<uint32_t>(S, 1)));
    CK(ctx->nchunks_x.ensure(8ull * std::max<uint32_t>(S, 1)));
    CK(ctx->cbase_x.ensure(8ull * std::max<uint32_t>(S, 1)));
    CK(ctx->rejected.ensure(4ull * std::max<uint32_t>(S, 1)));
    R.pairs = ctx->pairs.as<PairRec>();
    R.pair_src = ctx->pair_src.as<uint32_t>();
    R.nchunks = ctx->nchunks.as<unsigned long long>();
    R.cbase = ctx->cbase.as<unsigned long long>();
    R.nchunks_x = ctx->nchunks_x.as<unsigned long long>();
    R.cbase_x = ctx->cbase_x.as<unsigned long long>();
    R.rejected = ctx->rejected.as<uint32_t>();
    R.npairs = ctx->npairs.as<uint32_t>();
    R.counter = ctx->counter.as<unsigned long long>();
    R.states = ctx->states.as<unsigned long long>();
    R.chunk_blocks = uint32_t(ctx->chunk_blocks);
    R.xunit = ctx->xbits ? kXBitsBlocks : kXScalarBlocks;
    R.compact = mode == Z80B_MODE_FIRST && ctx->compact ? 1u : 0u;
    R.nchunks_c = R.compact ? ctx->nchunks_c.as<unsigned long long>() : nullptr;
    R.cbase_c = R.compact ? ctx->cbase_c.as<unsigned long long>() : nullptr;
    R.wide = mode == Z80B_MODE_FIRST && ctx->wide ? 1u : 0u;
    R.nchunks_w = R.wide ? ctx->nchunks_w.as<unsigned long long>() : nullptr;
    R.cbase_w = R.wide ? ctx->cbase_w.as<unsigned long long>() : nullptr;
    R.nchunks_r = R.wide ? ctx->nchunks_r.as<unsigned long long>() : nullptr;
    R.cbase_r = R.wide ? ctx->cbase_r.as<unsigned long long>() : nullptr;
    if (S) {
      launch_surv_targets(q, n, ctx->surv_target.as<uint32_t>(), s);
      CKR(check_launch(ctx, "surv_targets"));
      launch_midcheck(T, P, q.surv, ctx->surv_target.as<uint32_t>(), S, ctx->midpass.as<uint8_t>(), s);
      CKR(check_launch(ctx, "midcheck"));
      CK(cudaMemsetAsync(R.npairs, 0, 4, s));
      launch_pairs_from_survivors(T, P, q, ctx->midpass.as<uint8_t>(), S, ctx->surv_target.as<uint32_t>(), R, s);
      CKR(check_launch(ctx, "pairs"));
      uint32_t np = 0;
      CKR(fetch(ctx, &np, R.npairs));
      mid_surv = np;
      exh_pairs = np;
      CK(cudaMemsetAsync(ctx->flag.p, 0, 4ull * S, s));
      if (np) {
        rounds = 1;
        // without the ExhaustiveCheck tier every pair keeps the zero
        // rejection flag its build wrote
        if (!opts.no_exhaustive) CKR(sweep_round(ctx, T, P, R, np));
        launch_rule_count_all(R, np, ctx->flag.as<uint32_t>(), s);
        CKR(check_launch(ctx, "rule_count_all"));
      }
      CKR(scan(ctx, ctx->flag.as<uint32_t>(), ctx->rbase.as<uint32_t>(), S));
      uint32_t lb = 0, lc = 0;
      CK(cudaMemcpyAsync(&lb, ctx->rbase.as<uint32_t>() + (S - 1), 4, cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(&lc, ctx->flag.as<uint32_t>() + (S - 1), 4, cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      *nr = uint64_t(lb) + lc;
      CK(ctx->rules.ensure(sizeof(DevRule) * std::max<uint64_t>(*nr, 1)));
      launch_rule_write_all(ctx->flag.as<uint32_t>(), ctx->rbase.as<uint32_t>(), S, q.surv, q.sdiff,
                            ctx->surv_target.as<uint32_t>(), ctx->rules.as<DevRule>(), s);
      CKR(check_launch(ctx, "rule_write_all"));
    }
  }
  tall.stop();
  CK(cudaStreamSynchronize(s));
  trace("pipeline done: %llu rules, %u rounds", (unsigned long long)*nr, rounds);
  if (st) {
    unsigned long long checks = 0, checked = 0, states[2] = {0, 0};
    CKR(fetch(ctx, &checks, ctx->checks.as<unsigned long long>()));
    CKR(fetch(ctx, &checked, ctx->checked.as<unsigned long long>()));
    CKR(fetch(ctx, states, ctx->states.as<unsigned long long>(), 2));
    st->targets += n;
    st->checks += checks;
    st->checked_ref += (mode == Z80B_MODE_FIRST) ? checked : 0;
    st->qc_survivors += nsurv;
    st->mid_survivors += mid_surv;
    st->exhaustive_pairs += exh_pairs;
    st->exhaustive_states += states[0];
    st->exhaustive_evaluated += states[1];
    st->rules += *nr;
    st->rounds += rounds;
    double a = 0, b = 0;
    ksum(ctx, &a, &b);
    st->qc_ms += a;
    st->exh_ms += b;
    st->device_ms += tall.ms();
  }
  ctx->n_rules_dev = *nr;
  return Z80B_OK;
}

// Converts device rules to z80b_rule records.
void to_rules(z80b_ctx* ctx, const DevRule* dr, size_t ndr, const uint32_t* targets, const uint8_t* tlens,
              uint32_t tlen, uint32_t stride, uint32_t mode, uint32_t tindex_offset, z80b_rule* out) {
  const PoolBufs& P = (mode == Z80B_MODE_ALL) ? (ctx->loaded.loaded ? ctx->loaded : ctx->firstop) : ctx->pool8;
  // Records go out with streaming stores when the output is 16-byte
  // aligned: the 64-byte records (tens of MB for a large search) are written
  // once and not read here, so no cache line is fetched before its write.
  const bool stream = (reinterpret_cast<uintptr_t>(out) & 15u) == 0;
  host_parallel(ndr, [&](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; i++) {
      const DevRule& r = dr[i];
      z80b_rule o;
      const uint32_t* t = targets + (size_t)r.target * stride;
      int tl = tlens ? tlens[r.target] : int(tlen);
      const PoolBufs& PC = (r.clen == 2) ? ctx->pairpool->pool : P;
      const uint32_t* c = PC.host_insn.data() + (size_t)r.cand * PC.len;
      int cl = int(PC.len);
      o.src_len = tl;
      o.rep_len = cl;
      // every field is written (no memset first): the record is 64 bytes
      // and a search returns hundreds of thousands of them
      for (int k = 0; k < 4; k++) o.src[k] = k < tl ? t[k] : 0u;
      for (int k = 0; k < 4; k++) o.rep[k] = k < cl ? c[k] : 0u;
      o.reserved = 0;
      o.bytes_saved = seq_bytes(t, tl) - seq_bytes(c, cl);
      o.cycles_saved = seq_tstates(t, tl) - seq_tstates(c, cl);
      o.dead_flags = (r.kind == 0) ? 0 : int(r.diff & 0xFFu);
      o.dead_regs = (r.kind == 0) ? 0 : int(r.diff >> 8);
      o.target_index = int(r.target + tindex_offset);
#if defined(__SSE2__)
      if (stream) {
        static_assert(sizeof(z80b_rule) % 16 == 0, "whole 16-byte stores");
        const __m128i* src = reinterpret_cast<const __m128i*>(&o);
        __m128i* dst = reinterpret_cast<__m128i*>(out + i);
        for (size_t k = 0; k < sizeof(z80b_rule) / 16; k++) _mm_stream_si128(dst + k, _mm_loadu_si128(src + k));
        continue;
      }
#endif
      out[i] = o;
    }
#if defined(__SSE2__)
    if (stream) _mm_sfence();
#endif
  });
}

int Reporter::update(z80b_ctx* ctx, uint32_t n, const Lanes& L, const Lanes& L2, uint32_t max_cand, bool phase2,
                     bool last) {
  if (!cb || n == 0) return Z80B_OK;
  cudaStream_t s = ctx->stream;
  if (done.size() != n) done.assign(n, 0);
  n1.resize(2 * size_t(n));
  w1.resize(2 * size_t(n));
  d1.resize(2 * size_t(n));
  CK(cudaMemcpyAsync(n1.data(), L.next, 8ull * n, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(w1.data(), L.win, 8ull * n, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(d1.data(), L.windiff, 4ull * n, cudaMemcpyDeviceToHost, s));
  if (phase2 && L2.win) {
    n2.resize(2 * size_t(n));
    w2.resize(2 * size_t(n));
    d2.resize(2 * size_t(n));
    CK(cudaMemcpyAsync(n2.data(), L2.next, 8ull * n, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(w2.data(), L2.win, 8ull * n, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(d2.data(), L2.windiff, 4ull * n, cudaMemcpyDeviceToHost, s));
  }
  CK(cudaStreamSynchronize(s));
  const uint32_t kResolvedBit = 0x80000000u;
  std::vector<DevRule> dr;
  std::vector<z80b_rule> out;
  for (uint32_t t = 0; t < n; t++) {
    if (done[t]) continue;
    bool final_all = true;
    dr.clear();
    for (int kind = 0; kind < 2 && final_all; kind++) {
      const size_t i = 2 * size_t(t) + size_t(kind);
      DevRule r{};
      r.target = t;
      r.kind = uint8_t(kind);
      if (w1[i] != kNone) {
        r.cand = w1[i];
        r.diff = kind ? d1[i] : uint16_t(0);
        r.clen = 1;
        dr.push_back(r);
      } else if (max_cand >= 2) {
        // no length-1 winner: the answer is the length-2 pass's, which starts
        // once every length-1 lane is done
        if (!phase2 || !L2.win) {
          final_all = false;
        } else if (w2[i] != kNone) {
          r.cand = w2[i];
          r.diff = kind ? d2[i] : uint16_t(0);
          r.clen = 2;
          dr.push_back(r);
        } else if (!(n2[i] & kResolvedBit)) {
          final_all = last;
        }
      } else if (!(n1[i] & kResolvedBit)) {
        final_all = last;  // a lane without survivors is never offered to a round
      }
    }
    if (!final_all) continue;
    done[t] = 1;
    out.resize(dr.size());
    if (!dr.empty()) to_rules(ctx, dr.data(), dr.size(), targets, tlens, tlen, stride, Z80B_MODE_FIRST, 0, out.data());
    cb(user, t, out.data(), uint32_t(out.size()));
  }
  return Z80B_OK;
}

// Uploads the job's arrays straight from the caller's buffers (pinned
// buffers make this a DMA).  keep_host copies the targets for a later
// z80b_fetch_rules; z80b_search converts rules while the caller's buffers
// are still valid and skips the copy.
int upload_targets(z80b_ctx* ctx, Staged& S, const z80b_job* job, DevTargets* T, bool keep_host) {
  const uint32_t n = job->n_targets;
  const size_t words = (size_t)n * job->target_stride;
  S.targets.clear();
  if (keep_host) S.targets.assign(job->targets, job->targets + words);
  S.lens.clear();
  S.dead.clear();
  S.dregs.clear();
  if (job->target_lens) S.lens.assign(job->target_lens, job->target_lens + n);
  if (job->dead_flags) S.dead.assign(job->dead_flags, job->dead_flags + n);
  if (job->dead_regs) S.dregs.assign(job->dead_regs, job->dead_regs + n);
  S.job = *job;
  S.opts = PipeOpts{};
  S.opts.mode = job->mode;
  S.opts.max_cand = job->max_cand_len;
  S.opts.no_exhaustive = (job->flags & Z80B_JOB_NO_EXHAUSTIVE) != 0;
  if (job->max_cand_len >= 2)
    for (uint32_t i = 0; i < n; i++) {
      const uint32_t dr = job->dead_regs ? job->dead_regs[i] & 0x3Fu : 0u;
      const uint32_t df = job->dead_flags ? job->dead_flags[i] : job->global_dead_flags;
      if (dr || df) S.opts.dreg_masks |= 1ull << dr;
    }
  cudaStream_t s = ctx->stream;
  CK(S.d_targets.ensure(4ull * std::max<size_t>(words, 1)));
  S.up_chunks = 0;
  if (!keep_host && n >= kUpChunkMin) {
    // in chunks on the copy stream, so that the QuickCheck count of the
    // first chunks runs while the rest are copied
    if (!ctx->copy_stream) {
      CK(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
      for (auto& e : ctx->up_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    CK(cudaEventRecord(ctx->up_ev[kUpChunks], s));  // after the stream's earlier use of the buffers
    CK(cudaStreamWaitEvent(ctx->copy_stream, ctx->up_ev[kUpChunks], 0));
    const size_t stride = job->target_stride;
    for (int k = 0; k < kUpChunks; k++) {
      const size_t lo = (size_t)n * k / kUpChunks, hi = (size_t)n * (k + 1) / kUpChunks;
      if (hi > lo)
        CK(cudaMemcpyAsync(S.d_targets.as<uint32_t>() + lo * stride, job->targets + lo * stride,
                           4ull * (hi - lo) * stride, cudaMemcpyHostToDevice, ctx->copy_stream));
      CK(cudaEventRecord(ctx->up_ev[k], ctx->copy_stream));
      S.up_hi[k] = uint32_t(hi);
    }
    S.up_chunks = kUpChunks;
  } else if (n) {
    CK(cudaMemcpyAsync(S.d_targets.p, job->targets, 4ull * words, cudaMemcpyHostToDevice, s));
  }
  *T = DevTargets{};
  T->insn = S.d_targets.as<uint32_t>();
  T->n = n;
  T->stride = job->target_stride;
  T->fixed_len = job->target_len;
  T->global_dead = job->global_dead_flags;
  if (!S.lens.empty()) {
    CK(S.d_lens.ensure(n));
    CK(cudaMemcpyAsync(S.d_lens.p, S.lens.data(), n, cudaMemcpyHostToDevice, s));
    T->len = S.d_lens.as<uint8_t>();
  }
  if (!S.dead.empty()) {
    CK(S.d_dead.ensure(n));
    CK(cudaMemcpyAsync(S.d_dead.p, S.dead.data(), n, cudaMemcpyHostToDevice, s));
    T->dead = S.d_dead.as<uint8_t>();
  }
  if (!S.dregs.empty()) {
    CK(S.d_dregs.ensure(n));
    CK(cudaMemcpyAsync(S.d_dregs.p, S.dregs.data(), n, cudaMemcpyHostToDevice, s));
    T->dead_regs = S.d_dregs.as<uint8_t>();
  }
  S.valid = true;
  return Z80B_OK;
}

// Reads the first nr device rules into the context's pinned staging buffer
// (*out points there until the next call).
int rules_to_host(z80b_ctx* ctx, uint64_t nr, const DevRule** out) {
  *out = nullptr;
  if (!nr) return Z80B_OK;
  CK(ctx->h_rules.ensure(sizeof(DevRule) * nr));
  CK(cudaMemcpyAsync(ctx->h_rules.p, ctx->rules.p, sizeof(DevRule) * nr, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  *out = ctx->h_rules.as<DevRule>();
  return Z80B_OK;
}

DevTargets staged_targets(Staged& S) {
  DevTargets T{};
  T.insn = S.d_targets.as<uint32_t>();
  T.n = S.job.n_targets;
  T.stride = S.job.target_stride;
  T.fixed_len = S.job.target_len;
  T.global_dead = S.job.global_dead_flags;
  if (!S.lens.empty()) T.len = S.d_lens.as<uint8_t>();
  if (!S.dead.empty()) T.dead = S.d_dead.as<uint8_t>();
  if (!S.dregs.empty()) T.dead_regs = S.d_dregs.as<uint8_t>();
  return T;
}

// Runs the staged job (batched or plain path) and leaves rules on the device
// (batched) or appends them to host_rules (plain).
int run_staged(z80b_ctx* ctx, z80b_stats* st, uint64_t* nr, std::vector<z80b_rule>* host_rules,
               const uint32_t* host_targets) {
  Staged& S = ctx->staged;
  DevTargets T = staged_targets(S);
  const z80b_job& job = S.job;
  if (job.path == Z80B_PATH_BATCHED) return run_pipeline(ctx, T, S.opts, st, nr);
  // plain: one target per pipeline launch, synchronizing in between
  uint64_t total = 0;
  std::vector<DevRule> dr;
  for (uint32_t i = 0; i < T.n; i++) {
    DevTargets one = T;
    one.insn = T.insn + (size_t)i * T.stride;
    one.n = 1;
    if (T.len) one.len = T.len + i;
    if (T.dead) one.dead = T.dead + i;
    if (T.dead_regs) one.dead_regs = T.dead_regs + i;
    uint64_t k = 0;
    CKR(run_pipeline(ctx, one, S.opts, st, &k));
    if (k) {
      dr.resize(k);
      CK(cudaMemcpyAsync(dr.data(), ctx->rules.p, sizeof(DevRule) * k, cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
      if (host_rules) {
        size_t off = host_rules->size();
        host_rules->resize(off + k);
        to_rules(ctx, dr.data(), dr.size(), host_targets + (size_t)i * T.stride, S.lens.empty() ? nullptr : &S.lens[i],
                 job.target_len, T.stride, job.mode, i, host_rules->data() + off);
      }
    }
    total += k;
  }
  *nr = total;
  return Z80B_OK;
}

}  // namespace

// ============================================================== C ABI

extern "C" {

int z80b_version(void) { return 1; }

const char* z80b_status_string(int s) {
  switch (s) {
    case Z80B_OK: return "ok";
    case Z80B_EINVAL: return "invalid argument";
    case Z80B_ENOMEM: return "out of device memory";
    case Z80B_ECUDA: return "CUDA error";
    case Z80B_ETIMEOUT: return "device wait timed out";
    case Z80B_ECAPACITY: return "output buffer too small";
    case Z80B_ENODEV: return "no usable CUDA device";
    case Z80B_ESTATE: return "call out of order";
  }
  return "unknown status";
}

const char* z80b_last_error(const z80b_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int z80b_init(int device, z80b_ctx** out) {
  if (!out) return Z80B_EINVAL;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return Z80B_ENODEV;
  if (device < 0 || device >= ndev) return Z80B_EINVAL;
  cudaDeviceProp prop{};
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return Z80B_ENODEV;
  if (prop.major < 10) return Z80B_ENODEV;  // built for sm_100a only
  trace("init device %d (%s, cc %d.%d, %d SMs)", device, prop.name, prop.major, prop.minor,
        prop.multiProcessorCount);
  z80b_ctx* ctx = new z80b_ctx();
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return Z80B_ECUDA;
  }
  for (auto& e : ctx->ev) cudaEventCreate(&e);
  trace("init: stream and events");
  dev_upload_tables(ctx->stream);
  trace("init: tables queued");
  const auto& p8 = pool8();
  int r = build_pool(ctx, ctx->pool8, p8.data(), uint32_t(p8.size()), 1, nullptr, false);
  if (r != Z80B_OK) {
    z80b_destroy(ctx);
    return r;
  }
  trace("init done");
  *out = ctx;
  return Z80B_OK;
}

void z80b_destroy(z80b_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto& e : ctx->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : ctx->kev) cudaEventDestroy(e);
  if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
  for (auto& e : ctx->up_ev)
    if (e) cudaEventDestroy(e);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  for (int i = 0; i < 4; i++) {
    if (ctx->join_ev[i]) cudaEventDestroy(ctx->join_ev[i]);
    if (ctx->side[i]) cudaStreamDestroy(ctx->side[i]);
  }
  cudaStream_t s = ctx->stream;
  delete ctx;
  if (s) cudaStreamDestroy(s);
}

int z80b_fingerprints(z80b_ctx* ctx, const uint32_t* seqs, uint32_t n, uint32_t len, uint8_t* out) {
  if (!ctx) return Z80B_EINVAL;
  if ((n && (!seqs || !out)) || len < 1 || len > uint32_t(kMaxSeq)) return fail(ctx, Z80B_EINVAL, "bad arguments");
  if (!n) return Z80B_OK;
  for (uint32_t i = 0; i < n; i++)
    if (!valid_seq(seqs + (size_t)i * len, int(len))) return fail(ctx, Z80B_EINVAL, "sequence %u: opcode > 454", i);
  cudaSetDevice(ctx->device);
  CK(ctx->v_tgt.ensure(4ull * n * len));
  CK(ctx->v_out.ensure(80ull * n));
  CK(cudaMemcpyAsync(ctx->v_tgt.p, seqs, 4ull * n * len, cudaMemcpyHostToDevice, ctx->stream));
  launch_fingerprints(ctx->v_tgt.as<uint32_t>(), n, len, ctx->v_out.as<uint8_t>(), ctx->stream);
  CKR(check_launch(ctx, "fingerprints"));
  CK(cudaMemcpyAsync(out, ctx->v_out.p, 80ull * n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return Z80B_OK;
}

int z80b_exec(z80b_ctx* ctx, const z80b_state* in, const uint32_t* seqs, const uint8_t* lens, uint32_t len,
              uint32_t stride, uint32_t n, z80b_state* out) {
  if (!ctx) return Z80B_EINVAL;
  if (n && (!in || !seqs || !out)) return fail(ctx, Z80B_EINVAL, "null pointer");
  if (stride < 1 || stride > 64) return fail(ctx, Z80B_EINVAL, "bad stride");
  if (!n) return Z80B_OK;
  for (uint32_t i = 0; i < n; i++) {
    uint32_t l = lens ? lens[i] : len;
    if (l > uint32_t(kMaxSeq) || l > stride) return fail(ctx, Z80B_EINVAL, "sequence %u: bad length", i);
    if (!valid_seq(seqs + (size_t)i * stride, int(l))) return fail(ctx, Z80B_EINVAL, "sequence %u: opcode > 454", i);
  }
  cudaSetDevice(ctx->device);
  std::vector<uint32_t> packed(3ull * n);
  for (uint32_t i = 0; i < n; i++) {
    const z80b_state& s = in[i];
    packed[3 * i] = uint32_t(s.a) | uint32_t(s.f) << 8 | uint32_t(s.b) << 16 | uint32_t(s.c) << 24;
    packed[3 * i + 1] = uint32_t(s.d) | uint32_t(s.e) << 8 | uint32_t(s.h) << 16 | uint32_t(s.l) << 24;
    packed[3 * i + 2] = uint32_t(s.sp) | uint32_t(s.m) << 16;
  }
  CK(ctx->v_in.ensure(12ull * n));
  CK(ctx->v_outs.ensure(12ull * n));
  CK(ctx->v_tgt.ensure(4ull * n * stride));
  CK(ctx->v_tl.ensure(n));
  CK(cudaMemcpyAsync(ctx->v_in.p, packed.data(), 12ull * n, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->v_tgt.p, seqs, 4ull * n * stride, cudaMemcpyHostToDevice, ctx->stream));
  if (lens) CK(cudaMemcpyAsync(ctx->v_tl.p, lens, n, cudaMemcpyHostToDevice, ctx->stream));
  launch_exec(ctx->v_in.as<uint32_t>(), ctx->v_tgt.as<uint32_t>(), lens ? ctx->v_tl.as<uint8_t>() : nullptr, len,
              stride, n, ctx->v_outs.as<uint32_t>(), ctx->stream);
  CKR(check_launch(ctx, "exec"));
  CK(cudaMemcpyAsync(packed.data(), ctx->v_outs.p, 12ull * n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  for (uint32_t i = 0; i < n; i++) {
    z80b_state& s = out[i];
    uint32_t w0 = packed[3 * i], w1 = packed[3 * i + 1], w2 = packed[3 * i + 2];
    s.a = uint8_t(w0); s.f = uint8_t(w0 >> 8); s.b = uint8_t(w0 >> 16); s.c = uint8_t(w0 >> 24);
    s.d = uint8_t(w1); s.e = uint8_t(w1 >> 8); s.h = uint8_t(w1 >> 16); s.l = uint8_t(w1 >> 24);
    s.sp = uint16_t(w2); s.m = uint8_t(w2 >> 16); s.pad = 0;
  }
  return Z80B_OK;
}

int z80b_load_candidates(z80b_ctx* ctx, const uint32_t* cands, uint32_t count, uint32_t seq_len) {
  if (!ctx) return Z80B_EINVAL;
  if ((count && !cands) || seq_len < 1 || seq_len > 3) return fail(ctx, Z80B_EINVAL, "bad arguments");
  for (uint32_t i = 0; i < count; i++)
    if (!valid_seq(cands + (size_t)i * seq_len, int(seq_len)))
      return fail(ctx, Z80B_EINVAL, "candidate %u: opcode > 454", i);
  cudaSetDevice(ctx->device);
  return build_pool(ctx, ctx->loaded, cands, count, seq_len, nullptr, false);
}

int z80b_quickcheck(z80b_ctx* ctx, const uint8_t* fp80, uint32_t dead_flags, uint32_t* hits, uint32_t cap,
                    uint32_t* n_hits) {
  if (!ctx) return Z80B_EINVAL;
  if (!fp80 || !n_hits || (cap && !hits)) return fail(ctx, Z80B_EINVAL, "null pointer");
  if (!ctx->loaded.loaded) return fail(ctx, Z80B_ESTATE, "z80b_load_candidates has not been called");
  cudaSetDevice(ctx->device);
  // fingerprint bytes -> packed words (F byte masked on the device)
  uint32_t w[24];
  for (int v = 0; v < 8; v++) {
    const uint8_t* p = fp80 + v * 10;
    w[3 * v] = uint32_t(p[0]) | uint32_t(p[1]) << 8 | uint32_t(p[2]) << 16 | uint32_t(p[3]) << 24;
    w[3 * v + 1] = uint32_t(p[4]) | uint32_t(p[5]) << 8 | uint32_t(p[6]) << 16 | uint32_t(p[7]) << 24;
    w[3 * v + 2] = uint32_t(p[8]) << 8 | uint32_t(p[9]);
  }
  const uint32_t dev_cap = ctx->loaded.n;
  CK(ctx->fpq.ensure(sizeof w));
  CK(ctx->hits.ensure(4ull * std::max<uint32_t>(dev_cap, 1)));
  CK(ctx->nhits.ensure(4));
  CK(cudaMemcpyAsync(ctx->fpq.p, w, sizeof w, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(ctx->nhits.p, 0, 4, ctx->stream));
  launch_fp_query(ctx->loaded.dev, ctx->fpq.as<uint32_t>(), dead_flags & 0xFFu, ctx->hits.as<uint32_t>(),
                  ctx->nhits.as<uint32_t>(), dev_cap, ctx->stream);
  CKR(check_launch(ctx, "fp_query"));
  uint32_t nh = 0;
  CKR(fetch(ctx, &nh, ctx->nhits.as<uint32_t>()));
  std::vector<uint32_t> h(nh);
  if (nh) CKR(fetch(ctx, h.data(), ctx->hits.as<uint32_t>(), nh));
  std::sort(h.begin(), h.end());
  *n_hits = nh;
  for (uint32_t i = 0; i < nh && i < cap; i++) hits[i] = h[i];
  return nh > cap ? fail(ctx, Z80B_ECAPACITY, "%u hits, capacity %u", nh, cap) : Z80B_OK;
}

int z80b_verify_pairs(z80b_ctx* ctx, const uint32_t* tgt, const uint8_t* tlens, const uint32_t* cand,
                      const uint8_t* clens, uint32_t stride, uint32_t n, const uint8_t* dead, uint32_t tiers,
                      uint8_t* out, uint8_t* flagdiff) {
  if (!ctx) return Z80B_EINVAL;
  if (n && (!tgt || !tlens || !cand || !clens || !out)) return fail(ctx, Z80B_EINVAL, "null pointer");
  if (stride < 1 || stride > 64) return fail(ctx, Z80B_EINVAL, "bad stride");
  if (!n) return Z80B_OK;
  for (uint32_t i = 0; i < n; i++) {
    if (tlens[i] < 1 || tlens[i] > kMaxSeq || tlens[i] > stride || clens[i] < 1 || clens[i] > kMaxSeq - 1 ||
        clens[i] > stride)
      return fail(ctx, Z80B_EINVAL, "pair %u: bad length", i);
    if (!valid_seq(tgt + (size_t)i * stride, tlens[i]) || !valid_seq(cand + (size_t)i * stride, clens[i]))
      return fail(ctx, Z80B_EINVAL, "pair %u: opcode > 454", i);
  }
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  CK(ctx->v_tgt.ensure(4ull * n * stride));
  CK(ctx->v_cand.ensure(4ull * n * stride));
  CK(ctx->v_tl.ensure(n));
  CK(ctx->v_cl.ensure(n));
  CK(ctx->v_dead.ensure(n));
  CK(ctx->v_out.ensure(n));
  CK(ctx->v_fd.ensure(n));
  CK(cudaMemcpyAsync(ctx->v_tgt.p, tgt, 4ull * n * stride, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(ctx->v_cand.p, cand, 4ull * n * stride, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(ctx->v_tl.p, tlens, n, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(ctx->v_cl.p, clens, n, cudaMemcpyHostToDevice, s));
  if (dead) CK(cudaMemcpyAsync(ctx->v_dead.p, dead, n, cudaMemcpyHostToDevice, s));
  else CK(cudaMemsetAsync(ctx->v_dead.p, 0, n, s));
  launch_verify_small(ctx->v_tgt.as<uint32_t>(), ctx->v_tl.as<uint8_t>(), ctx->v_cand.as<uint32_t>(),
                      ctx->v_cl.as<uint8_t>(), stride, n, ctx->v_dead.as<uint8_t>(), tiers, ctx->v_out.as<uint8_t>(),
                      ctx->v_fd.as<uint8_t>(), s);
  CKR(check_launch(ctx, "verify_small"));
  std::vector<uint8_t> res(n), fd(n);
  CK(cudaMemcpyAsync(res.data(), ctx->v_out.p, n, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(fd.data(), ctx->v_fd.p, n, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (tiers & 4u) {
    // ExhaustiveCheck of every pair: pairs are (i, i) of a target batch and
    // a candidate pool with per-candidate lengths
    DevTargets T{};
    T.insn = ctx->v_tgt.as<uint32_t>();
    T.len = ctx->v_tl.as<uint8_t>();
    T.dead = ctx->v_dead.as<uint8_t>();
    T.n = n;
    T.stride = stride;
    DevPool P{};
    P.insn = ctx->v_cand.as<uint32_t>();
    P.lens = ctx->v_cl.as<uint8_t>();
    P.n = n;
    P.stride = stride;
    std::vector<PairRec> pr(n);
    std::vector<unsigned long long> cb(n), cbx(n);
    unsigned long long tot = 0, totx = 0;  // chunks of the bit-sliced / A-independent pairs
    for (uint32_t i = 0; i < n; i++) {
      uint16_t rd = uint16_t(seq_reads(tgt + (size_t)i * stride, tlens[i]) | seq_reads(cand + (size_t)i * stride, clens[i]));
      Sweep w = sweep_for(rd);
      pr[i] = PairRec{};
      pr[i].target = i;
      pr[i].cand = i;
      pr[i].reads = rd;
      pr[i].nblocks = w.states / 256;
      pr[i].keepF = uint8_t(~(dead ? dead[i] : 0u));
      pr[i].keepR = 0x3F;
      // sweep units (see the sweep kernel): 128 A-blocks for A-independent
      // pairs, 4 A-blocks (bit-sliced) for the others
      unsigned long long units = (pr[i].nblocks + 3) / 4;
      if (seq_aflow(tgt + (size_t)i * stride, tlens[i]) && seq_aflow(cand + (size_t)i * stride, clens[i])) {
        pr[i].keepR |= 0x40;
        units = (pr[i].nblocks + 127) / 128;
      }
      unsigned long long c = (units + ctx->chunk_blocks - 1) / uint64_t(ctx->chunk_blocks);
      if (c > (1ull << 20)) c = 1ull << 20;
      cb[i] = tot;
      cbx[i] = totx;
      if (pr[i].keepR & 0x40) totx += c;
      else tot += c;
    }
    CK(ctx->pairs.ensure(sizeof(PairRec) * n));
    CK(ctx->cbase.ensure(8ull * n));
    CK(ctx->cbase_x.ensure(8ull * n));
    CK(ctx->rejected.ensure(4ull * n));
    CK(ctx->counter.ensure(40));
    CK(ctx->states.ensure(16));
    CK(cudaMemcpyAsync(ctx->pairs.p, pr.data(), sizeof(PairRec) * n, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->cbase.p, cb.data(), 8ull * n, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->cbase_x.p, cbx.data(), 8ull * n, cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(ctx->rejected.p, 0, 4ull * n, s));
    CK(cudaMemsetAsync(ctx->counter.p, 0, 16, s));
    RoundBuf R{};
    R.pairs = ctx->pairs.as<PairRec>();
    R.cbase = ctx->cbase.as<unsigned long long>();
    R.cbase_x = ctx->cbase_x.as<unsigned long long>();
    R.rejected = ctx->rejected.as<uint32_t>();
    R.counter = ctx->counter.as<unsigned long long>();
    R.states = ctx->states.as<unsigned long long>();
    const int nl = launch_exhaustive(T, P, R, n, tot, totx, 0, 0, 0, ctx->exh_k, s);
    CKR(check_launch(ctx, "exhaustive"));
    if (nl > 1) ctx->launches += uint32_t(nl - 1);
    std::vector<uint32_t> rej(n);
    CK(cudaMemcpyAsync(rej.data(), ctx->rejected.p, 4ull * n, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (uint32_t i = 0; i < n; i++)
      if (!rej[i]) res[i] |= 4;
  }
  std::memcpy(out, res.data(), n);
  if (flagdiff) std::memcpy(flagdiff, fd.data(), n);
  return Z80B_OK;
}

int z80b_set_option(z80b_ctx* ctx, int option, int value) {
  if (!ctx) return Z80B_EINVAL;
  switch (option) {
    case Z80B_OPT_EXH_LANE_STATES:
      if (value != 1 && value != 2 && value != 4 && value != 8)
        return fail(ctx, Z80B_EINVAL, "lane states must be 1, 2, 4 or 8");
      ctx->exh_k = value;
      return Z80B_OK;
    case Z80B_OPT_EXH_CHUNK_BLOCKS:
      if (value < 1 || value > 4096) return fail(ctx, Z80B_EINVAL, "chunk blocks must be 1..4096");
      ctx->chunk_blocks = value;
      return Z80B_OK;
    case Z80B_OPT_STREAM_PRIORITY: {
      if (value < -1 || value > 1) return fail(ctx, Z80B_EINVAL, "stream priority must be -1, 0 or 1");
      int lo = 0, hi = 0;  // numerically lower is higher priority
      CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
      const int prio = value < 0 ? hi : (value > 0 ? lo : 0);
      cudaSetDevice(ctx->device);
      CK(cudaStreamSynchronize(ctx->stream));
      cudaStream_t ns = nullptr;
      CK(cudaStreamCreateWithPriority(&ns, cudaStreamNonBlocking, prio));
      CK(cudaStreamDestroy(ctx->stream));
      ctx->stream = ns;
      ctx->priority = value;
      return Z80B_OK;
    }
    case Z80B_OPT_QC_INDEX:
      if (value != 0 && value != 1) return fail(ctx, Z80B_EINVAL, "QuickCheck index option must be 0 or 1");
      ctx->qc_index = value;
      return Z80B_OK;
    case Z80B_OPT_XINDEP_BITS:
      if (value != 0 && value != 1) return fail(ctx, Z80B_EINVAL, "A-independent sweep option must be 0 or 1");
      ctx->xbits = value;
      return Z80B_OK;
    case Z80B_OPT_COMPACT_SWEEP:
      if (value != 0 && value != 1) return fail(ctx, Z80B_EINVAL, "compact sweep option must be 0 or 1");
      ctx->compact = value;
      return Z80B_OK;
    case Z80B_OPT_GRAPH_ROUNDS:
      if (value != 0 && value != 1) return fail(ctx, Z80B_EINVAL, "graph rounds option must be 0 or 1");
      ctx->graph_rounds = value;
      return Z80B_OK;
    case Z80B_OPT_WIDE_SWEEP:
      if (value != 0 && value != 1) return fail(ctx, Z80B_EINVAL, "wide sweep option must be 0 or 1");
      ctx->wide = value;
      return Z80B_OK;
    case Z80B_OPT_CONCURRENT_SWEEPS:
      if (value != 0 && value != 1) return fail(ctx, Z80B_EINVAL, "concurrent sweeps option must be 0 or 1");
      ctx->concurrent_sweeps = value;
      return Z80B_OK;
    case Z80B_OPT_QC_SINGLE_PASS:
      if (value != 0 && value != 1) return fail(ctx, Z80B_EINVAL, "QuickCheck single-pass option must be 0 or 1");
      ctx->qc_single = value;
      return Z80B_OK;
  }
  return fail(ctx, Z80B_EINVAL, "unknown option %d", option);
}

int z80b_get_option(const z80b_ctx* ctx, int option, int* value) {
  if (!ctx || !value) return Z80B_EINVAL;
  switch (option) {
    case Z80B_OPT_EXH_LANE_STATES: *value = ctx->exh_k; return Z80B_OK;
    case Z80B_OPT_EXH_CHUNK_BLOCKS: *value = ctx->chunk_blocks; return Z80B_OK;
    case Z80B_OPT_STREAM_PRIORITY: *value = ctx->priority; return Z80B_OK;
    case Z80B_OPT_QC_INDEX: *value = ctx->qc_index; return Z80B_OK;
    case Z80B_OPT_XINDEP_BITS: *value = ctx->xbits; return Z80B_OK;
    case Z80B_OPT_COMPACT_SWEEP: *value = ctx->compact; return Z80B_OK;
    case Z80B_OPT_GRAPH_ROUNDS: *value = ctx->graph_rounds; return Z80B_OK;
    case Z80B_OPT_WIDE_SWEEP: *value = ctx->wide; return Z80B_OK;
    case Z80B_OPT_CONCURRENT_SWEEPS: *value = ctx->concurrent_sweeps; return Z80B_OK;
    case Z80B_OPT_QC_SINGLE_PASS: *value = ctx->qc_single; return Z80B_OK;
  }
  return Z80B_EINVAL;
}

// The sweep kernels of a kSweep* mask, by name ("k_exhaustive<K,CLS>" joined
// by '+').
static void sweep_kernel_names(uint32_t mask, char* out, size_t cap) {
  std::string r;
  auto add = [&](const char* n) {
    if (!r.empty()) r += "+";
    r += n;
  };
  if (mask & kSweepBits) add("k_exhaustive<1,0>");
  if (mask & kSweepXBits) add("k_exhaustive<1,2>");
  if (mask & kSweepCompact) add("k_exhaustive<1,3>");
  if (mask & kSweepWide) add("k_exhaustive<1,4>");
  if (mask & kSweepRegs) add("k_exhaustive<1,5>");
  const char* scalar[4] = {"k_exhaustive<1,1>", "k_exhaustive<2,1>", "k_exhaustive<4,1>", "k_exhaustive<8,1>"};
  for (int i = 0; i < 4; i++)
    if (mask & (kSweepScalarK1 << i)) add(scalar[i]);
  std::snprintf(out, cap, "%s", r.c_str());
}

// Runs the sample job once for every sweep configuration of the grid and
// keeps the fastest (device time of the whole pipeline): the kernel for
// A-independent pairs (bit-sliced, or scalar with 1, 2, 4 or 8 states per
// lane per dispatch), units per work chunk, and whether pairs that fit the
// compact states take the compact kernels (both the A/F/B/C state and the
// wide one, or neither).  Every cell of the
// grid is a distinct kernel configuration; each trial records the sweep
// kernels it launched.
int z80b_autotune(z80b_ctx* ctx, const z80b_job* sample, z80b_tune_result* out) {
  if (!ctx) return Z80B_EINVAL;
  CKR(validate_job(ctx, sample));
  CKR(validate_targets(ctx, sample));
  if (sample->path != Z80B_PATH_BATCHED) return fail(ctx, Z80B_EINVAL, "autotune runs the batched path");
  cudaSetDevice(ctx->device);
  DevTargets T;
  CKR(upload_targets(ctx, ctx->staged, sample, &T, true));
  // A-independent kernel: {xbits, lane states}
  const int xv[5][2] = {{1, 0}, {0, 1}, {0, 2}, {0, 4}, {0, 8}};
  const int cs[4] = {8, 32, 128, 512};
  const int k0 = ctx->exh_k;
  double best = 1e300;
  int bk = ctx->exh_k, bc = ctx->chunk_blocks, bx = ctx->xbits, bm = ctx->compact;
  z80b_tune_result r{};
  for (int m = 0; m < 2; m++)
    for (int a = 0; a < 5; a++)
      for (int b = 0; b < 4; b++) {
        ctx->xbits = xv[a][0];
        ctx->exh_k = xv[a][1] ? xv[a][1] : k0;
        ctx->chunk_blocks = cs[b];
        ctx->compact = m;
        ctx->wide = m;
        z80b_stats st{};
        uint64_t nr = 0;
        CKR(run_pipeline(ctx, T, ctx->staged.opts, &st, &nr));  // warm
        std::memset(&st, 0, sizeof st);
        ctx->sweep_kernels = 0;
        CKR(run_pipeline(ctx, T, ctx->staged.opts, &st, &nr));
        if (r.n_trials < Z80B_TUNE_MAX_TRIALS) {
          z80b_tune_trial& t = r.trials[r.n_trials++];
          t.xindep_bits = xv[a][0];
          t.lane_states = xv[a][1];
          t.chunk_blocks = cs[b];
          t.compact = m;
          t.ms = st.device_ms;
          sweep_kernel_names(ctx->sweep_kernels, t.kernels, sizeof t.kernels);
        }
        if (st.device_ms < best) {
          best = st.device_ms;
          bk = ctx->exh_k;
          bc = cs[b];
          bx = xv[a][0];
          bm = m;
        }
      }
  ctx->exh_k = bk;
  ctx->chunk_blocks = bc;
  ctx->xbits = bx;
  ctx->compact = bm;
  ctx->wide = bm;
  r.lane_states = bk;
  r.chunk_blocks = bc;
  r.xindep_bits = bx;
  r.compact = bm;
  if (out) *out = r;
  trace("autotune: xbits %d, lane states %d, chunk %d, compact %d (%.3f ms)", bx, bk, bc, bm, best);
  return Z80B_OK;
}

int z80b_stage_job(z80b_ctx* ctx, const z80b_job* job) {
  if (!ctx) return Z80B_EINVAL;
  CKR(validate_job(ctx, job));
  cudaSetDevice(ctx->device);
  DevTargets T;
  CKR(upload_targets(ctx, ctx->staged, job, &T, true));
  const int v = validate_targets(ctx, job);  // while the copy runs
  CK(cudaStreamSynchronize(ctx->stream));
  if (v != Z80B_OK) ctx->staged.valid = false;
  return v;
}

int z80b_run_staged(z80b_ctx* ctx, uint64_t* n_rules, z80b_stats* stats) {
  if (!ctx) return Z80B_EINVAL;
  if (!ctx->staged.valid) return fail(ctx, Z80B_ESTATE, "no staged job");
  if (ctx->staged.job.path != Z80B_PATH_BATCHED) return fail(ctx, Z80B_EINVAL, "staged runs use the batched path");
  cudaSetDevice(ctx->device);
  if (stats) std::memset(stats, 0, sizeof *stats);
  ctx->launches = 0;
  uint64_t nr = 0;
  CKR(run_staged(ctx, stats, &nr, nullptr, ctx->staged.targets.data()));
  if (stats) stats->launches = ctx->launches;
  if (n_rules) *n_rules = nr;
  return Z80B_OK;
}

int z80b_fetch_rules(z80b_ctx* ctx, z80b_rule* out, uint64_t cap, uint64_t* n_rules) {
  if (!ctx) return Z80B_EINVAL;
  if (!ctx->staged.valid) return fail(ctx, Z80B_ESTATE, "no staged job");
  uint64_t nr = ctx->n_rules_dev;
  if (n_rules) *n_rules = nr;
  if (nr > cap) return fail(ctx, Z80B_ECAPACITY, "%llu rules, capacity %llu", (unsigned long long)nr,
                            (unsigned long long)cap);
  if (nr && !out) return fail(ctx, Z80B_EINVAL, "null output");
  const DevRule* dr = nullptr;
  CKR(rules_to_host(ctx, nr, &dr));
  const Staged& S = ctx->staged;
  to_rules(ctx, dr, nr, S.targets.data(), S.lens.empty() ? nullptr : S.lens.data(), S.job.target_len,
           S.job.target_stride, S.job.mode, 0, out);
  return Z80B_OK;
}

static int search_impl(z80b_ctx* ctx, const z80b_job* job, z80b_rule* out, uint64_t cap, uint64_t* n_rules,
                       z80b_stats* stats, Reporter* rep) {
  if (!ctx) return Z80B_EINVAL;
  if (!n_rules) return fail(ctx, Z80B_EINVAL, "n_rules is null");
  CKR(validate_job(ctx, job));
  cudaSetDevice(ctx->device);
  if (stats) std::memset(stats, 0, sizeof *stats);
  ctx->launches = 0;
  DevTargets T;
  CKR(upload_targets(ctx, ctx->staged, job, &T, false));
  ctx->staged.valid = false;  // this job's targets are not kept for z80b_fetch_rules
  {
    // the host scan of the targets runs while their copy is in flight; on
    // an error the copy ends before the caller gets its buffers back
    const int v = validate_targets(ctx, job);
    if (v != Z80B_OK) {
      cudaStreamSynchronize(ctx->stream);
      if (ctx->staged.up_chunks) cudaStreamSynchronize(ctx->copy_stream);
      return v;
    }
  }
  uint64_t nr = 0;
  if (job->path == Z80B_PATH_PLAIN) {
    std::vector<z80b_rule> hr;
    // one target per launch: the whole upload first (nothing of the copy
    // is left in flight whatever run_staged returns)
    if (ctx->staged.up_chunks) CK(cudaStreamSynchronize(ctx->copy_stream));
    CKR(run_staged(ctx, stats, &nr, &hr, job->targets));
    *n_rules = nr;
    if (stats) stats->launches = ctx->launches;
    for (uint64_t i = 0; i < nr && i < cap; i++) out[i] = hr[i];
    return nr > cap ? fail(ctx, Z80B_ECAPACITY, "%llu rules, capacity %llu", (unsigned long long)nr,
                           (unsigned long long)cap)
                    : Z80B_OK;
  }
  PipeOpts opts = ctx->staged.opts;
  opts.up_chunks = ctx->staged.up_chunks;
  opts.up_hi = ctx->staged.up_hi;
  if (rep && job->mode == Z80B_MODE_FIRST) {
    rep->targets = job->targets;
    rep->tlens = job->target_lens;
    rep->tlen = job->target_len;
    rep->stride = job->target_stride;
    rep->done.assign(job->n_targets, 0);
    opts.rep = rep;
  }
  {
    const int r = run_pipeline(ctx, T, opts, stats, &nr);
    // copies still reading the caller's targets end before it gets them back
    if (opts.up_chunks) cudaStreamSynchronize(ctx->copy_stream);
    CKR(r);
  }
  if (stats) stats->launches = ctx->launches;
  *n_rules = nr;
  if (nr > cap)
    return fail(ctx, Z80B_ECAPACITY, "%llu rules, capacity %llu", (unsigned long long)nr, (unsigned long long)cap);
  if (nr && !out) return fail(ctx, Z80B_EINVAL, "null output");
  const DevRule* dr = nullptr;
  CKR(rules_to_host(ctx, nr, &dr));
  to_rules(ctx, dr, nr, job->targets, job->target_lens, job->target_len, job->target_stride, job->mode, 0, out);
  return Z80B_OK;
}

int z80b_search(z80b_ctx* ctx, const z80b_job* job, z80b_rule* out, uint64_t cap, uint64_t* n_rules,
                z80b_stats* stats) {
  return search_impl(ctx, job, out, cap, n_rules, stats, nullptr);
}

int z80b_search_cb(z80b_ctx* ctx, const z80b_job* job, z80b_rule* out, uint64_t cap, uint64_t* n_rules,
                   z80b_stats* stats, z80b_rule_cb cb, void* user) {
  if (!cb) return search_impl(ctx, job, out, cap, n_rules, stats, nullptr);
  if (job && (job->mode != Z80B_MODE_FIRST || job->path != Z80B_PATH_BATCHED))
    return fail(ctx, Z80B_EINVAL, "per-target answers need the batched first-found path");
  Reporter rep;
  rep.cb = cb;
  rep.user = user;
  return search_impl(ctx, job, out, cap, n_rules, stats, &rep);
}


int z80b_mul_pool(int pool, int* n_ops, int* max_len, const char** names, int* tstates, int cap) {
  if (pool < 0 || pool >= mul::kNumPools) return Z80B_EINVAL;
  const mul::PoolInfo& pi = mul::pool_info(pool);
  if (n_ops) *n_ops = pi.n;
  if (max_len) *max_len = pi.max_len;
  for (int i = 0; i < pi.n && i < cap; i++) {
    if (names) names[i] = pi.names[i];
    if (tstates) tstates[i] = pi.tstates[i];
  }
  return Z80B_OK;
}

int z80b_mul_search(z80b_ctx* ctx, int pool, uint8_t init_b, uint8_t init_c, uint8_t init_f, int min_len,
                    int max_len, const int32_t* ks, uint32_t n_k, z80b_mul_result* out, z80b_mul_stats* stats) {
  if (!ctx) return Z80B_EINVAL;
  if (pool < 0 || pool >= mul::kNumPools) return fail(ctx, Z80B_EINVAL, "unknown pool %d", pool);
  const mul::PoolInfo& pi = mul::pool_info(pool);
  if (min_len < 1 || max_len < min_len || max_len > pi.max_len)
    return fail(ctx, Z80B_EINVAL, "lengths %d..%d outside 1..%d", min_len, max_len, pi.max_len);
  std::vector<int> kl;
  if (ks) {
    for (uint32_t i = 0; i < n_k; i++) {
      if (ks[i] < 2 || ks[i] > 255) return fail(ctx, Z80B_EINVAL, "constant %d outside 2..255", ks[i]);
      kl.push_back(ks[i]);
    }
  } else {
    for (int k = 2; k <= 255; k++) kl.push_back(k);
  }
  if (!kl.empty() && !out) return fail(ctx, Z80B_EINVAL, "null output");
  cudaSetDevice(ctx->device);
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
  CK(ctx->mul_best.ensure(256 * sizeof(unsigned long long)));
  CK(ctx->mul_stats.ensure(sizeof(mul::LenStats)));
  mul::SearchArgs a{};
  a.pool = pool;
  a.b = init_b;
  a.c = init_c;
  a.f = init_f;
  a.min_len = min_len;
  a.max_len = max_len;
  for (int k : kl) a.want[k >> 5] |= 1u << (k & 31);
  for (size_t i = 0; i < kl.size(); i++) {
    std::memset(&out[i], 0, sizeof out[i]);
    out[i].k = kl[i];
  }
  z80b_mul_stats st{};
  int found_len[256] = {};
  unsigned long long found_key[256] = {};
  double nl = 1;
  for (int i = 0; i < min_len - 1; i++) nl *= pi.n;
  for (int len = min_len; len <= max_len; len++) {
    nl *= pi.n;
    bool any = false;
    for (int w = 0; w < 8; w++) any = any || a.want[w];
    if (!any) break;
    CK(cudaMemsetAsync(ctx->mul_best.p, 0xFF, 256 * sizeof(unsigned long long), ctx->stream));
    CK(cudaMemsetAsync(ctx->mul_stats.p, 0, sizeof(mul::LenStats), ctx->stream));
    Timer tm{ctx, 0, 1};
    tm.start();
    cudaError_t e = mul::launch_length(a, len, ctx->mul_best.as<unsigned long long>(),
                                       ctx->mul_stats.as<mul::LenStats>(), sms, ctx->stream);
    if (e != cudaSuccess) return fail(ctx, Z80B_ECUDA, "mulopt length %d launch: %s", len, cudaGetErrorString(e));
    tm.stop();
    st.launches++;
    unsigned long long best[256];
    mul::LenStats ls{};
    CK(cudaMemcpyAsync(best, ctx->mul_best.p, sizeof best, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(&ls, ctx->mul_stats.p, sizeof ls, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    st.device_ms += tm.ms();
    st.lengths++;
    st.sequences += (uint64_t)nl;
    st.filter_nodes += ls.filter_nodes;
    st.full_checks += ls.full_checks;
    st.full_pass += ls.full_pass;
    for (int k = 2; k < 256; k++) {
      if (!((a.want[k >> 5] >> (k & 31)) & 1u)) continue;
      st.per_k_sequences += (uint64_t)nl;
      if (best[k] != mul::kNoKey) {
        found_len[k] = len;
        found_key[k] = best[k];
        a.want[k >> 5] &= ~(1u << (k & 31));
      }
    }
    trace("mulopt pool %d length %d: %.3f ms, %llu nodes filtered, %llu full checks", pool, len, st.device_ms,
          (unsigned long long)ls.filter_nodes, (unsigned long long)ls.full_checks);
  }
  for (size_t i = 0; i < kl.size(); i++) {
    const int k = kl[i];
    if (!found_len[k]) continue;
    z80b_mul_result& r = out[i];
    r.found = 1;
    r.length = found_len[k];
    r.tstates = int32_t(found_key[k] >> mul::kKeyShift);
    r.index = found_key[k] & ((1ull << mul::kKeyShift) - 1);
    unsigned long long v = r.index;
    for (int j = r.length - 1; j >= 0; j--) {
      r.ops[j] = uint8_t(v % unsigned(pi.n));
      v /= unsigned(pi.n);
    }
  }
  if (stats) *stats = st;
  return Z80B_OK;
}

}  // extern "C"

namespace z80b {

uint64_t target_frontier_bytes(const uint32_t* seq, int len, int max_cand, bool masked) {
  // unpruned 8-bit candidates per target byte size (the QuickCheck units of
  // one pass), computed once
  static const std::vector<uint32_t> elig_lt = [] {
    std::vector<uint32_t> e(16, 0);
    for (uint32_t w : pool8()) {
      const int b = op_table()[insn_op(w)].size;
      if (should_prune(&w, 1)) continue;
      for (int t = b + 1; t < 16; t++) e[size_t(t)]++;
    }
    return e;
  }();
  const int tb = std::min(seq_bytes(seq, len), 15);
  const uint64_t passes = masked ? 2 : 1;
  uint64_t b = 4ull * 4 + 4 + 3;                          // target words, length, dead flags and registers
  b += 4ull * 4 + sizeof(TargetMeta);                      // cnt_f, cnt_m, cnt_all, base, meta
  b += 4ull * kQCSlots;                                    // survivors the count pass keeps
  b += passes * uint64_t(elig_lt[size_t(tb)]) * (4 + 2);   // survivor indices and flag differences
  b += 8 + 8 + 4 + 2;                                      // next, win, windiff, spec
  b += 128ull * (sizeof(PairRec) + 4 + 8 * 6 + 4 + 1);     // pair slots of the windows (cap 128 per target)
  if (max_cand >= 2)
    b += 8 + 8 + 4 + 8 + 8 + 2 + uint64_t(kSlots2) * 2 * (4 + 2);  // length-2 lanes and survivor slots
  return b;
}

}  // namespace z80b
