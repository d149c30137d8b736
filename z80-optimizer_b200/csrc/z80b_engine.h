// z80b_engine.h -- facts about the search engine's device buffers that host
// code outside the engine needs (the serving loop's admission).
#pragma once
#include <cstdint>

namespace z80b {

// Device bytes that one target of a first-found job holds while the job
// runs: its share of every per-target buffer of the pipeline (z80b_engine.cu
// run_pipeline), its share of the ExhaustiveCheck pair slots, and its
// QuickCheck survivor records at their upper bound (every unpruned
// candidate shorter than the target, in each pass it runs: the masked pass
// runs when flags or registers are dead), plus the length-2 lanes and
// survivor slots when max_cand is 2.
uint64_t target_frontier_bytes(const uint32_t* seq, int len, int max_cand, bool masked);

}  // namespace z80b
