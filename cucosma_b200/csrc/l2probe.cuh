// l2probe.cuh -- hardware-counter reading of a piece of GPU work (CUPTI
// range profiler, loaded on demand; see l2probe.cu).
#pragma once
#include <cuda_runtime.h>

#include <functional>

namespace cucosma {

struct CounterReading {
  double l2_hit_pct;        // lts__t_sector_hit_rate.pct, -1 when not measured
  double dram_read_bytes;   // dram__bytes_read.sum
  double dram_write_bytes;  // dram__bytes_write.sum
  int passes;               // times run() was called (one per counter pass)
  const char* why;          // reason when the reading is unavailable
};

// Profiles the work that run() enqueues on stream st (run() is called once
// per counter pass and must be repeatable; it returns false on failure).
// Returns false, with out->why set and out->l2_hit_pct = -1, when CUPTI or
// the counters are unavailable.  Serialised within the process.
bool measure_counters(const std::function<bool()>& run, cudaStream_t st, CounterReading* out);

}  // namespace cucosma
