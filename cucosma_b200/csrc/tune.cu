// tune.cu -- on-device autotuner and tuning cache.
//
// Replaces the reference's ScheduleGenerator (ScheduleGenerator/
// ScheduleGeneratorv4.h:13-391), which brute-forced tile sizes, LOAD_K and
// split-K on the host and ranked them by a communication-volume model; the
// thesis found that model a poor predictor and named occupancy and L2 hit rate
// as what matters (thesis p.41-42).  Here the candidates -- split-K factor,
// raster band / block-index remap width, and tile variant (including the
// 256-row CTA-pair tiles of the tensor-core paths) -- are run on the device on
// the caller's buffers and ranked by measured time.  Each result records the
// chosen kernel's occupancy (CUDA occupancy API) and the L2 hit rate and DRAM
// bytes its tiling and raster achieve, read from the hardware counters with
// the CUPTI range profiler (l2probe.cu; -1 when profiling is unavailable).
// The winner is stored in a process-wide cache keyed by (SM count, dtype,
// precision, slices, m, n, k); cucosma_gemm consults it whenever the
// descriptor leaves split_k, swizzle and tile at 0, and the grouped planner
// consults the grouped entries (cucosma_tune_grouped).  The cache persists as
// a text file (cucosma_tune_cache_save / _load; loaded automatically from
// $CUCOSMA_TUNE_CACHE on first use; CUCOSMA_TUNE=off disables lookups;
// CUCOSMA_TUNE_COUNTERS=off skips the counter reading).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "../../include/cucosma.h"
#include "api_internal.cuh"
#include "simt_gemm.cuh"
#include "skinny.cuh"
#include "l2probe.cuh"

namespace cucosma {
namespace {

using Key = std::tuple<int, int, int, int, int64_t, int64_t, int64_t>;  // sms dtype precision slices m n k
struct Val {
  int split_k, swizzle, tile;
  double ms;
  double l2_hit;      // measured L2 hit rate (percent), -1 when not measured
  double dram_bytes;  // measured DRAM bytes read + written per call, -1 when not measured
};

std::mutex g_mu;
std::map<Key, Val> g_cache;
bool g_env_loaded = false;

Key key_of(const cucosma_gemm_desc* d, int sms) {
  return Key(sms, d->dtype, d->precision, d->slices, d->m, d->n, d->k);
}

bool lookups_enabled() {
  const char* t = std::getenv("CUCOSMA_TUNE");
  return !(t && std::strcmp(t, "off") == 0);
}

cucosma_status load_locked(const char* path) {
  FILE* f = std::fopen(path, "r");
  if (!f) return CUCOSMA_STATUS_INVALID_VALUE;
  // Lines: "v1 sms dtype precision slices m n k split_k swizzle tile ms" or
  // "v2 ... ms l2_hit dram_bytes" (v2 adds the counter readings).
  char line[512];
  while (std::fgets(line, sizeof line, f)) {
    char tag[16];
    int sms, dt, pr, sl, sk, sw, ti;
    long long m, n, k;
    double ms, l2 = -1.0, dram = -1.0;
    const int got = std::sscanf(line, "%15s %d %d %d %d %lld %lld %lld %d %d %d %lf %lf %lf", tag, &sms, &dt, &pr, &sl,
                                &m, &n, &k, &sk, &sw, &ti, &ms, &l2, &dram);
    if (got < 12) continue;
    if (std::strcmp(tag, "v1") == 0) {
      l2 = dram = -1.0;
    } else if (std::strcmp(tag, "v2") != 0 || got != 14) {
      continue;
    }
    g_cache[Key(sms, dt, pr, sl, m, n, k)] = Val{sk, sw, ti, ms, l2, dram};
  }
  std::fclose(f);
  return CUCOSMA_STATUS_SUCCESS;
}

void load_env_locked() {
  if (g_env_loaded) return;
  g_env_loaded = true;
  const char* p = std::getenv("CUCOSMA_TUNE_CACHE");
  if (p && *p) load_locked(p);
}

double elapsed_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}


}  // namespace

// Grouped entries: the key's m is -count and n a 62-bit FNV-1a hash of the
// problems' (m, n, k) in order (k = -1 marks the entry), so a batch is found
// again by its shape mix.
static Key grouped_key(const cucosma_gemm_desc* d, const cucosma_gemm_problem* pr, int count, int sms) {
  uint64_t h = 1469598103934665603ull;
  auto mix = [&](int64_t v) {
    for (int b = 0; b < 8; ++b) {
      h ^= (uint64_t)((v >> (8 * b)) & 0xff);
      h *= 1099511628211ull;
    }
  };
  mix(count);
  for (int i = 0; i < count; ++i) {
    mix(pr[i].m);
    mix(pr[i].n);
    mix(pr[i].k);
  }
  return Key(sms, d->dtype, d->precision, d->slices, -(int64_t)count, (int64_t)(h >> 2), -1);
}

int grouped_tuned_tile(const cucosma_gemm_desc* d, const cucosma_gemm_problem* pr, int count, const DeviceInfo* di) {
  if (!d || !pr || count <= 0 || !di || !lookups_enabled()) return 0;
  std::lock_guard<std::mutex> lk(g_mu);
  load_env_locked();
  auto it = g_cache.find(grouped_key(d, pr, count, di->sms));
  return it == g_cache.end() ? 0 : it->second.tile;
}

const cucosma_gemm_desc* apply_tuning(const cucosma_gemm_desc* d, cucosma_gemm_desc* tmp, const DeviceInfo* di) {
  if (!d || !di || d->split_k || d->swizzle || d->tile || !lookups_enabled()) return d;
  std::lock_guard<std::mutex> lk(g_mu);
  load_env_locked();
  auto it = g_cache.find(key_of(d, di->sms));
  if (it == g_cache.end()) return d;
  *tmp = *d;
  tmp->split_k = it->second.split_k;
  tmp->swizzle = it->second.swizzle;
  tmp->tile = it->second.tile;
  return tmp;
}

}  // namespace cucosma

using namespace cucosma;

extern "C" cucosma_status cucosma_tune(const cucosma_gemm_desc* d, const void* A, const void* B, void* C,
                                       void* workspace, size_t workspace_bytes, int max_candidates,
                                       cucosma_tune_result* out, void* stream) {
  cucosma_status s = validate(d, A, B, C);
  if (s != CUCOSMA_STATUS_SUCCESS) return s;
  if (d->m == 0 || d->n == 0 || d->k == 0) return CUCOSMA_STATUS_INVALID_VALUE;
  const DeviceInfo* di = device_info();
  if (!di) return CUCOSMA_STATUS_LAUNCH_FAILED;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cucosma_gemm_desc base = *d;
  base.split_k = base.swizzle = base.tile = 0;

  // Candidate set.
  cucosma_plan_info pi;
  if ((s = cucosma_gemm_get_plan(&base, &pi)) != CUCOSMA_STATUS_SUCCESS) return s;
  const int64_t kblocks = (d->k + pi.tile_k - 1) / pi.tile_k;
  std::vector<int> splits = {pi.splits};
  for (int sk : {1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64})
    if (sk != pi.splits && sk <= std::max<int64_t>(1, kblocks / 4)) splits.push_back(sk);
  std::vector<int> bands;
  std::vector<int> tiles = {0};
  if (d->precision == CUCOSMA_PRECISION_NATIVE) {
    bands = {1, 2, 4, 8};
    // FP32 tile kernel: 128-row (tile 1) and 64-row (tile 2) CTA tiles
    if (d->dtype == CUCOSMA_R_32F) tiles = {1, 2};
    // a skinny shape: its kernel (tile 0, no block remap) against the tile kernel (tile 1)
    if (plan_skinny(d->m, d->n, d->k, d->dtype == CUCOSMA_R_32F ? 4 : 8, 0, 0, di->sms).kind) {
      bands = {1};
      tiles = {0, 1};
    }
  } else {
    bands = {8, 4, 16};
    // tensor-core tiles: BF16x3 128x128, 128x256, 256x256 (CTA pair);
    // BF16x6 128x128, 256x128 (pair), 256x256 (pair); with operands of 32 MB
    // or more also the fused-split pair (BF16x3 tile 5, BF16x6 tile 4); Ozaki
    // one tile per slice count
    const bool big = ((double)d->m * d->k + (double)d->k * d->n) * 4.0 >= 32.0 * (1 << 20) && d->flags == 0;
    if (d->precision == CUCOSMA_PRECISION_BF16X3) tiles = big ? std::vector<int>{2, 3, 4, 5} : std::vector<int>{2, 3, 4};
    if (d->precision == CUCOSMA_PRECISION_BF16X6) tiles = big ? std::vector<int>{1, 2, 3, 4} : std::vector<int>{1, 2, 3};
  }
  struct Cand {
    int sk, sw, ti;
  };
  std::vector<Cand> cands;
  for (int ti : tiles)
    for (int sw : bands)
      for (int sk : splits) cands.push_back({sk, sw, ti});
  if (max_candidates > 0 && (int)cands.size() > max_candidates) cands.resize(max_candidates);

  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return CUCOSMA_STATUS_LAUNCH_FAILED;
  double best = 1e300;
  Cand pick{0, 0, 0};
  int measured = 0;
  for (const Cand& c : cands) {
    cucosma_gemm_desc t = base;
    t.split_k = c.sk;
    t.swizzle = c.sw;
    t.tile = c.ti;
    size_t need = 0;
    if (cucosma_gemm_workspace_size(&t, &need) != CUCOSMA_STATUS_SUCCESS || need > workspace_bytes) continue;
    if (gemm(&t, A, B, C, workspace, workspace_bytes, st) != CUCOSMA_STATUS_SUCCESS) continue;  // warm-up
    double tmin = 1e300;
    for (int r = 0; r < 3; ++r) {
      cudaEventRecord(e0, st);
      gemm(&t, A, B, C, workspace, workspace_bytes, st);
      cudaEventRecord(e1, st);
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return CUCOSMA_STATUS_LAUNCH_FAILED;
      }
      tmin = std::min(tmin, elapsed_ms(e0, e1));
    }
    ++measured;
    if (tmin < best) {
      best = tmin;
      pick = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (measured == 0) return CUCOSMA_STATUS_WORKSPACE_TOO_SMALL;
  // Hardware counters of the chosen configuration (one profiled call per
  // counter pass).
  CounterReading cr{};
  cr.l2_hit_pct = -1.0;
  {
    const char* e = std::getenv("CUCOSMA_TUNE_COUNTERS");
    if (!(e && std::strcmp(e, "off") == 0)) {
      cucosma_gemm_desc t = base;
      t.split_k = pick.sk;
      t.swizzle = pick.sw;
      t.tile = pick.ti;
      measure_counters([&] { return gemm(&t, A, B, C, workspace, workspace_bytes, st) == CUCOSMA_STATUS_SUCCESS; }, st,
                       &cr);
    } else {
      cr.why = "disabled by CUCOSMA_TUNE_COUNTERS=off";
    }
  }
  const double dram = cr.l2_hit_pct >= 0.0 ? cr.dram_read_bytes + cr.dram_write_bytes : -1.0;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    load_env_locked();
    g_cache[key_of(d, di->sms)] = Val{pick.sk, pick.sw, pick.ti, best, cr.l2_hit_pct, dram};
  }
  if (out) {
    std::memset(out, 0, sizeof(*out));
    out->split_k = pick.sk;
    out->swizzle = pick.sw;
    out->tile = pick.ti;
    out->ms = best;
    out->tflops = 2.0 * (double)d->m * (double)d->n * (double)d->k / (best * 1e-3) / 1e12;
    out->candidates = measured;
    cucosma_gemm_desc t = base;
    t.split_k = pick.sk;
    t.swizzle = pick.sw;
    t.tile = pick.ti;
    cucosma_plan_info pk;
    cucosma_gemm_get_plan(&t, &pk);
    if (d->precision == CUCOSMA_PRECISION_NATIVE)
      out->occupancy = d->dtype == CUCOSMA_R_32F ? simt::occupancy<float>(pk.tile_m == 64 ? 64 : simt::BM)
                                                 : simt::occupancy<double>();
    else
      out->occupancy = 1;  // persistent kernel, one CTA per SM by construction
    out->l2_hit_rate = cr.l2_hit_pct;
    out->dram_bytes = dram;
    out->counter_passes = cr.passes;
  }
  return CUCOSMA_STATUS_SUCCESS;
}

extern "C" cucosma_status cucosma_tune_grouped(const cucosma_gemm_desc* d, const cucosma_gemm_problem* problems,
                                               int count, void* workspace, size_t workspace_bytes,
                                               cucosma_tune_result* out, void* stream) {
  if (!d || !problems || count <= 0) return CUCOSMA_STATUS_INVALID_VALUE;
  const DeviceInfo* di = device_info();
  if (!di) return CUCOSMA_STATUS_LAUNCH_FAILED;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // Candidate tiles of the grouped launch (see cucosma_grouped_plan_create).
  std::vector<int> tiles;
  if (d->precision == CUCOSMA_PRECISION_BF16X3) tiles = {1, 2, 3};
  else if (d->precision == CUCOSMA_PRECISION_BF16X6) tiles = {1, 2};
  else tiles = {1};
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return CUCOSMA_STATUS_LAUNCH_FAILED;
  double best = 1e300;
  int pick = 0, measured = 0;
  cucosma_status s = CUCOSMA_STATUS_SUCCESS;
  for (int ti : tiles) {
    cucosma_gemm_desc t = *d;
    t.tile = ti;
    cucosma_grouped_plan plan = nullptr;
    if (cucosma_grouped_plan_create(&t, problems, count, workspace, workspace_bytes, &plan) != CUCOSMA_STATUS_SUCCESS)
      continue;
    double tmin = 1e300;
    bool ok = cucosma_gemm_grouped(plan, stream) == CUCOSMA_STATUS_SUCCESS;  // warm-up
    for (int r = 0; ok && r < 3; ++r) {
      cudaEventRecord(e0, st);
      ok = cucosma_gemm_grouped(plan, stream) == CUCOSMA_STATUS_SUCCESS;
      cudaEventRecord(e1, st);
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        ok = false;
        s = CUCOSMA_STATUS_LAUNCH_FAILED;
      }
      tmin = std::min(tmin, elapsed_ms(e0, e1));
    }
    cucosma_grouped_plan_destroy(plan);
    if (!ok) continue;
    ++measured;
    if (tmin < best) {
      best = tmin;
      pick = ti;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (s != CUCOSMA_STATUS_SUCCESS) return s;
  if (measured == 0) return CUCOSMA_STATUS_WORKSPACE_TOO_SMALL;
  CounterReading cr{};
  cr.l2_hit_pct = -1.0;
  const char* env = std::getenv("CUCOSMA_TUNE_COUNTERS");
  if (!(env && std::strcmp(env, "off") == 0)) {
    cucosma_gemm_desc t = *d;
    t.tile = pick;
    cucosma_grouped_plan plan = nullptr;
    if (cucosma_grouped_plan_create(&t, problems, count, workspace, workspace_bytes, &plan) == CUCOSMA_STATUS_SUCCESS) {
      measure_counters([&] { return cucosma_gemm_grouped(plan, stream) == CUCOSMA_STATUS_SUCCESS; }, st, &cr);
      cucosma_grouped_plan_destroy(plan);
    }
  }
  const double dram = cr.l2_hit_pct >= 0.0 ? cr.dram_read_bytes + cr.dram_write_bytes : -1.0;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    load_env_locked();
    g_cache[grouped_key(d, problems, count, di->sms)] = Val{0, 0, pick, best, cr.l2_hit_pct, dram};
  }
  if (out) {
    std::memset(out, 0, sizeof(*out));
    out->tile = pick;
    out->candidates = measured;
    out->occupancy = 1;
    out->ms = best;
    double flop = 0.0;
    for (int i = 0; i < count; ++i) flop += 2.0 * (double)problems[i].m * (double)problems[i].n * (double)problems[i].k;
    out->tflops = flop / (best * 1e-3) / 1e12;
    out->l2_hit_rate = cr.l2_hit_pct;
    out->dram_bytes = dram;
    out->counter_passes = cr.passes;
  }
  return CUCOSMA_STATUS_SUCCESS;
}

extern "C" cucosma_status cucosma_tune_cache_save(const char* path) {
  if (!path) return CUCOSMA_STATUS_INVALID_VALUE;
  std::lock_guard<std::mutex> lk(g_mu);
  FILE* f = std::fopen(path, "w");
  if (!f) return CUCOSMA_STATUS_INVALID_VALUE;
  for (const auto& kv : g_cache) {
    const Key& k = kv.first;
    std::fprintf(f, "v2 %d %d %d %d %lld %lld %lld %d %d %d %.6f %.3f %.0f\n", std::get<0>(k), std::get<1>(k),
                 std::get<2>(k), std::get<3>(k), (long long)std::get<4>(k), (long long)std::get<5>(k),
                 (long long)std::get<6>(k), kv.second.split_k, kv.second.swizzle, kv.second.tile, kv.second.ms,
                 kv.second.l2_hit, kv.second.dram_bytes);
  }
  std::fclose(f);
  return CUCOSMA_STATUS_SUCCESS;
}

extern "C" cucosma_status cucosma_tune_cache_load(const char* path) {
  if (!path) return CUCOSMA_STATUS_INVALID_VALUE;
  std::lock_guard<std::mutex> lk(g_mu);
  return load_locked(path);
}

extern "C" cucosma_status cucosma_tune_cache_clear(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_cache.clear();
  g_env_loaded = true;  // an explicit clear also drops the environment file
  return CUCOSMA_STATUS_SUCCESS;
}

extern "C" int cucosma_tune_cache_size(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  return (int)g_cache.size();
}
