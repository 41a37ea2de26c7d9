// tune.cu -- on-device autotuner and tuning cache.
//
// Replaces the reference's ScheduleGenerator (ScheduleGenerator/
// ScheduleGeneratorv4.h:13-391), which brute-forced tile sizes, LOAD_K and
// split-K on the host and ranked them by a communication-volume model; the
// thesis found that model a poor predictor and named occupancy and L2 hit rate
// as what matters (thesis p.41-42).  Here the candidates -- split-K factor,
// raster band / block-index remap width, and tile variant -- are run on the
// device on the caller's buffers and ranked by measured time.  Each result
// records the chosen kernel's occupancy (CUDA occupancy API) and a model of
// the L2 reuse its raster achieves.  The winner is stored in a process-wide
// cache keyed by (SM count, dtype, precision, slices, m, n, k); cucosma_gemm
// consults it whenever the descriptor leaves split_k, swizzle and tile at 0.
// The cache persists as a text file (cucosma_tune_cache_save / _load; loaded
// automatically from $CUCOSMA_TUNE_CACHE on first use; CUCOSMA_TUNE=off
// disables lookups).
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

namespace cucosma {
namespace {

using Key = std::tuple<int, int, int, int, int64_t, int64_t, int64_t>;  // sms dtype precision slices m n k
struct Val {
  int split_k, swizzle, tile;
  double ms;
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
  char tag[16];
  int sms, dt, pr, sl, sk, sw, ti;
  long long m, n, k;
  double ms;
  while (std::fscanf(f, "%15s %d %d %d %d %lld %lld %lld %d %d %d %lf", tag, &sms, &dt, &pr, &sl, &m, &n, &k, &sk, &sw,
                     &ti, &ms) == 12) {
    if (std::strcmp(tag, "v1") != 0) continue;
    g_cache[Key(sms, dt, pr, sl, m, n, k)] = Val{sk, sw, ti, ms};
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

// Fraction of operand-tile loads a wave can serve from L2 under a banded
// raster of height `band`: a wave of `ctas` tiles touches `band` row tiles of A
// and ctas/band column tiles of B per k-block.  A model, not a measurement.
double l2_reuse_model(int tiles_m, int tiles_n, int ctas, int band, double a_tile, double b_tile) {
  const int wave = std::max(1, std::min(ctas, tiles_m * tiles_n));
  const int rows = std::max(1, std::min({band, tiles_m, wave}));
  const int cols = std::max(1, std::min(tiles_n, (wave + rows - 1) / rows));
  const double loaded = (double)wave * (a_tile + b_tile);
  const double distinct = rows * a_tile + cols * b_tile;
  return loaded > 0 ? std::max(0.0, 1.0 - distinct / loaded) : 0.0;
}

}  // namespace

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
    if (d->precision == CUCOSMA_PRECISION_BF16X3) tiles = {0, 1, 2};
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
  {
    std::lock_guard<std::mutex> lk(g_mu);
    load_env_locked();
    g_cache[key_of(d, di->sms)] = Val{pick.sk, pick.sw, pick.ti, best};
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
    const int es = d->precision == CUCOSMA_PRECISION_NATIVE ? (d->dtype == CUCOSMA_R_32F ? 4 : 8)
                   : d->precision == CUCOSMA_PRECISION_OZAKI ? pk.slices
                                                             : 2 * pk.slices;
    const int64_t tiles_m = (d->m + pk.tile_m - 1) / pk.tile_m, tiles_n = (d->n + pk.tile_n - 1) / pk.tile_n;
    out->l2_reuse_model = l2_reuse_model((int)tiles_m, (int)tiles_n, di->sms * std::max(1, out->occupancy),
                                         std::max(1, pk.band), (double)pk.tile_m * es, (double)pk.tile_n * es);
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
    std::fprintf(f, "v1 %d %d %d %d %lld %lld %lld %d %d %d %.6f\n", std::get<0>(k), std::get<1>(k), std::get<2>(k),
                 std::get<3>(k), (long long)std::get<4>(k), (long long)std::get<5>(k), (long long)std::get<6>(k),
                 kv.second.split_k, kv.second.swizzle, kv.second.tile, kv.second.ms);
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
