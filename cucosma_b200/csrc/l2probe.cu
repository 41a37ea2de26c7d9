// l2probe.cu -- on-device L2 hit rate and DRAM traffic of a piece of GPU
// work, measured with the CUPTI range profiler.
//
// The autotuner (tune.cu) ranks its candidates by measured time; this adds
// the quantity the reference's schedule study found to matter beside
// occupancy (thesis p.41-42): the L2 hit rate the chosen tiling and raster
// actually achieve, read from the hardware counters (lts__t_sector_hit_rate,
// dram__bytes_read / _write) instead of modelled.  CUPTI is loaded with
// dlopen when first needed, so the library runs without it; when it is
// missing, when profiling is not permitted, or when another profiler (such
// as Nsight Compute) holds the counters, the measurement reports itself
// unavailable and the tuner records -1.
//
// Protocol (CUPTI range profiler, user range, user replay): one range around
// the work, replayed once per counter pass by calling run() again -- the work
// must therefore be repeatable (the tuner's candidate GEMM on scratch
// output is).
#include <dlfcn.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include <cupti_profiler_host.h>
#include <cupti_profiler_target.h>
#include <cupti_range_profiler.h>
#include <cupti_target.h>

#include "api_internal.cuh"
#include "l2probe.cuh"

namespace cucosma {
namespace {

struct Cupti {
  bool ok = false;
  const char* why = "not loaded";
  CUptiResult (*init)(CUpti_Profiler_Initialize_Params*) = nullptr;
  CUptiResult (*chip)(CUpti_Device_GetChipName_Params*) = nullptr;
  CUptiResult (*avail)(CUpti_Profiler_GetCounterAvailability_Params*) = nullptr;
  CUptiResult (*host_init)(CUpti_Profiler_Host_Initialize_Params*) = nullptr;
  CUptiResult (*host_deinit)(CUpti_Profiler_Host_Deinitialize_Params*) = nullptr;
  CUptiResult (*add_metrics)(CUpti_Profiler_Host_ConfigAddMetrics_Params*) = nullptr;
  CUptiResult (*cfg_size)(CUpti_Profiler_Host_GetConfigImageSize_Params*) = nullptr;
  CUptiResult (*cfg_image)(CUpti_Profiler_Host_GetConfigImage_Params*) = nullptr;
  CUptiResult (*evaluate)(CUpti_Profiler_Host_EvaluateToGpuValues_Params*) = nullptr;
  CUptiResult (*rp_enable)(CUpti_RangeProfiler_Enable_Params*) = nullptr;
  CUptiResult (*rp_disable)(CUpti_RangeProfiler_Disable_Params*) = nullptr;
  CUptiResult (*rp_data_size)(CUpti_RangeProfiler_GetCounterDataSize_Params*) = nullptr;
  CUptiResult (*rp_data_init)(CUpti_RangeProfiler_CounterDataImage_Initialize_Params*) = nullptr;
  CUptiResult (*rp_set_config)(CUpti_RangeProfiler_SetConfig_Params*) = nullptr;
  CUptiResult (*rp_start)(CUpti_RangeProfiler_Start_Params*) = nullptr;
  CUptiResult (*rp_stop)(CUpti_RangeProfiler_Stop_Params*) = nullptr;
  CUptiResult (*rp_push)(CUpti_RangeProfiler_PushRange_Params*) = nullptr;
  CUptiResult (*rp_pop)(CUpti_RangeProfiler_PopRange_Params*) = nullptr;
  CUptiResult (*rp_decode)(CUpti_RangeProfiler_DecodeData_Params*) = nullptr;
};

template <class F>
bool sym(void* h, const char* name, F& f) {
  f = reinterpret_cast<F>(dlsym(h, name));
  return f != nullptr;
}

Cupti& cupti() {
  static Cupti c;
  static std::once_flag once;
  std::call_once(once, [] {
    void* h = nullptr;
    for (const char* name : {"libcupti.so.12", "libcupti.so", "/usr/local/cuda/extras/CUPTI/lib64/libcupti.so",
                             "/usr/local/cuda/lib64/libcupti.so"}) {
      h = dlopen(name, RTLD_NOW | RTLD_LOCAL);
      if (h) break;
    }
    if (!h) {
      c.why = "libcupti not found";
      return;
    }
    const bool all = sym(h, "cuptiProfilerInitialize", c.init) && sym(h, "cuptiDeviceGetChipName", c.chip) &&
                     sym(h, "cuptiProfilerGetCounterAvailability", c.avail) &&
                     sym(h, "cuptiProfilerHostInitialize", c.host_init) &&
                     sym(h, "cuptiProfilerHostDeinitialize", c.host_deinit) &&
                     sym(h, "cuptiProfilerHostConfigAddMetrics", c.add_metrics) &&
                     sym(h, "cuptiProfilerHostGetConfigImageSize", c.cfg_size) &&
                     sym(h, "cuptiProfilerHostGetConfigImage", c.cfg_image) &&
                     sym(h, "cuptiProfilerHostEvaluateToGpuValues", c.evaluate) &&
                     sym(h, "cuptiRangeProfilerEnable", c.rp_enable) &&
                     sym(h, "cuptiRangeProfilerDisable", c.rp_disable) &&
                     sym(h, "cuptiRangeProfilerGetCounterDataSize", c.rp_data_size) &&
                     sym(h, "cuptiRangeProfilerCounterDataImageInitialize", c.rp_data_init) &&
                     sym(h, "cuptiRangeProfilerSetConfig", c.rp_set_config) &&
                     sym(h, "cuptiRangeProfilerStart", c.rp_start) && sym(h, "cuptiRangeProfilerStop", c.rp_stop) &&
                     sym(h, "cuptiRangeProfilerPushRange", c.rp_push) &&
                     sym(h, "cuptiRangeProfilerPopRange", c.rp_pop) &&
                     sym(h, "cuptiRangeProfilerDecodeData", c.rp_decode);
    if (!all) {
      c.why = "libcupti lacks the range profiler";
      return;
    }
    CUpti_Profiler_Initialize_Params ip{};
    ip.structSize = CUpti_Profiler_Initialize_Params_STRUCT_SIZE;
    if (c.init(&ip) != CUPTI_SUCCESS) {
      c.why = "cuptiProfilerInitialize failed";
      return;
    }
    c.ok = true;
    c.why = "";
  });
  return c;
}

using GetCtxFn = CUresult (*)(CUcontext*);

CUcontext current_context() {
  static GetCtxFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<GetCtxFn>(p);
  });
  CUcontext ctx = nullptr;
  if (fn) fn(&ctx);
  return ctx;
}

std::mutex g_probe_mu;  // one profiling session at a time in this process

}  // namespace

bool measure_counters(const std::function<bool()>& run, cudaStream_t st, CounterReading* out) {
  *out = CounterReading{};
  out->l2_hit_pct = -1.0;
  Cupti& c = cupti();
  if (!c.ok) {
    out->why = c.why;
    return false;
  }
  std::lock_guard<std::mutex> lk(g_probe_mu);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaFree(nullptr) != cudaSuccess) {
    out->why = "no current device";
    return false;
  }
  CUcontext ctx = current_context();
  if (!ctx) {
    out->why = "no current context";
    return false;
  }
  static const char* kMetrics[3] = {"lts__t_sector_hit_rate.pct", "dram__bytes_read.sum", "dram__bytes_write.sum"};

  CUpti_Device_GetChipName_Params cp{};
  cp.structSize = CUpti_Device_GetChipName_Params_STRUCT_SIZE;
  cp.deviceIndex = (size_t)dev;
  if (c.chip(&cp) != CUPTI_SUCCESS) {
    out->why = "chip name unavailable";
    return false;
  }
  CUpti_Profiler_GetCounterAvailability_Params ap{};
  ap.structSize = CUpti_Profiler_GetCounterAvailability_Params_STRUCT_SIZE;
  ap.ctx = ctx;
  if (c.avail(&ap) != CUPTI_SUCCESS) {
    out->why = "counters unavailable (profiling not permitted or in use)";
    return false;
  }
  std::vector<uint8_t> avail(ap.counterAvailabilityImageSize);
  ap.pCounterAvailabilityImage = avail.data();
  if (c.avail(&ap) != CUPTI_SUCCESS) {
    out->why = "counters unavailable (profiling not permitted or in use)";
    return false;
  }
  CUpti_Profiler_Host_Initialize_Params hp{};
  hp.structSize = CUpti_Profiler_Host_Initialize_Params_STRUCT_SIZE;
  hp.profilerType = CUPTI_PROFILER_TYPE_RANGE_PROFILER;
  hp.pChipName = cp.pChipName;
  hp.pCounterAvailabilityImage = avail.data();
  if (c.host_init(&hp) != CUPTI_SUCCESS) {
    out->why = "profiler host initialisation failed";
    return false;
  }
  CUpti_Profiler_Host_Object* host = hp.pHostObject;
  auto host_done = [&] {
    CUpti_Profiler_Host_Deinitialize_Params dp{};
    dp.structSize = CUpti_Profiler_Host_Deinitialize_Params_STRUCT_SIZE;
    dp.pHostObject = host;
    c.host_deinit(&dp);
  };
  CUpti_Profiler_Host_ConfigAddMetrics_Params mp{};
  mp.structSize = CUpti_Profiler_Host_ConfigAddMetrics_Params_STRUCT_SIZE;
  mp.pHostObject = host;
  mp.ppMetricNames = kMetrics;
  mp.numMetrics = 3;
  CUpti_Profiler_Host_GetConfigImageSize_Params sp{};
  sp.structSize = CUpti_Profiler_Host_GetConfigImageSize_Params_STRUCT_SIZE;
  sp.pHostObject = host;
  if (c.add_metrics(&mp) != CUPTI_SUCCESS || c.cfg_size(&sp) != CUPTI_SUCCESS) {
    host_done();
    out->why = "metric configuration failed";
    return false;
  }
  std::vector<uint8_t> config(sp.configImageSize);
  CUpti_Profiler_Host_GetConfigImage_Params gp{};
  gp.structSize = CUpti_Profiler_Host_GetConfigImage_Params_STRUCT_SIZE;
  gp.pHostObject = host;
  gp.configImageSize = config.size();
  gp.pConfigImage = config.data();
  if (c.cfg_image(&gp) != CUPTI_SUCCESS) {
    host_done();
    out->why = "metric configuration failed";
    return false;
  }

  CUpti_RangeProfiler_Enable_Params ep{};
  ep.structSize = CUpti_RangeProfiler_Enable_Params_STRUCT_SIZE;
  ep.ctx = ctx;
  if (c.rp_enable(&ep) != CUPTI_SUCCESS) {
    host_done();
    out->why = "range profiler unavailable (profiling not permitted or in use)";
    return false;
  }
  CUpti_RangeProfiler_Object* rp = ep.pRangeProfilerObject;
  bool ok = false;
  std::vector<uint8_t> data;
  do {
    CUpti_RangeProfiler_GetCounterDataSize_Params dsp{};
    dsp.structSize = CUpti_RangeProfiler_GetCounterDataSize_Params_STRUCT_SIZE;
    dsp.pRangeProfilerObject = rp;
    dsp.pMetricNames = kMetrics;
    dsp.numMetrics = 3;
    dsp.maxNumOfRanges = 1;
    dsp.maxNumRangeTreeNodes = 1;
    if (c.rp_data_size(&dsp) != CUPTI_SUCCESS) break;
    data.assign(dsp.counterDataSize, 0);
    CUpti_RangeProfiler_CounterDataImage_Initialize_Params dip{};
    dip.structSize = CUpti_RangeProfiler_CounterDataImage_Initialize_Params_STRUCT_SIZE;
    dip.pRangeProfilerObject = rp;
    dip.counterDataSize = data.size();
    dip.pCounterData = data.data();
    if (c.rp_data_init(&dip) != CUPTI_SUCCESS) break;
    CUpti_RangeProfiler_SetConfig_Params scp{};
    scp.structSize = CUpti_RangeProfiler_SetConfig_Params_STRUCT_SIZE;
    scp.pRangeProfilerObject = rp;
    scp.configSize = config.size();
    scp.pConfig = config.data();
    scp.counterDataImageSize = data.size();
    scp.pCounterDataImage = data.data();
    scp.range = CUPTI_UserRange;
    scp.replayMode = CUPTI_UserReplay;
    scp.maxRangesPerPass = 1;
    scp.numNestingLevels = 1;
    scp.minNestingLevel = 1;
    scp.passIndex = 0;
    scp.targetNestingLevel = 1;
    if (c.rp_set_config(&scp) != CUPTI_SUCCESS) break;
    bool submitted = false, failed = false;
    for (int pass = 0; pass < 16 && !submitted && !failed; ++pass) {
      CUpti_RangeProfiler_Start_Params stp{};
      stp.structSize = CUpti_RangeProfiler_Start_Params_STRUCT_SIZE;
      stp.pRangeProfilerObject = rp;
      CUpti_RangeProfiler_PushRange_Params pup{};
      pup.structSize = CUpti_RangeProfiler_PushRange_Params_STRUCT_SIZE;
      pup.pRangeProfilerObject = rp;
      pup.pRangeName = "work";
      CUpti_RangeProfiler_PopRange_Params pop{};
      pop.structSize = CUpti_RangeProfiler_PopRange_Params_STRUCT_SIZE;
      pop.pRangeProfilerObject = rp;
      CUpti_RangeProfiler_Stop_Params stop{};
      stop.structSize = CUpti_RangeProfiler_Stop_Params_STRUCT_SIZE;
      stop.pRangeProfilerObject = rp;
      if (c.rp_start(&stp) != CUPTI_SUCCESS || c.rp_push(&pup) != CUPTI_SUCCESS) {
        failed = true;
        break;
      }
      const bool ran = run() && cudaStreamSynchronize(st) == cudaSuccess;
      if (c.rp_pop(&pop) != CUPTI_SUCCESS || c.rp_stop(&stop) != CUPTI_SUCCESS || !ran) failed = true;
      submitted = stop.isAllPassSubmitted != 0;
      ++out->passes;
    }
    if (failed || !submitted) break;
    CUpti_RangeProfiler_DecodeData_Params dd{};
    dd.structSize = CUpti_RangeProfiler_DecodeData_Params_STRUCT_SIZE;
    dd.pRangeProfilerObject = rp;
    if (c.rp_decode(&dd) != CUPTI_SUCCESS) break;
    double values[3] = {-1.0, -1.0, -1.0};
    CUpti_Profiler_Host_EvaluateToGpuValues_Params ev{};
    ev.structSize = CUpti_Profiler_Host_EvaluateToGpuValues_Params_STRUCT_SIZE;
    ev.pHostObject = host;
    ev.pCounterDataImage = data.data();
    ev.counterDataImageSize = data.size();
    ev.rangeIndex = 0;
    ev.ppMetricNames = kMetrics;
    ev.numMetrics = 3;
    ev.pMetricValues = values;
    if (c.evaluate(&ev) != CUPTI_SUCCESS) break;
    // the counter ratio can read a few hundredths of a percent above 100
    out->l2_hit_pct = values[0] < 0.0 ? 0.0 : (values[0] > 100.0 ? 100.0 : values[0]);
    out->dram_read_bytes = values[1];
    out->dram_write_bytes = values[2];
    ok = true;
  } while (false);
  CUpti_RangeProfiler_Disable_Params dp{};
  dp.structSize = CUpti_RangeProfiler_Disable_Params_STRUCT_SIZE;
  dp.pRangeProfilerObject = rp;
  c.rp_disable(&dp);
  host_done();
  if (!ok) out->why = "range profiling failed";
  return ok;
}

}  // namespace cucosma
