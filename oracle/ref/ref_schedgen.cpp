// Runs the reference ScheduleGenerator (ScheduleGenerator/ScheduleGeneratorv4.h:13,
// generateSchedulev3) for shapes given on the command line and prints one CSV
// row per shape in the column order of ScheduleGenerator/main.cpp:309-331.
// Compiled from the reference sources where they lie by oracle/build_ref.py.
// TEST INFRASTRUCTURE ONLY.
#include <cstdint>
#include <cstdlib>
#include <iostream>
#include <string>
#include "Parameters.h"
#include "Schedule.h"
#include "Threadblock.h"
#include "Threadtile.h"
#include "Warptile.h"
#include "matrix.h"
#include "ScheduleGeneratorv4.h"

int main(int argc, char** argv) {
  // argv: m n k [m n k ...]  (alpha/beta are fixed constants of Parameters, ParametersV100.h:52-53)
  if (argc < 4 || (argc - 1) % 3 != 0) {
    std::cerr << "usage: ref_schedgen m n k [m n k ...]\n";
    return 2;
  }
  Parameters p;
  // main.cpp:257-263
  p.registers_per_threadblock = std::min(p.registers_per_SM / 2, p.registers_per_threadblock);
  p.shared_memory_per_threadblock = std::min(p.shared_memory_per_SM / 2, p.shared_memory_per_threadblock);
  p.registers_per_warp = p.registers_per_threadblock;
  p.register_per_thread = std::min((long long int)(p.registers_per_warp / p.threads_per_warp), p.max_registers_per_thread);
  for (int a = 1; a + 2 < argc; a += 3) {
    p.m = std::atoll(argv[a]);
    p.n = std::atoll(argv[a + 1]);
    p.k = std::atoll(argv[a + 2]);
    Threadblock tb;
    Warptile wt;
    Threadtile tt;
    std::streambuf* old = std::cout.rdbuf(nullptr);  // generateSchedulev3 prints progress
    bool ok = generateSchedulev3(p, tb, wt, tt);
    std::cout.rdbuf(old);
    if (!ok) {
      std::cout << "none," << p.m << "," << p.n << "," << p.k << "\n";
      continue;
    }
    const char* atomic = (p.m * p.n * tb.numTilesK < 260 * 260 * 32) ? "true" : "false";  // main.cpp:302-306
    std::cout << tb.occupancy << "," << p.type << "," << p.vectortype2 << "," << p.vectortype4 << ","
              << p.m << "," << p.n << "," << p.k << "," << tb.tileSizeM << "," << tb.tileSizeN << ","
              << tb.tileSizeK << "," << tb.k_load << "," << wt.tileSizeM << "," << wt.tileSizeN << ","
              << tt.tileSizeM << "," << tt.tileSizeN << "," << tb.numTilesK << "," << p.alpha << ","
              << p.beta << "," << 1 << "," << tb.A_Offset << "," << tb.B_Offset << "," << atomic << "\n";
  }
  return 0;
}
