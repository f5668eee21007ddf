// gdf_oracle_count.cpp -- the CPU oracle built on the counting scalar of
// flopcount.h: the same source (gdf_oracle.cpp) with every double of its
// arithmetic counted. TEST AND MEASUREMENT INFRASTRUCTURE ONLY. Built
// single-threaded (no OpenMP pragmas), so the tally is exact; the values
// equal the plain oracle's (tests/test_flop_count.py checks it).
#include "flopcount.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <omp.h>
#include <vector>

#include "../include/gdf.h"
#include "../include/gdf_p3.h"

FlopTally g_flops;

#define GDF_ORACLE_NO_P3 1
#define double fcnt
#include "gdf_oracle.cpp"
#undef double

extern "C" {
// counters since the last reset: add (+ and -), mul, div, sqrt, pow
void orc_flops(uint64_t* out) {
  out[0] = g_flops.add;
  out[1] = g_flops.mul;
  out[2] = g_flops.div;
  out[3] = g_flops.sqrt;
  out[4] = g_flops.pow;
}
void orc_flops_reset(void) { g_flops = FlopTally(); }
}
