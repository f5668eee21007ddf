// gdf_peak.cu -- FP64 FMA throughput probe (no counterpart in the
// reference). The GDF step is FP64-bound, so its roofline needs a measured
// FP64 ceiling beside the measured HBM one: this kernel keeps every SM's
// FP64 pipe busy with independent fused multiply-add chains and nothing
// else (no memory traffic inside the loop), and the host times it with CUDA
// events. Explicit __fma_rn calls make it a DFMA stream in every build,
// whatever the contraction flags of the library.
#include <cuda_runtime.h>

#include <string>

#include "../../include/gdf.h"

namespace gdf {
int set_last_error(int code, const char* msg);
}

namespace {

constexpr int PEAK_BS = 256;
constexpr int PEAK_CHAINS = 8;   // independent dependency chains per thread

__global__ void __launch_bounds__(PEAK_BS) k_fp64_fma(double* __restrict__ out, int iters, double a, double b) {
  double x[PEAK_CHAINS];
#pragma unroll
  for (int c = 0; c < PEAK_CHAINS; ++c) x[c] = 1e-3 * (threadIdx.x + 1) + c;
#pragma unroll 1
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u)
#pragma unroll
      for (int c = 0; c < PEAK_CHAINS; ++c) x[c] = __fma_rn(x[c], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < PEAK_CHAINS; ++c) s += x[c];
  // a store the compiler cannot drop; the chains converge to b / (1 - a)
  if (s == 12345.678) out[blockIdx.x * PEAK_BS + threadIdx.x] = s;
}

}  // namespace

extern "C" int gdf_fp64_fma_peak(int32_t blocks_per_sm, int32_t iters, double* tflops, double* ms_out) {
  if (!tflops || blocks_per_sm < 1 || blocks_per_sm > 32 || iters < 1)
    return gdf::set_last_error(GDF_ERR_ARG, "gdf_fp64_fma_peak: bad argument");
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return gdf::set_last_error(GDF_ERR_CUDA, "gdf_fp64_fma_peak: no device");
  const int blocks = sms * blocks_per_sm;
  double* out = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  std::string err;
  if (cudaMalloc(&out, sizeof(double) * blocks * PEAK_BS) != cudaSuccess || cudaStreamCreate(&st) != cudaSuccess ||
      cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    err = "gdf_fp64_fma_peak: set-up failed";
  } else {
    const double a = 0.999999, b = 1e-7;
    k_fp64_fma<<<blocks, PEAK_BS, 0, st>>>(out, iters, a, b);    // warm-up
    cudaEventRecord(e0, st);
    k_fp64_fma<<<blocks, PEAK_BS, 0, st>>>(out, iters, a, b);
    cudaEventRecord(e1, st);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e != cudaSuccess) {
      err = std::string("gdf_fp64_fma_peak: ") + cudaGetErrorString(e);
    } else {
      const double flops = 2.0 * PEAK_CHAINS * 16.0 * (double)iters * (double)blocks * PEAK_BS;
      *tflops = flops / (ms * 1e-3) / 1e12;
      if (ms_out) *ms_out = ms;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  if (out) cudaFree(out);
  if (!err.empty()) return gdf::set_last_error(GDF_ERR_CUDA, err.c_str());
  return GDF_OK;
}
