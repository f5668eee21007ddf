// gdf_mlp.cuh -- the learned troubled-cell indicator: a 90-64-64-1 MLP
// (GELU, GELU, sigmoid) whose matrix products run on the tensor cores as
// BF16 mma.sync.m16n8k16 tiles with FP32 accumulation.
//
// Weights in BF16 for the tensor-core products, biases and the last layer
// in FP32. Shared-memory tile layouts (row-major, padded rows so that the
// fragment loads of a warp touch 32 distinct banks):
//   X   [rows][MLP_LDX]  inputs, 90 used, 96 (6 k-steps of 16) multiplied
//   W1t [64][MLP_LDX]    W1 transposed (hidden unit, input)
//   W2t [64][MLP_LDH]    W2 transposed (output unit, hidden unit)
//   H1  [rows][MLP_LDH]  first hidden layer
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace gdf {

constexpr int MLP_IN = 90;
constexpr int MLP_INP = 96;   // padded input width
constexpr int MLP_H = 64;
constexpr int MLP_LDX = 104;  // 96 + 8: 52 words per row
constexpr int MLP_LDH = 72;   // 64 + 8: 36 words per row
// packed FP32 parameter vector (numpy layout): W1[90][64], b1[64], W2[64][64], b2[64], w3[64], b3
constexpr int MLP_OFF_W1 = 0;
constexpr int MLP_OFF_B1 = MLP_IN * MLP_H;
constexpr int MLP_OFF_W2 = MLP_OFF_B1 + MLP_H;
constexpr int MLP_OFF_B2 = MLP_OFF_W2 + MLP_H * MLP_H;
constexpr int MLP_OFF_W3 = MLP_OFF_B2 + MLP_H;
constexpr int MLP_OFF_B3 = MLP_OFF_W3 + MLP_H;
constexpr int MLP_NPARAM = MLP_OFF_B3 + 1;   // 10049

// Device copy of the network for the kernels.
struct MlpDev {
  __nv_bfloat16 W1t[MLP_H * MLP_INP];   // [n][k], k >= 90 zero
  __nv_bfloat16 W2t[MLP_H * MLP_H];     // [o][i]
  __nv_bfloat16 W2n[MLP_H * MLP_H];     // [i][o] (for the backward product)
  float b1[MLP_H], b2[MLP_H], w3[MLP_H], b3;   // w3 holds bf16-rounded values
};

__device__ __forceinline__ void mma16816(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// A fragment (16x16 at rows r0.., cols k0..) of a row-major bf16 tile
__device__ __forceinline__ void load_a(uint32_t a[4], const __nv_bfloat16* A, int ld, int r0, int k0, int lane) {
  const int g = lane >> 2, t = lane & 3;
  a[0] = *reinterpret_cast<const uint32_t*>(A + (r0 + g) * ld + k0 + 2 * t);
  a[1] = *reinterpret_cast<const uint32_t*>(A + (r0 + g + 8) * ld + k0 + 2 * t);
  a[2] = *reinterpret_cast<const uint32_t*>(A + (r0 + g) * ld + k0 + 8 + 2 * t);
  a[3] = *reinterpret_cast<const uint32_t*>(A + (r0 + g + 8) * ld + k0 + 8 + 2 * t);
}

// B fragment (16x8 at k0.., n0..) of B given transposed (Bt[n][k], row-major)
__device__ __forceinline__ void load_b(uint32_t b[2], const __nv_bfloat16* Bt, int ld, int k0, int n0, int lane) {
  const int g = lane >> 2, t = lane & 3;
  b[0] = *reinterpret_cast<const uint32_t*>(Bt + (n0 + g) * ld + k0 + 2 * t);
  b[1] = *reinterpret_cast<const uint32_t*>(Bt + (n0 + g) * ld + k0 + 8 + 2 * t);
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float x) {
  return 0.5f * (1.f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// Inference for the 16-row tiles r0 = 16*w, 16*(w+nw), ... of X (rows
// samples): p[row] = sigmoid(w3 . gelu(gelu(X W1 + b1) W2 + b2) + b3).
// H1 is a scratch tile of the same rows. Called by every thread of the
// block; returns after a __syncthreads().
__device__ __forceinline__ void mlp_infer_tiles(const __nv_bfloat16* X, const __nv_bfloat16* W1t,
                                                const __nv_bfloat16* W2t, const float* b1, const float* b2,
                                                const float* w3, float b3, __nv_bfloat16* H1, float* z_out,
                                                int rows) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  for (int r0 = 16 * warp; r0 < rows; r0 += 16 * nw) {
    float c[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) c[nt][e] = 0.f;
#pragma unroll
    for (int k0 = 0; k0 < MLP_INP; k0 += 16) {
      uint32_t a[4];
      load_a(a, X, MLP_LDX, r0, k0, lane);
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        uint32_t b[2];
        load_b(b, W1t, MLP_LDX, k0, nt * 8, lane);
        mma16816(c[nt], a, b);
      }
    }
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int col = nt * 8 + 2 * t;
      H1[(r0 + g) * MLP_LDH + col] = __float2bfloat16_rn(gelu(c[nt][0] + b1[col]));
      H1[(r0 + g) * MLP_LDH + col + 1] = __float2bfloat16_rn(gelu(c[nt][1] + b1[col + 1]));
      H1[(r0 + g + 8) * MLP_LDH + col] = __float2bfloat16_rn(gelu(c[nt][2] + b1[col]));
      H1[(r0 + g + 8) * MLP_LDH + col + 1] = __float2bfloat16_rn(gelu(c[nt][3] + b1[col + 1]));
    }
    __syncwarp();
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) c[nt][e] = 0.f;
#pragma unroll
    for (int k0 = 0; k0 < MLP_H; k0 += 16) {
      uint32_t a[4];
      load_a(a, H1, MLP_LDH, r0, k0, lane);
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        uint32_t b[2];
        load_b(b, W2t, MLP_LDH, k0, nt * 8, lane);
        mma16816(c[nt], a, b);
      }
    }
    float s0 = 0.f, s1 = 0.f;   // rows g and g+8
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int col = nt * 8 + 2 * t;
      s0 += gelu(c[nt][0] + b2[col]) * w3[col] + gelu(c[nt][1] + b2[col + 1]) * w3[col + 1];
      s1 += gelu(c[nt][2] + b2[col]) * w3[col] + gelu(c[nt][3] + b2[col + 1]) * w3[col + 1];
    }
    s0 += __shfl_xor_sync(0xffffffffu, s0, 1);
    s0 += __shfl_xor_sync(0xffffffffu, s0, 2);
    s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
    s1 += __shfl_xor_sync(0xffffffffu, s1, 2);
    if (t == 0) {
      z_out[r0 + g] = s0 + b3;
      z_out[r0 + g + 8] = s1 + b3;
    }
  }
  __syncthreads();
}

}  // namespace gdf
