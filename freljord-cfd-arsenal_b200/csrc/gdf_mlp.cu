// gdf_mlp.cu -- training and inference kernels of the learned troubled-cell
// indicator (90-64-64-1 MLP, BF16 tensor-core products, FP32 accumulation,
// Adam on FP32 master weights), and its part of the C ABI.
//
// One training step over a minibatch of B samples:
//   k_mlp_fwdbwd   64 samples per block: forward, loss, backward, and the
//                  block's gradient written to its own slot (no atomics)
//   k_mlp_reduce   gradient = sum of the block slots in block order
//   k_mlp_adam     Adam update of the FP32 master parameters
//   k_mlp_sync     BF16 / transposed device copy for the next step
// Roundings to BF16 (the operands of the tensor-core products): inputs X,
// W1, W2, w3, the first hidden layer H1, and the back-propagated dZ2, dZ1.
// Everything else is FP32. tests/test_mlp.py restates this in numpy.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/gdf.h"
#include "gdf_mlp.cuh"

using namespace gdf;

namespace gdf {
// gdf_mlp_tc.cu: the training tile on tcgen05 (128 samples per CTA)
int mlp_tc_samples_per_block();
cudaError_t mlp_fwdbwd_tc_launch(const MlpDev* D, const __nv_bfloat16* X, const float* y, const int* idx, int nsel,
                                 float pos_w, float inv_b, float* partial, float* loss_part, int* err,
                                 cudaStream_t st);
}  // namespace gdf

namespace {

thread_local std::string g_mlp_err;
int mfail(int code, const std::string& m) {
  g_mlp_err = m;
  return code;
}
#define MCK(call)                                                                          \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) return mfail(GDF_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
  } while (0)

constexpr int TB = 64;        // samples per block
constexpr int LDT = 72;       // transposed tiles: 64 samples + 8
constexpr int MLP_THREADS = 128;

struct FwdSmem {
  __nv_bfloat16 Xs[TB * MLP_LDX];
  __nv_bfloat16 Xt[MLP_INP * LDT];
  __nv_bfloat16 W1t[MLP_H * MLP_LDX];
  __nv_bfloat16 W2t[MLP_H * MLP_LDH];
  __nv_bfloat16 W2n[MLP_H * MLP_LDH];
  __nv_bfloat16 H1b[TB * MLP_LDH];
  __nv_bfloat16 H1t[MLP_H * LDT];
  __nv_bfloat16 dZ2b[TB * MLP_LDH];
  __nv_bfloat16 dZ2t[MLP_H * LDT];
  __nv_bfloat16 dZ1t[MLP_H * LDT];
  float b1[MLP_H], b2[MLP_H], w3[MLP_H];
  float yv[TB], wv[TB], g3[TB], lossv[TB];
  float red_b1[4][MLP_H], red_b2[4][MLP_H], red_w3[4][MLP_H];
};

static_assert(GDF_MLP_NPARAM == MLP_NPARAM, "gdf.h and gdf_mlp.cuh disagree on the parameter count");

__global__ void k_mlp_sync(const float* __restrict__ P, MlpDev* __restrict__ D) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < MLP_H * MLP_INP) {
    const int n = t / MLP_INP, k = t % MLP_INP;
    D->W1t[t] = __float2bfloat16_rn(k < MLP_IN ? P[MLP_OFF_W1 + k * MLP_H + n] : 0.f);
  }
  if (t < MLP_H * MLP_H) {
    const int o = t / MLP_H, i = t % MLP_H;
    D->W2t[t] = __float2bfloat16_rn(P[MLP_OFF_W2 + i * MLP_H + o]);
    D->W2n[t] = __float2bfloat16_rn(P[MLP_OFF_W2 + o * MLP_H + i]);
  }
  if (t < MLP_H) {
    D->b1[t] = P[MLP_OFF_B1 + t];
    D->b2[t] = P[MLP_OFF_B2 + t];
    D->w3[t] = __bfloat162float(__float2bfloat16_rn(P[MLP_OFF_W3 + t]));
  }
  if (t == 0) D->b3 = P[MLP_OFF_B3];
}

// Forward + backward of one 64-sample tile; block b writes its gradient to
// partial[b * MLP_NPARAM ...] and its loss to loss_part[b].
__global__ void __launch_bounds__(MLP_THREADS) k_mlp_fwdbwd(const MlpDev* __restrict__ D,
                                                            const __nv_bfloat16* __restrict__ X,
                                                            const float* __restrict__ y,
                                                            const int* __restrict__ idx, int nsel, float pos_w,
                                                            float inv_b, float* __restrict__ partial,
                                                            float* __restrict__ loss_part) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  FwdSmem& S = *reinterpret_cast<FwdSmem*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int base = blockIdx.x * TB;
  // parameters
  for (int k = tid; k < MLP_H * MLP_INP; k += MLP_THREADS) S.W1t[(k / MLP_INP) * MLP_LDX + k % MLP_INP] = D->W1t[k];
  for (int k = tid; k < MLP_H * MLP_H; k += MLP_THREADS) {
    S.W2t[(k / MLP_H) * MLP_LDH + k % MLP_H] = D->W2t[k];
    S.W2n[(k / MLP_H) * MLP_LDH + k % MLP_H] = D->W2n[k];
  }
  if (tid < MLP_H) {
    S.b1[tid] = D->b1[tid];
    S.b2[tid] = D->b2[tid];
    S.w3[tid] = D->w3[tid];
  }
  // samples
  for (int k = tid; k < TB * MLP_INP; k += MLP_THREADS) {
    const int r = k / MLP_INP, c = k % MLP_INP;
    const int q = base + r;
    __nv_bfloat16 v = __float2bfloat16_rn(0.f);
    if (q < nsel) v = X[(long long)idx[q] * MLP_INP + c];
    S.Xs[r * MLP_LDX + c] = v;
    S.Xt[c * LDT + r] = v;
  }
  if (tid < TB) {
    const int q = base + tid;
    const float yy = q < nsel ? y[idx[q]] : 0.f;
    S.yv[tid] = yy;
    S.wv[tid] = q < nsel ? (yy > 0.5f ? pos_w : 1.f) : 0.f;
  }
  __syncthreads();
  const float b3 = D->b3;
  const int r0 = 16 * warp;
  // layer 1
  float z1[8][4];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
#pragma unroll
    for (int e = 0; e < 4; ++e) z1[nt][e] = 0.f;
#pragma unroll
  for (int k0 = 0; k0 < MLP_INP; k0 += 16) {
    uint32_t a[4];
    load_a(a, S.Xs, MLP_LDX, r0, k0, lane);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      uint32_t b[2];
      load_b(b, S.W1t, MLP_LDX, k0, nt * 8, lane);
      mma16816(z1[nt], a, b);
    }
  }
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const int col = nt * 8 + 2 * t;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int row = r0 + g + (e >= 2 ? 8 : 0), cc = col + (e & 1);
      z1[nt][e] += S.b1[cc];
      const __nv_bfloat16 h = __float2bfloat16_rn(gelu(z1[nt][e]));
      S.H1b[row * MLP_LDH + cc] = h;
      S.H1t[cc * LDT + row] = h;
    }
  }
  __syncwarp();
  // layer 2
  float z2[8][4];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
#pragma unroll
    for (int e = 0; e < 4; ++e) z2[nt][e] = 0.f;
#pragma unroll
  for (int k0 = 0; k0 < MLP_H; k0 += 16) {
    uint32_t a[4];
    load_a(a, S.H1b, MLP_LDH, r0, k0, lane);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      uint32_t b[2];
      load_b(b, S.W2t, MLP_LDH, k0, nt * 8, lane);
      mma16816(z2[nt], a, b);
    }
  }
  float s0 = 0.f, s1 = 0.f;
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const int col = nt * 8 + 2 * t;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int cc = col + (e & 1);
      z2[nt][e] += S.b2[cc];
      const float h2 = gelu(z2[nt][e]);
      if (e < 2) s0 += h2 * S.w3[cc]; else s1 += h2 * S.w3[cc];
    }
  }
  s0 += __shfl_xor_sync(0xffffffffu, s0, 1);
  s0 += __shfl_xor_sync(0xffffffffu, s0, 2);
  s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
  s1 += __shfl_xor_sync(0xffffffffu, s1, 2);
  if (t == 0) {
    // stable weighted binary cross-entropy and dL/dz3 = w (p - y) / B
    for (int h = 0; h < 2; ++h) {
      const int row = r0 + g + 8 * h;
      const float z = (h == 0 ? s0 : s1) + b3;
      const float p = 1.f / (1.f + expf(-z));
      const float yy = S.yv[row], wt = S.wv[row];
      const float sp_pos = fmaxf(z, 0.f) + log1pf(expf(-fabsf(z)));   // softplus(z) = -log(1-p)
      const float l = yy * (sp_pos - z) + (1.f - yy) * sp_pos;            // -y log p - (1-y) log(1-p)
      S.lossv[row] = wt * l * inv_b;
      S.g3[row] = wt * (p - yy) * inv_b;
    }
  }
  __syncwarp();
  const float ga = S.g3[r0 + g], gb = S.g3[r0 + g + 8];
  // dZ2 = (g3 w3) * gelu'(z2); bias and w3 gradients (FP32)
  float db2p[8][2], dw3p[8][2];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const int col = nt * 8 + 2 * t;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int row = r0 + g + (e >= 2 ? 8 : 0), cc = col + (e & 1);
      const float gr = e >= 2 ? gb : ga;
      const float h2 = gelu(z2[nt][e]);
      const float dz = gr * S.w3[cc] * gelu_d(z2[nt][e]);
      const __nv_bfloat16 dzb = __float2bfloat16_rn(dz);
      S.dZ2b[row * MLP_LDH + cc] = dzb;
      S.dZ2t[cc * LDT + row] = dzb;
      if (e < 2) { db2p[nt][e] = dz; dw3p[nt][e] = gr * h2; }
      else { db2p[nt][e - 2] += dz; dw3p[nt][e - 2] += gr * h2; }
    }
  }
  // reduce over the 8 row groups of the warp, then store the warp's column sums
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      float a = db2p[nt][e], b = dw3p[nt][e];
      for (int m = 4; m < 32; m <<= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, m);
        b += __shfl_xor_sync(0xffffffffu, b, m);
      }
      if (g == 0) {
        S.red_b2[warp][nt * 8 + 2 * t + e] = a;
        S.red_w3[warp][nt * 8 + 2 * t + e] = b;
      }
    }
  __syncwarp();
  // dH1 = dZ2 W2^T, dZ1 = dH1 * gelu'(z1)
  float d1[8][4];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
#pragma unroll
    for (int e = 0; e < 4; ++e) d1[nt][e] = 0.f;
#pragma unroll
  for (int k0 = 0; k0 < MLP_H; k0 += 16) {
    uint32_t a[4];
    load_a(a, S.dZ2b, MLP_LDH, r0, k0, lane);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      uint32_t b[2];
      load_b(b, S.W2n, MLP_LDH, k0, nt * 8, lane);
      mma16816(d1[nt], a, b);
    }
  }
  float db1p[8][2];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const int col = nt * 8 + 2 * t;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int row = r0 + g + (e >= 2 ? 8 : 0), cc = col + (e & 1);
      const float dz = d1[nt][e] * gelu_d(z1[nt][e]);
      S.dZ1t[cc * LDT + row] = __float2bfloat16_rn(dz);
      if (e < 2) db1p[nt][e] = dz; else db1p[nt][e - 2] += dz;
    }
  }
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      float a = db1p[nt][e];
      for (int m = 4; m < 32; m <<= 1) a += __shfl_xor_sync(0xffffffffu, a, m);
      if (g == 0) S.red_b1[warp][nt * 8 + 2 * t + e] = a;
    }
  __syncthreads();
  float* out = partial + (long long)blockIdx.x * MLP_NPARAM;
  // dW2t[o][i] = sum_s dZ2t[o][s] H1t[i][s]: warp rows o = 16w..16w+15
  {
    float c[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) c[nt][e] = 0.f;
#pragma unroll
    for (int k0 = 0; k0 < TB; k0 += 16) {
      uint32_t a[4];
      load_a(a, S.dZ2t, LDT, r0, k0, lane);
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        uint32_t b[2];
        load_b(b, S.H1t, LDT, k0, nt * 8, lane);
        mma16816(c[nt], a, b);
      }
    }
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int o = r0 + g + (e >= 2 ? 8 : 0), i = nt * 8 + 2 * t + (e & 1);
        out[MLP_OFF_W2 + i * MLP_H + o] = c[nt][e];
      }
  }
  // dW1t[n][k] = sum_s dZ1t[n][s] Xt[k][s]: warp rows n = 16w.., 12 column tiles
  {
#pragma unroll 1
    for (int half = 0; half < 2; ++half) {
      float c[6][4];
#pragma unroll
      for (int nt = 0; nt < 6; ++nt)
#pragma unroll
        for (int e = 0; e < 4; ++e) c[nt][e] = 0.f;
#pragma unroll
      for (int k0 = 0; k0 < TB; k0 += 16) {
        uint32_t a[4];
        load_a(a, S.dZ1t, LDT, r0, k0, lane);
#pragma unroll
        for (int nt = 0; nt < 6; ++nt) {
          uint32_t b[2];
          load_b(b, S.Xt, LDT, k0, (half * 6 + nt) * 8, lane);
          mma16816(c[nt], a, b);
        }
      }
#pragma unroll
      for (int nt = 0; nt < 6; ++nt)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int n = r0 + g + (e >= 2 ? 8 : 0), k = (half * 6 + nt) * 8 + 2 * t + (e & 1);
          if (k < MLP_IN) out[MLP_OFF_W1 + k * MLP_H + n] = c[nt][e];
        }
    }
  }
  if (tid < MLP_H) {
    out[MLP_OFF_B1 + tid] = ((S.red_b1[0][tid] + S.red_b1[1][tid]) + S.red_b1[2][tid]) + S.red_b1[3][tid];
    out[MLP_OFF_B2 + tid] = ((S.red_b2[0][tid] + S.red_b2[1][tid]) + S.red_b2[2][tid]) + S.red_b2[3][tid];
    out[MLP_OFF_W3 + tid] = ((S.red_w3[0][tid] + S.red_w3[1][tid]) + S.red_w3[2][tid]) + S.red_w3[3][tid];
  }
  if (tid == 0) {
    float gs = 0.f, ls = 0.f;
    for (int r = 0; r < TB; ++r) {
      gs += S.g3[r];
      ls += S.lossv[r];
    }
    out[MLP_OFF_B3] = gs;
    loss_part[blockIdx.x] = ls;
  }
}

// grad[p] = sum over blocks (in block order) of partial[b][p]
__global__ void k_mlp_reduce(const float* __restrict__ partial, int nb, float* __restrict__ grad,
                             const float* __restrict__ loss_part, float* __restrict__ loss) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < MLP_NPARAM) {
    float s = 0.f;
    for (int b = 0; b < nb; ++b) s += partial[(long long)b * MLP_NPARAM + p];
    grad[p] = s;
  }
  if (p == 0 && loss) {
    float s = 0.f;
    for (int b = 0; b < nb; ++b) s += loss_part[b];
    *loss = s;
  }
}

__global__ void k_mlp_adam(float* __restrict__ P, float* __restrict__ M, float* __restrict__ V,
                           const float* __restrict__ grad, float lr, float b1, float b2, float eps, float c1,
                           float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= MLP_NPARAM) return;
  const float gr = grad[p];
  const float m = b1 * M[p] + (1.f - b1) * gr;
  const float v = b2 * V[p] + (1.f - b2) * gr * gr;
  M[p] = m;
  V[p] = v;
  P[p] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
}

__global__ void __launch_bounds__(MLP_THREADS) k_mlp_predict(const MlpDev* __restrict__ D,
                                                             const __nv_bfloat16* __restrict__ X, int n,
                                                             float* __restrict__ out) {
  __shared__ __align__(16) __nv_bfloat16 Xs[TB * MLP_LDX];
  __shared__ __align__(16) __nv_bfloat16 W1t[MLP_H * MLP_LDX];
  __shared__ __align__(16) __nv_bfloat16 W2t[MLP_H * MLP_LDH];
  __shared__ __align__(16) __nv_bfloat16 H1[TB * MLP_LDH];
  __shared__ float z[TB];
  const int tid = threadIdx.x, base = blockIdx.x * TB;
  for (int k = tid; k < MLP_H * MLP_INP; k += MLP_THREADS) W1t[(k / MLP_INP) * MLP_LDX + k % MLP_INP] = D->W1t[k];
  for (int k = tid; k < MLP_H * MLP_H; k += MLP_THREADS) W2t[(k / MLP_H) * MLP_LDH + k % MLP_H] = D->W2t[k];
  for (int k = tid; k < TB * MLP_INP; k += MLP_THREADS) {
    const int r = k / MLP_INP, c = k % MLP_INP;
    Xs[r * MLP_LDX + c] = base + r < n ? X[(long long)(base + r) * MLP_INP + c] : __float2bfloat16_rn(0.f);
  }
  __syncthreads();
  mlp_infer_tiles(Xs, W1t, W2t, D->b1, D->b2, D->w3, D->b3, H1, z, TB);
  if (tid < TB && base + tid < n) out[base + tid] = 1.f / (1.f + expf(-z[tid]));
}

// FP32 host features [n][90] -> BF16 device rows [n][96]
__global__ void k_to_bf16(const float* __restrict__ Xf, __nv_bfloat16* __restrict__ Xb, long long n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * MLP_INP) return;
  const long long r = t / MLP_INP;
  const int c = (int)(t % MLP_INP);
  Xb[t] = __float2bfloat16_rn(c < MLP_IN ? Xf[r * MLP_IN + c] : 0.f);
}

}  // namespace

struct GdfMlp {
  cudaStream_t st = nullptr;
  float *P = nullptr, *M = nullptr, *V = nullptr, *grad = nullptr, *loss = nullptr;
  MlpDev* D = nullptr;
  float* partial = nullptr;
  float* loss_part = nullptr;
  int part_blocks = 0;
  __nv_bfloat16* X = nullptr;
  float* y = nullptr;
  int* idx = nullptr;
  long long cap = 0;
  long long adam_t = 0;
  int tc = 1;                 // products: 1 tcgen05 (UMMA, TMEM), 0 mma.sync
  int* err = nullptr;         // set by a tcgen05 tile whose bounded wait gave up
};

// samples per training block of the selected products
static int mlp_tile(const GdfMlp* m) { return m->tc ? mlp_tc_samples_per_block() : TB; }

static int mlp_ensure(GdfMlp* m, long long n, int blocks) {
  if (n > m->cap) {
    if (m->X) cudaFree(m->X);
    if (m->y) cudaFree(m->y);
    if (m->idx) cudaFree(m->idx);
    m->X = nullptr; m->y = nullptr; m->idx = nullptr;
    MCK(cudaMalloc((void**)&m->X, (size_t)n * MLP_INP * sizeof(__nv_bfloat16)));
    MCK(cudaMalloc((void**)&m->y, (size_t)n * sizeof(float)));
    MCK(cudaMalloc((void**)&m->idx, (size_t)n * sizeof(int)));
    m->cap = n;
  }
  if (blocks > m->part_blocks) {
    if (m->partial) cudaFree(m->partial);
    if (m->loss_part) cudaFree(m->loss_part);
    m->partial = nullptr; m->loss_part = nullptr;
    MCK(cudaMalloc((void**)&m->partial, (size_t)blocks * MLP_NPARAM * sizeof(float)));
    MCK(cudaMalloc((void**)&m->loss_part, (size_t)blocks * sizeof(float)));
    m->part_blocks = blocks;
  }
  return GDF_OK;
}

static int mlp_upload_x(GdfMlp* m, const float* X, long long n) {
  float* tmp = nullptr;
  MCK(cudaMallocAsync((void**)&tmp, (size_t)n * MLP_IN * sizeof(float), m->st));
  MCK(cudaMemcpyAsync(tmp, X, (size_t)n * MLP_IN * sizeof(float), cudaMemcpyHostToDevice, m->st));
  const long long tot = n * MLP_INP;
  k_to_bf16<<<(unsigned)((tot + 255) / 256), 256, 0, m->st>>>(tmp, m->X, n);
  MCK(cudaGetLastError());
  MCK(cudaFreeAsync(tmp, m->st));
  return GDF_OK;
}

static int mlp_sync(GdfMlp* m) {
  k_mlp_sync<<<(MLP_H * MLP_INP + 255) / 256, 256, 0, m->st>>>(m->P, m->D);
  MCK(cudaGetLastError());
  return GDF_OK;
}

static int fwdbwd_attr() {
  MCK(cudaFuncSetAttribute(k_mlp_fwdbwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(FwdSmem)));
  return GDF_OK;
}

// forward + backward of nsel samples (idx) into m->partial / loss_part
static int fwdbwd_launch(GdfMlp* m, const int* idx, long long nsel, float pos_w, float inv_b, int& nb) {
  nb = (int)((nsel + mlp_tile(m) - 1) / mlp_tile(m));
  if (m->tc) {
    MCK(mlp_fwdbwd_tc_launch(m->D, m->X, m->y, idx, (int)nsel, pos_w, inv_b, m->partial, m->loss_part, m->err,
                             m->st));
  } else {
    int rc = fwdbwd_attr();
    if (rc) return rc;
    k_mlp_fwdbwd<<<nb, MLP_THREADS, sizeof(FwdSmem), m->st>>>(m->D, m->X, m->y, idx, (int)nsel, pos_w, inv_b,
                                                              m->partial, m->loss_part);
    MCK(cudaGetLastError());
  }
  return GDF_OK;
}

// the error word of the tcgen05 tiles (read back after a synchronisation)
static int check_err(GdfMlp* m) {
  int e = 0;
  MCK(cudaMemcpyAsync(&e, m->err, sizeof(int), cudaMemcpyDeviceToHost, m->st));
  MCK(cudaStreamSynchronize(m->st));
  if (e) {
    MCK(cudaMemsetAsync(m->err, 0, sizeof(int), m->st));
    return mfail(GDF_ERR_TIMEOUT, "a tensor-core training tile gave up waiting for its products");
  }
  return GDF_OK;
}

static int mlp_grad_launch(GdfMlp* m, long long nsel, float pos_w, float inv_b) {
  int nb = 0;
  int rc = fwdbwd_launch(m, m->idx, nsel, pos_w, inv_b, nb);
  if (rc) return rc;
  k_mlp_reduce<<<(MLP_NPARAM + 255) / 256, 256, 0, m->st>>>(m->partial, nb, m->grad, m->loss_part, m->loss);
  MCK(cudaGetLastError());
  return GDF_OK;
}

extern "C" {

const char* gdf_mlp_last_error(void) { return g_mlp_err.c_str(); }

int gdf_mlp_create(int32_t seed, GdfMlp** out) {
  if (!out) return mfail(GDF_ERR_ARG, "null handle pointer");
  GdfMlp* m = new GdfMlp();
  bool ok = cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&m->P, MLP_NPARAM * sizeof(float)) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&m->M, MLP_NPARAM * sizeof(float)) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&m->V, MLP_NPARAM * sizeof(float)) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&m->grad, MLP_NPARAM * sizeof(float)) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&m->loss, sizeof(float)) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&m->D, sizeof(MlpDev)) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&m->err, sizeof(int)) == cudaSuccess && cudaMemset(m->err, 0, sizeof(int)) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    gdf_mlp_destroy(m);
    return mfail(GDF_ERR_CUDA, "allocation of the indicator network failed (is a CUDA device present?)");
  }
  // Glorot-uniform weights, zero biases, from a seeded generator
  std::vector<float> p(MLP_NPARAM, 0.f);
  std::mt19937 rng((uint32_t)seed);
  auto fill = [&](int off, int fan_in, int fan_out, int count) {
    const float a = std::sqrt(6.f / (float)(fan_in + fan_out));
    std::uniform_real_distribution<float> u(-a, a);
    for (int q = 0; q < count; ++q) p[off + q] = u(rng);
  };
  fill(MLP_OFF_W1, MLP_IN, MLP_H, MLP_IN * MLP_H);
  fill(MLP_OFF_W2, MLP_H, MLP_H, MLP_H * MLP_H);
  fill(MLP_OFF_W3, MLP_H, 1, MLP_H);
  int rc = gdf_mlp_set_params(m, p.data());
  if (rc) {
    gdf_mlp_destroy(m);
    return rc;
  }
  *out = m;
  return GDF_OK;
}

int gdf_mlp_destroy(GdfMlp* m) {
  if (!m) return GDF_OK;
  void* bufs[] = {m->P, m->M, m->V, m->grad, m->loss, m->D, m->partial, m->loss_part, m->X, m->y, m->idx, m->err};
  for (void* b : bufs)
    if (b) cudaFree(b);
  if (m->st) cudaStreamDestroy(m->st);
  delete m;
  return GDF_OK;
}

int gdf_mlp_set_params(GdfMlp* m, const float* params) {
  if (!m || !params) return mfail(GDF_ERR_ARG, "null argument");
  MCK(cudaMemcpyAsync(m->P, params, MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice, m->st));
  MCK(cudaMemsetAsync(m->M, 0, MLP_NPARAM * sizeof(float), m->st));
  MCK(cudaMemsetAsync(m->V, 0, MLP_NPARAM * sizeof(float), m->st));
  m->adam_t = 0;
  int rc = mlp_sync(m);
  if (rc) return rc;
  MCK(cudaStreamSynchronize(m->st));
  return GDF_OK;
}

int gdf_mlp_get_params(GdfMlp* m, float* params) {
  if (!m || !params) return mfail(GDF_ERR_ARG, "null argument");
  MCK(cudaMemcpyAsync(params, m->P, MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, m->st));
  MCK(cudaStreamSynchronize(m->st));
  return GDF_OK;
}

int gdf_mlp_grad(GdfMlp* m, const float* X, const float* y, int64_t n, float pos_weight, float* grad,
                 float* loss) {
  if (!m || !X || !y || !grad || n < 1) return mfail(GDF_ERR_ARG, "bad argument");
  const int nb = (int)((n + mlp_tile(m) - 1) / mlp_tile(m));
  int rc = mlp_ensure(m, n, nb);
  if (rc) return rc;
  if ((rc = mlp_upload_x(m, X, n))) return rc;
  MCK(cudaMemcpyAsync(m->y, y, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, m->st));
  std::vector<int> id((size_t)n);
  for (long long q = 0; q < n; ++q) id[q] = (int)q;
  MCK(cudaMemcpyAsync(m->idx, id.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, m->st));
  if ((rc = mlp_grad_launch(m, n, pos_weight, 1.f / (float)n))) return rc;
  MCK(cudaMemcpyAsync(grad, m->grad, MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, m->st));
  if (loss) MCK(cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->st));
  MCK(cudaStreamSynchronize(m->st));
  return check_err(m);
}

int gdf_mlp_train(GdfMlp* m, const float* X, const float* y, int64_t n, int32_t epochs, int32_t batch, float lr,
                  float pos_weight, int32_t seed, float* epoch_loss) {
  if (!m || !X || !y || n < 1 || epochs < 1 || batch < TB) return mfail(GDF_ERR_ARG, "bad argument");
  const int nb_max = (batch + mlp_tile(m) - 1) / mlp_tile(m);
  int rc = mlp_ensure(m, n, nb_max);
  if (rc) return rc;
  if ((rc = mlp_upload_x(m, X, n))) return rc;
  MCK(cudaMemcpyAsync(m->y, y, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, m->st));
  std::vector<int> id((size_t)n);
  for (long long q = 0; q < n; ++q) id[q] = (int)q;
  std::mt19937 rng((uint32_t)seed);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  if ((rc = fwdbwd_attr())) return rc;
  std::vector<float> lossv;
  for (int ep = 0; ep < epochs; ++ep) {
    std::shuffle(id.begin(), id.end(), rng);
    MCK(cudaMemcpyAsync(m->idx, id.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, m->st));
    MCK(cudaStreamSynchronize(m->st));   // id is reshuffled next epoch
    double ep_loss = 0.0;
    for (long long off = 0; off < n; off += batch) {
      const long long nsel = std::min<long long>(batch, n - off);
      int nb = 0;
      if ((rc = fwdbwd_launch(m, m->idx + off, nsel, pos_weight, 1.f / (float)nsel, nb))) return rc;
      k_mlp_reduce<<<(MLP_NPARAM + 255) / 256, 256, 0, m->st>>>(m->partial, nb, m->grad, m->loss_part, m->loss);
      m->adam_t += 1;
      const float c1 = 1.f - std::pow(b1, (float)m->adam_t), c2 = 1.f - std::pow(b2, (float)m->adam_t);
      k_mlp_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, m->st>>>(m->P, m->M, m->V, m->grad, lr, b1, b2, eps, c1, c2);
      if ((rc = mlp_sync(m))) return rc;
      float l = 0.f;
      MCK(cudaMemcpyAsync(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->st));
      MCK(cudaStreamSynchronize(m->st));
      ep_loss += (double)l * (double)nsel;
    }
    if (epoch_loss) epoch_loss[ep] = (float)(ep_loss / (double)n);
    if ((rc = check_err(m))) return rc;
  }
  return GDF_OK;
}

int gdf_mlp_predict(GdfMlp* m, const float* X, int64_t n, float* p) {
  if (!m || !X || !p || n < 1) return mfail(GDF_ERR_ARG, "bad argument");
  int rc = mlp_ensure(m, n, 1);
  if (rc) return rc;
  if ((rc = mlp_upload_x(m, X, n))) return rc;
  float* dp = nullptr;
  MCK(cudaMallocAsync((void**)&dp, (size_t)n * sizeof(float), m->st));
  k_mlp_predict<<<(unsigned)((n + TB - 1) / TB), MLP_THREADS, 0, m->st>>>(m->D, m->X, (int)n, dp);
  MCK(cudaGetLastError());
  MCK(cudaMemcpyAsync(p, dp, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, m->st));
  MCK(cudaFreeAsync(dp, m->st));
  MCK(cudaStreamSynchronize(m->st));
  return GDF_OK;
}

// products of the training step: 1 tcgen05 (default), 0 mma.sync
int gdf_mlp_set_products(GdfMlp* m, int32_t tcgen05) {
  if (!m || (tcgen05 != 0 && tcgen05 != 1)) return mfail(GDF_ERR_ARG, "bad argument");
  m->tc = tcgen05;
  return GDF_OK;
}

// device copy of the network for the solver library (same process)
const void* gdf_mlp_device_params(GdfMlp* m) { return m ? (const void*)m->D : nullptr; }

}  // extern "C"
