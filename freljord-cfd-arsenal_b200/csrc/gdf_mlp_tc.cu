// gdf_mlp_tc.cu -- the indicator network's training step with its five
// matrix products on the fifth-generation tensor cores (tcgen05.mma, BF16
// operands in shared memory, FP32 accumulators in tensor memory), one
// 128-sample tile per CTA.
//
// Per tile (rows = samples s, 128 per CTA; 128 threads, thread t <-> row t
// <-> tensor-memory lane t):
//   Z1 [s][n]  = X [s][k]  . W1t[n][k]      M 128, N 64, K 96   TMEM cols   0..63
//   Z2 [s][o]  = H1[s][i]  . W2t[o][i]      M 128, N 64, K 64   TMEM cols  64..127
//   dH1[s][i]  = dZ2[s][o] . W2n[i][o]      M 128, N 64, K 64   TMEM cols  64..127 (after Z2 is read)
//   dW2[i][o]  = H1t[i][s] . dZ2t[o][s]     M 128 (64 used), N 64, K 128   cols 128..191
//   dW1[k][n]  = Xt[k][s]  . dZ1t[n][s]     M 128 (90 used), N 64, K 128   cols 192..255
// Every operand sits in shared memory in the canonical no-swizzle K-major
// layout: 8-row x 16-byte core matrices, element (r, k) of a tile with K
// columns at (r/8)*(K/8)*128 + (k/8)*128 + (r%8)*16 + (k%8)*2 bytes
// (core matrices adjacent in K 128 B apart, in M/N (K/8)*128 B apart).
// One elected thread issues the products and commits them to an mbarrier;
// every wait on it is bounded (2 s of %globaltimer), after which the CTA
// sets the error word, still frees its tensor memory and returns.
//
// Numerics are those of k_mlp_fwdbwd (gdf_mlp.cu): the same BF16 roundings
// (X, W1, W2, w3, H1, dZ2, dZ1), FP32 accumulation, FP32 biases, loss and
// bias gradients; only the summation order inside the products differs.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/gdf.h"
#include "gdf_mlp.cuh"

namespace gdf {

namespace {

constexpr int TCM = 128;          // samples per CTA (UMMA M)
constexpr int TC_THREADS = 128;
constexpr int TMEM_COLS = 256;
constexpr unsigned long long WAIT_NS = 2000000000ull;

// byte sizes of the canonical tiles
constexpr int SZ_X = TCM * MLP_INP * 2;       // 24576  X   [128 s][96 k]
constexpr int SZ_XT = 128 * TCM * 2;          // 32768  Xt  [128 k (96 used)][128 s]
constexpr int SZ_W1T = MLP_H * MLP_INP * 2;   // 12288  W1t [64 n][96 k]
constexpr int SZ_W2 = MLP_H * MLP_H * 2;      //  8192  W2t [64 o][64 i], W2n [64 i][64 o]
constexpr int SZ_H1 = TCM * MLP_H * 2;        // 16384  H1  [128 s][64 i], dZ2 [128 s][64 o]
constexpr int SZ_H1T = 128 * TCM * 2;         // 32768  H1t [128 i (64 used)][128 s]
constexpr int SZ_T64 = MLP_H * TCM * 2;       // 16384  dZ2t [64 o][128 s], dZ1t [64 n][128 s]

struct TcSmem {
  alignas(128) unsigned char X[SZ_X];
  alignas(128) unsigned char Xt[SZ_XT];
  alignas(128) unsigned char W1t[SZ_W1T];
  alignas(128) unsigned char W2t[SZ_W2];
  alignas(128) unsigned char W2n[SZ_W2];
  alignas(128) unsigned char H1[SZ_H1];
  alignas(128) unsigned char H1t[SZ_H1T];
  alignas(128) unsigned char dZ2[SZ_H1];
  alignas(128) unsigned char dZ2t[SZ_T64];
  alignas(128) unsigned char dZ1t[SZ_T64];
  float b1[MLP_H], b2[MLP_H], w3[MLP_H];
  float yv[TCM], wv[TCM], g3[TCM], lossv[TCM];
  float red[3][4][MLP_H];       // per-warp column sums of db1, db2, dw3
  alignas(8) uint64_t mbar;
  uint32_t tmem_base;
};

// element offset (bytes) of (r, k) in a canonical K-major tile with K columns
__device__ __forceinline__ uint32_t cofs(int r, int k, int K) {
  return (uint32_t)((r >> 3) * (K >> 3) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}
__device__ __forceinline__ void st_bf16(unsigned char* tile, int r, int k, int K, __nv_bfloat16 v) {
  *reinterpret_cast<__nv_bfloat16*>(tile + cofs(r, k, K)) = v;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: start, leading (K) and stride (M/N)
// byte offsets, sm100 descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t sdesc(const void* p, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((smem_u32(p) & 0x3FFFFu) >> 4);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// instruction descriptor of kind::f16: BF16 A and B (K-major), FP32 D
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// bounded wait for the mbarrier phase `parity`; false when the limit passed
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const unsigned long long t0 = gtimer();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
    if (gtimer() - t0 > WAIT_NS) return false;
  }
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive FP32 columns of this thread's tensor-memory lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
      "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 32; ++q) v[q] = __uint_as_float(r[q]);
}

// one product: D (+)= A . B^T over K (multiples of 16), operands K-major
__device__ __forceinline__ void gemm(uint32_t d_tmem, const unsigned char* A, int KA, const unsigned char* B, int KB,
                                     int K, int N) {
  const uint32_t id = idesc_bf16(TCM, N);
  for (int kk = 0; kk < K / 16; ++kk) {
    const uint64_t a = sdesc(A + kk * 256, 128, (uint32_t)(KA / 8) * 128);
    const uint64_t b = sdesc(B + kk * 256, 128, (uint32_t)(KB / 8) * 128);
    umma(d_tmem, a, b, id, kk > 0 ? 1u : 0u);
  }
}

__device__ __forceinline__ float gelu_f(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_df(float x) {
  return 0.5f * (1.f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// column sums over the CTA's 128 rows of per-thread vectors (fixed order:
// lanes by a shuffle tree, then the four warps in order)
__device__ __forceinline__ void warp_colsum(float v, float* red_warp_col, int lane) {
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
  if (lane == 0) *red_warp_col = v;
}

__global__ void __launch_bounds__(TC_THREADS, 1) k_mlp_fwdbwd_tc(const MlpDev* __restrict__ D,
                                                                  const __nv_bfloat16* __restrict__ X,
                                                                  const float* __restrict__ y,
                                                                  const int* __restrict__ idx, int nsel, float pos_w,
                                                                  float inv_b, float* __restrict__ partial,
                                                                  float* __restrict__ loss_part,
                                                                  int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char tc_raw[];
  TcSmem& S = *reinterpret_cast<TcSmem*>(tc_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int base = blockIdx.x * TCM;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem_base)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // parameters and samples into the canonical tiles
  for (int q = tid; q < MLP_H * MLP_INP; q += TC_THREADS) st_bf16(S.W1t, q / MLP_INP, q % MLP_INP, MLP_INP, D->W1t[q]);
  for (int q = tid; q < MLP_H * MLP_H; q += TC_THREADS) {
    st_bf16(S.W2t, q / MLP_H, q % MLP_H, MLP_H, D->W2t[q]);
    st_bf16(S.W2n, q / MLP_H, q % MLP_H, MLP_H, D->W2n[q]);
  }
  if (tid < MLP_H) {
    S.b1[tid] = D->b1[tid];
    S.b2[tid] = D->b2[tid];
    S.w3[tid] = D->w3[tid];
  }
  {
    const int q = base + tid;
    const bool in = q < nsel;
    const long long src = in ? (long long)idx[q] * MLP_INP : 0;
    for (int k = 0; k < MLP_INP; ++k) {
      const __nv_bfloat16 v = in ? X[src + k] : __float2bfloat16_rn(0.f);
      st_bf16(S.X, tid, k, MLP_INP, v);
      st_bf16(S.Xt, k, tid, TCM, v);
    }
    for (int k = MLP_INP; k < 128; ++k) st_bf16(S.Xt, k, tid, TCM, __float2bfloat16_rn(0.f));
    for (int i = MLP_H; i < 128; ++i) st_bf16(S.H1t, i, tid, TCM, __float2bfloat16_rn(0.f));
    const float yy = in ? y[idx[q]] : 0.f;
    S.yv[tid] = yy;
    S.wv[tid] = in ? (yy > 0.5f ? pos_w : 1.f) : 0.f;
  }
  fence_async_smem();
  tc_before_sync();
  __syncthreads();
  tc_after_sync();
  const uint32_t tm = S.tmem_base;
  const uint32_t lane_off = (uint32_t)(32 * warp) << 16;
  uint32_t phase = 0;
  bool ok = true;
  // issue (thread 0), commit, wait: `ok` stays uniform over the CTA; after a
  // timeout `phase` names the product still in flight
  auto run = [&](auto issue) {
    if (!ok) return;
    if (tid == 0) {
      issue();
      umma_commit(&S.mbar);
    }
    const bool w = mbar_wait(&S.mbar, phase);
    ok = __syncthreads_and(w) != 0;
    if (ok) phase ^= 1;
    tc_after_sync();
  };
  auto handoff = [&]() {   // smem operands written, tensor-memory reads done
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
  };

  // Z1 = X . W1t^T ; H1 = gelu(Z1 + b1)
  run([&] { gemm(tm + 0, S.X, MLP_INP, S.W1t, MLP_INP, MLP_INP, MLP_H); });
  if (ok) {
    float z[32];
#pragma unroll 1
    for (int h = 0; h < 2; ++h) {
      tmem_ld32(tm + lane_off + 32 * h, z);
#pragma unroll
      for (int q = 0; q < 32; ++q) {
        const int c = 32 * h + q;
        const __nv_bfloat16 v = __float2bfloat16_rn(gelu_f(z[q] + S.b1[c]));
        st_bf16(S.H1, tid, c, MLP_H, v);
        st_bf16(S.H1t, c, tid, TCM, v);
      }
    }
  }
  handoff();

  // Z2 = H1 . W2t^T ; loss, dL/dz3, dZ2, db2, dw3
  run([&] { gemm(tm + 64, S.H1, MLP_H, S.W2t, MLP_H, MLP_H, MLP_H); });
  if (ok) {
    float z2[MLP_H];
    tmem_ld32(tm + lane_off + 64, z2);
    tmem_ld32(tm + lane_off + 96, z2 + 32);
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < MLP_H; ++c) {
      z2[c] += S.b2[c];
      s += gelu_f(z2[c]) * S.w3[c];
    }
    const float z = s + D->b3;
    const float p = 1.f / (1.f + expf(-z));
    const float yy = S.yv[tid], wt = S.wv[tid];
    const float sp_pos = fmaxf(z, 0.f) + log1pf(expf(-fabsf(z)));
    S.lossv[tid] = wt * (yy * (sp_pos - z) + (1.f - yy) * sp_pos) * inv_b;
    const float g3 = wt * (p - yy) * inv_b;
    S.g3[tid] = g3;
#pragma unroll 1
    for (int c = 0; c < MLP_H; ++c) {
      const float dz = g3 * S.w3[c] * gelu_df(z2[c]);
      const __nv_bfloat16 b = __float2bfloat16_rn(dz);
      st_bf16(S.dZ2, tid, c, MLP_H, b);
      st_bf16(S.dZ2t, c, tid, TCM, b);
      warp_colsum(dz, &S.red[1][warp][c], lane);
      warp_colsum(g3 * gelu_f(z2[c]), &S.red[2][warp][c], lane);
    }
  }
  handoff();

  // dH1 = dZ2 . W2n^T (over Z2's columns) and dW2 = H1t . dZ2t^T
  run([&] {
    gemm(tm + 64, S.dZ2, MLP_H, S.W2n, MLP_H, MLP_H, MLP_H);
    gemm(tm + 128, S.H1t, TCM, S.dZ2t, TCM, TCM, MLP_H);
  });
  float* out = partial + (long long)blockIdx.x * MLP_NPARAM;
  if (ok) {
    float dh[32], z1[32];
#pragma unroll 1
    for (int h = 0; h < 2; ++h) {
      tmem_ld32(tm + lane_off + 64 + 32 * h, dh);
      tmem_ld32(tm + lane_off + 32 * h, z1);
#pragma unroll 1
      for (int q = 0; q < 32; ++q) {
        const int c = 32 * h + q;
        const float dz = dh[q] * gelu_df(z1[q] + S.b1[c]);
        st_bf16(S.dZ1t, c, tid, TCM, __float2bfloat16_rn(dz));
        warp_colsum(dz, &S.red[0][warp][c], lane);
      }
    }
    float w2r[32];
#pragma unroll 1
    for (int h = 0; h < 2; ++h) {
      tmem_ld32(tm + lane_off + 128 + 32 * h, w2r);
      if (tid < MLP_H) {
#pragma unroll 1
        for (int q = 0; q < 32; ++q) out[MLP_OFF_W2 + tid * MLP_H + 32 * h + q] = w2r[q];
      }
    }
  }
  handoff();

  // dW1 = Xt . dZ1t^T
  run([&] { gemm(tm + 192, S.Xt, TCM, S.dZ1t, TCM, TCM, MLP_H); });
  if (ok) {
    float w1r[32];
#pragma unroll 1
    for (int h = 0; h < 2; ++h) {
      tmem_ld32(tm + lane_off + 192 + 32 * h, w1r);
      if (tid < MLP_IN) {
#pragma unroll 1
        for (int q = 0; q < 32; ++q) out[MLP_OFF_W1 + tid * MLP_H + 32 * h + q] = w1r[q];
      }
    }
  }
  tc_before_sync();
  __syncthreads();
  tc_after_sync();
  if (ok && tid < MLP_H) {
    for (int q = 0; q < 3; ++q) {
      const float v = ((S.red[q][0][tid] + S.red[q][1][tid]) + S.red[q][2][tid]) + S.red[q][3][tid];
      out[(q == 0 ? MLP_OFF_B1 : q == 1 ? MLP_OFF_B2 : MLP_OFF_W3) + tid] = v;
    }
  }
  if (tid == 0) {
    if (ok) {
      float gs = 0.f, ls = 0.f;
      for (int r = 0; r < TCM; ++r) {
        gs += S.g3[r];
        ls += S.lossv[r];
      }
      out[MLP_OFF_B3] = gs;
      loss_part[blockIdx.x] = ls;
    } else {
      atomicExch(err, 1);
      // the product still in flight: wait for it (bounded again) before
      // the tensor memory goes back
      mbar_wait(&S.mbar, phase);
    }
  }
  tc_before_sync();
  __syncthreads();
  tc_after_sync();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm), "r"(TMEM_COLS));
  }
}

}  // namespace

// Launch of the tcgen05 training tile kernel; 128 samples per CTA.
int mlp_tc_samples_per_block() { return TCM; }
size_t mlp_tc_smem_bytes() { return sizeof(TcSmem) + 1024; }

cudaError_t mlp_fwdbwd_tc_launch(const MlpDev* D, const __nv_bfloat16* X, const float* y, const int* idx, int nsel,
                                 float pos_w, float inv_b, float* partial, float* loss_part, int* err,
                                 cudaStream_t st) {
  const size_t smem = mlp_tc_smem_bytes();
  cudaError_t e = cudaFuncSetAttribute(k_mlp_fwdbwd_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int nb = (nsel + TCM - 1) / TCM;
  k_mlp_fwdbwd_tc<<<nb, TC_THREADS, smem, st>>>(D, X, y, idx, nsel, pos_w, inv_b, partial, loss_part, err);
  return cudaGetLastError();
}

}  // namespace gdf
