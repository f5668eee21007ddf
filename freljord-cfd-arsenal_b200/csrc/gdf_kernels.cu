// gdf_kernels.cu -- sm_100a kernels of the GDF P2 step and the C ABI of
// include/gdf.h.
//
// One SSP-RK3 step (RK3.f90:60-151) is:
//   k_dt_partial + k_dt_final                 calculate_dt + t update
//   3 x [ k_set_bc                            set_bc (stage 1 only; the
//                                             other stages reuse the one
//                                             that ends the previous stage)
//         k_face<0>, k_face<1>                Lh traces + Riemann (Fxhat,
//                                             Fyhat) + LhEz face Ez
//         k_vertex                            LhEz vertex Ez (2-D solvers)
//         k_cell                              Lh volume + surface integral,
//                                             fused with the RK combine
//         k_bface                             LhEz dEz + face-B combine
//         k_limit                             TVB_Limiter_P2 (+KXRCF, +pp)
//                                             fused with div_free_Balsara
//         k_set_bc ]
// Every kernel is one thread per item (face point, vertex, cell, face) and
// computes that item sequentially in the reference's order, so a build with
// --fmad=false reproduces the reference arithmetic value for value.
// All device waits are stream-ordered; no kernel spins.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/gdf.h"
#include "gdf_device.cuh"

#ifndef GDF_EXACT
#define GDF_EXACT 0
#endif
// minimum resident blocks per SM requested of the face/vertex (128-thread)
// and residual (64-thread) kernels: the register budget per thread they
// allow (65536 / (threads x blocks)); arithmetic is the same for any value.
// Faces at 4 blocks (128 registers, ~300 B spilled) ran 20% faster than at
// the unconstrained 168 registers; the residual kernel gained nothing.
#ifndef GDF_FACE_MINB
#define GDF_FACE_MINB 4
#endif
// faces through the shared-memory staged kernel (k_face_tile) or one
// thread per face point reading global memory (k_face, the default: the
// staged form measured 30% slower, blast 2048^2, same values)
#ifndef GDF_FACE_STAGED
#define GDF_FACE_STAGED 0
#endif
// face points numbered point-fastest, the five points of a face on
// adjacent lanes (face_item<DIR, true>): face kernels 3.04 / 3.21 against
// 2.83 / 2.91 ms on the blast 2048^2 (step 47.8 against 45.6 ms, same
// values), so the product keeps faces fastest
#ifndef GDF_FACE_GFAST
#define GDF_FACE_GFAST 0
#endif
// vertex kernel at 3 blocks (168 registers, no spill): timed alone a
// launch is 10% slower than at 4 blocks, but the blast 2048^2 step replayed
// from its graph is 2% shorter (45.9 against 46.9 ms, same values)
#ifndef GDF_VERTEX_MINB
#define GDF_VERTEX_MINB 3
#endif
#ifndef GDF_CELL_MINB
#define GDF_CELL_MINB 1
#endif
// k_cell reads its staged modes in pairs (GDF_CELL_PAIRS, in
// gdf_device.cuh). GDF_CELL_SHFL=1 loads every x-face flux once and passes the left
// face of a cell from the lane below by a warp shuffle: 12% slower k_cell
// (246 registers, the surface loads taken out of the interior branch), off.
#ifndef GDF_CELL_SHFL
#define GDF_CELL_SHFL 0
#endif
#ifndef GDF_LIMIT_MINB
#define GDF_LIMIT_MINB 1
#endif
// the learned indicator's stage-1 inference in its own kernel (k_infer)
// ahead of the limiter, instead of inside the 255-register limiter blocks
#ifndef GDF_INFER_APART
#define GDF_INFER_APART 1
#endif
// the learned gate's limiter in two passes as KXRCF's (gated cells listed,
// then limited over full warps); 0: one pass
#ifndef GDF_LEARNED_TWO_PASS
#define GDF_LEARNED_TWO_PASS 0
#endif


namespace gdf {

// ------------------------------------------- single-problem kernels -----
// One thread per item; a kernel whose sc is given does nothing once the
// step has stopped (sc->active == 0).
__global__ void k_set_bc(const __grid_constant__ Consts K, double* __restrict__ U, int zeroB,
                         const Scal* __restrict__ sc) {
  if (sc && !sc->active) return;
  const long long t = gtid();
  if (t >= set_bc_items(K)) return;
  set_bc_item(K, U, zeroB, t);
}

template <int DIR>
__global__ void __launch_bounds__(128, GDF_FACE_MINB) k_face(const __grid_constant__ Consts K, const double* __restrict__ U,
                                              double* __restrict__ Fh_out, double* __restrict__ Ez_out,
                                              const Scal* __restrict__ sc) {
  if (sc && !sc->active) return;
  const long long item = gtid();
  if (GDF_FACE_GFAST) {
    // the face basis of this direction in shared memory: low cell's table,
    // then the high cell's
    __shared__ double sb[2 * NG * NP];
    const double* lo = DIR == 0 ? &c_basis.phiGR[0][0] : &c_basis.phiGU[0][0];
    const double* hi = DIR == 0 ? &c_basis.phiGL[0][0] : &c_basis.phiGD[0][0];
    for (int k = threadIdx.x; k < 2 * NG * NP; k += blockDim.x) sb[k] = k < NG * NP ? lo[k] : hi[k - NG * NP];
    __syncthreads();
    if (item >= face_items<DIR>(K)) return;
    face_item<DIR, true>(K, U, Fh_out, Ez_out, item, sb);
    return;
  }
  if (item >= face_items<DIR>(K)) return;
  face_item<DIR>(K, U, Fh_out, Ez_out, item);
}

// The staged form of k_face: block (bx, by) takes faces bx*FACE_TILE ..
// of face row by at all quadrature points.
template <int DIR>
__global__ void __launch_bounds__(128, GDF_FACE_MINB) k_face_tile(const __grid_constant__ Consts K,
                                                    const double* __restrict__ U, double* __restrict__ Fh_out,
                                                    double* __restrict__ Ez_out, const Scal* __restrict__ sc) {
  __shared__ double ms[NLIVE][2 * FACE_TILE_W];
  if (sc && !sc->active) return;
  face_tile<DIR>(K, U, Fh_out, Ez_out, (int)blockIdx.x * FACE_TILE, (int)blockIdx.y, ms);
}

__global__ void __launch_bounds__(128, GDF_VERTEX_MINB) k_vertex(const __grid_constant__ Consts K, const double* __restrict__ U,
                                                double* __restrict__ EzV, const Scal* __restrict__ sc) {
  if (sc && !sc->active) return;
  const long long item = gtid();
  if (item >= K.vplane) return;
  vertex_item(K, U, EzV, item);
}

__global__ void __launch_bounds__(CELL_BS, GDF_CELL_MINB) k_cell(const __grid_constant__ Consts K, const double* __restrict__ U,
                                                  double* __restrict__ U0, double* __restrict__ UI,
                                                  const double* __restrict__ Fxh, const double* __restrict__ Fyh,
                                                  double* __restrict__ duout, const Scal* __restrict__ sc, int stage) {
  __shared__ __align__(16) double ms[NLIVE * CELL_BS];
  if (sc && !sc->active) return;
  const long long item = gtid();
  if (GDF_CELL_SHFL) {
    // every lane takes part in the x-face shuffles, past the end too
    cell_item<true, GDF_CELL_PAIRS != 0>(K, U, U0, UI, Fxh, Fyh, duout, sc, stage, item, ms, item < K.plane);
    return;
  }
  if (item >= K.plane) return;
  cell_item<false, GDF_CELL_PAIRS != 0>(K, U, U0, UI, Fxh, Fyh, duout, sc, stage, item, ms);
}

__global__ void __launch_bounds__(128) k_bface(const __grid_constant__ Consts K, const double* __restrict__ EzRL,
                                               const double* __restrict__ EzUD, const double* __restrict__ EzV,
                                               double* __restrict__ BX, double* __restrict__ BX0,
                                               double* __restrict__ BXI, double* __restrict__ BY,
                                               double* __restrict__ BY0, double* __restrict__ BYI,
                                               double* __restrict__ dez1, double* __restrict__ dez2,
                                               const Scal* __restrict__ sc, int stage) {
  if (sc && !sc->active) return;
  const long long item = gtid();
  if (item >= K.fxplane + K.fyplane) return;
  bface_item(K, EzRL, EzUD, EzV, BX, BX0, BXI, BY, BY0, BYI, dez1, dez2, sc, stage, item);
}

__global__ void k_qmodes(const __grid_constant__ Consts K, const double* __restrict__ S, float* __restrict__ QM) {
  const long long c = gtid();
  if (c >= K.plane) return;
  qmodes_item(K, S, QM, c);
}

__global__ void k_features(const __grid_constant__ Consts K, const float* __restrict__ QM, float* __restrict__ X) {
  const long long item = gtid();
  if (item >= (long long)K.nx * K.ny) return;
  const int i = (int)(item % K.nx) + 1, j = (int)(item / K.nx) + 1;
  float f[NFEAT];
  gather_features(K, QM, i + (long long)K.nx2 * j, f);
#pragma unroll
  for (int k = 0; k < NFEAT; ++k) X[item * NFEAT + k] = f[k];
}

// The learned indicator of every interior cell ahead of the stage-1 limiter:
// resident blocks stage the BF16 weights once and walk the LIM_BS-cell
// tiles of the grid (features gathered from QM, the two tensor-core
// products, the sigmoid), storing each cell's probability in pnet. A tile
// computes what the limiter block with inference computes for the same
// cells (same features, roundings and product order per row), so the
// stored probabilities are those of k_limit<LIM_INFER>, at the occupancy of
// a 128-register kernel instead of the FP64 limiter's 255 registers.
__global__ void __launch_bounds__(LIM_BS) k_infer(const __grid_constant__ Consts K, const MlpDev* __restrict__ net,
                                                     const float* __restrict__ QM, float* __restrict__ pnet,
                                                     const Scal* __restrict__ gate_sc) {
  extern __shared__ __align__(16) unsigned char lsm[];
  if (gate_sc && !gate_sc->active) return;
  __nv_bfloat16* Xs = reinterpret_cast<__nv_bfloat16*>(lsm);
  __nv_bfloat16* W1t = Xs + LIM_BS * MLP_LDX;
  __nv_bfloat16* W2t = W1t + MLP_H * MLP_LDX;
  __nv_bfloat16* H1 = W2t + MLP_H * MLP_LDH;
  float* zz = reinterpret_cast<float*>(H1 + LIM_BS * MLP_LDH);
  const int tid = threadIdx.x;
  const uint4* g1 = reinterpret_cast<const uint4*>(net->W1t);
  const uint4* g2 = reinterpret_cast<const uint4*>(net->W2t);
  for (int k = tid; k < MLP_H * (MLP_INP / 8); k += LIM_BS) {
    const int r = k / (MLP_INP / 8), q = k % (MLP_INP / 8);
    *reinterpret_cast<uint4*>(W1t + r * MLP_LDX + 8 * q) = g1[k];
  }
  for (int k = tid; k < MLP_H * (MLP_H / 8); k += LIM_BS) {
    const int r = k / (MLP_H / 8), q = k % (MLP_H / 8);
    *reinterpret_cast<uint4*>(W2t + r * MLP_LDH + 8 * q) = g2[k];
  }
  const long long ncell = (long long)K.nx * K.ny;
  for (long long base = (long long)blockIdx.x * LIM_BS; base < ncell; base += (long long)gridDim.x * LIM_BS) {
    const long long item = base + tid;
    const bool valid = item < ncell;
    float f[MLP_INP];
    if (valid) {
      const int i = (int)(item % K.nx) + 1, j = (int)(item / K.nx) + 1;
      gather_features(K, QM, i + (long long)K.nx2 * j, f);
    } else {
#pragma unroll
      for (int k = 0; k < NFEAT; ++k) f[k] = 0.f;
    }
#pragma unroll
    for (int k = NFEAT; k < MLP_INP; ++k) f[k] = 0.f;
#pragma unroll
    for (int q = 0; q < MLP_INP / 8; ++q) {
      __nv_bfloat162 a = __floats2bfloat162_rn(f[8 * q], f[8 * q + 1]);
      __nv_bfloat162 b = __floats2bfloat162_rn(f[8 * q + 2], f[8 * q + 3]);
      __nv_bfloat162 cc = __floats2bfloat162_rn(f[8 * q + 4], f[8 * q + 5]);
      __nv_bfloat162 d = __floats2bfloat162_rn(f[8 * q + 6], f[8 * q + 7]);
      uint4 v;
      v.x = *reinterpret_cast<uint32_t*>(&a);
      v.y = *reinterpret_cast<uint32_t*>(&b);
      v.z = *reinterpret_cast<uint32_t*>(&cc);
      v.w = *reinterpret_cast<uint32_t*>(&d);
      *reinterpret_cast<uint4*>(Xs + tid * MLP_LDX + 8 * q) = v;
    }
    // the weights (first tile) and this tile's rows are in place
    __syncthreads();
    // ends with a barrier: zz holds the tile's logits, Xs and H1 are free
    mlp_infer_tiles(Xs, W1t, W2t, net->b1, net->b2, net->w3, net->b3, H1, zz, LIM_BS);
    if (valid) pnet[item] = 1.f / (1.f + expf(-zz[tid]));
  }
}

template <int LM, bool COMPACT>
__global__ void __launch_bounds__(LIM_BS, GDF_LIMIT_MINB) k_limit(const __grid_constant__ Consts K, const double* __restrict__ S,
                                                  double* __restrict__ D, const double* __restrict__ BX,
                                                  const double* __restrict__ BY, int32_t* __restrict__ flags,
                                                  int32_t* __restrict__ trouble, int stage, int divfree,
                                                  const Scal* __restrict__ gate_sc, Scal* __restrict__ sc,
                                                  const MlpDev* __restrict__ net, const float* __restrict__ QM,
                                                  float* __restrict__ pnet, float t_lo, float t_hi,
                                                  int32_t* __restrict__ list, int32_t* __restrict__ count) {
  extern __shared__ __align__(16) unsigned char lsm[];
  if (gate_sc && !gate_sc->active) return;
  limit_item<LM, COMPACT>(K, S, D, BX, BY, flags, trouble, stage, divfree, sc, net, QM, pnet, t_lo, t_hi, gtid(), lsm,
                          list, count);
}

// The cells k_limit<LM, true> deferred, one per thread (the grid covers
// every interior cell; threads past the count return).
__global__ void __launch_bounds__(LIM_BS, GDF_LIMIT_MINB) k_limit_tvb(const __grid_constant__ Consts K,
                                                  const double* __restrict__ S, double* __restrict__ D,
                                                  const double* __restrict__ BX, const double* __restrict__ BY,
                                                  int32_t* __restrict__ flags, int stage, int divfree,
                                                  const Scal* __restrict__ gate_sc, Scal* __restrict__ sc,
                                                  const int32_t* __restrict__ list,
                                                  const int32_t* __restrict__ count) {
  if (gate_sc && !gate_sc->active) return;
  const long long t = gtid();
  if (t >= *count) return;
  limit_tvb_item(K, S, D, BX, BY, flags, stage, divfree, sc, list[t]);
}

__global__ void k_faceb_limit(const __grid_constant__ Consts K, const double* __restrict__ S,
                              double* __restrict__ BX, double* __restrict__ BY, const Scal* __restrict__ sc) {
  if (sc && !sc->active) return;
  faceb_item(K, S, BX, BY, gtid());
}

__global__ void k_divfree(const __grid_constant__ Consts K, double* __restrict__ D, const double* __restrict__ BX,
                          const double* __restrict__ BY, const Scal* __restrict__ sc) {
  if (sc && !sc->active) return;
  const long long item = gtid();
  if (item >= (long long)K.nx * K.ny) return;
  divfree_item(K, D, BX, BY, item);
}

// The step state in its smallest form (gdf_upload_state/gdf_download_state):
// modes 1-6 of the six variables a step evolves in the cell (rho, rho u,
// rho v, rho w, E, Bz) over the interior cells, packed as
// cells[i + nx*(j + ny*(d + 6*v))]. The cell Bx/By modes are not part of
// it: div_free_Balsara rebuilds them from the face fields at the end of
// every stage, and the ghosts are set_bc of the interior.
__device__ __forceinline__ long long state_slot(const Consts& K, long long item) {
  const long long ncell = (long long)K.nx * K.ny;
  const int s = (int)(item / ncell);
  const long long q = item - s * ncell;
  const int i = (int)(q % K.nx) + 1, j = (int)(q / K.nx) + 1;
  const int d = s % 6, v = s / 6;
  const int n = v < 5 ? v : 7;
  return i + (long long)K.nx2 * j + K.plane * (d + 10 * n);
}
__global__ void k_pack_state(const __grid_constant__ Consts K, const double* __restrict__ U,
                             double* __restrict__ cells) {
  const long long item = gtid();
  if (item >= 36LL * K.nx * K.ny) return;
  cells[item] = U[state_slot(K, item)];
}
__global__ void k_unpack_state(const __grid_constant__ Consts K, const double* __restrict__ cells,
                               double* __restrict__ U) {
  const long long item = gtid();
  if (item >= 36LL * K.nx * K.ny) return;
  U[state_slot(K, item)] = cells[item];
}

// calculate_dt.f90:11-25: per-block maxima of |u_n +- c_f| over the cell
// averages, then one block folds them and advances t (RK3.f90:60-71).
__global__ void __launch_bounds__(DT_BS) k_dt_partial(const __grid_constant__ Consts K, const double* __restrict__ U,
                                                      double* __restrict__ part, Scal* __restrict__ sc) {
  __shared__ double sx[DT_BS], sy[DT_BS];
  const long long item = gtid();
  double ax = 0.0, ay = 0.0;
  if (item < (long long)K.nx * K.ny) dt_cell_speeds(K, U, item, ax, ay, sc);
  sx[threadIdx.x] = ax;
  sy[threadIdx.x] = ay;
  __syncthreads();
  for (int s = DT_BS / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      sx[threadIdx.x] = max_ign_nan(sx[threadIdx.x], sx[threadIdx.x + s]);
      sy[threadIdx.x] = max_ign_nan(sy[threadIdx.x], sy[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = sx[0];
    part[2 * blockIdx.x + 1] = sy[0];
  }
}

// mode 0: gdf_dt (dt only); mode 1: a time step (t update, active flag)
__global__ void __launch_bounds__(DT_BS) k_dt_final(const __grid_constant__ Consts K, const double* __restrict__ part,
                                                    int nblocks, Scal* __restrict__ sc, int mode) {
  __shared__ double sx[DT_BS], sy[DT_BS];
  double ax = 0.0, ay = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += DT_BS) {
    ax = max_ign_nan(ax, part[2 * b]);
    ay = max_ign_nan(ay, part[2 * b + 1]);
  }
  sx[threadIdx.x] = ax;
  sy[threadIdx.x] = ay;
  __syncthreads();
  for (int s = DT_BS / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      sx[threadIdx.x] = max_ign_nan(sx[threadIdx.x], sx[threadIdx.x + s]);
      sy[threadIdx.x] = max_ign_nan(sy[threadIdx.x], sy[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) dt_advance(K, sx[0], sy[0], sc, mode);
}

// ------------------------------------------------------ diagnostics -------
// calculate_umax.f90, calculate_totaldiv.f90, calculate_pmin.f90, and the
// number of flagged cells. Per-block partials, folded by k_diag_final.
__global__ void __launch_bounds__(DT_BS) k_diag_partial(const __grid_constant__ Consts K, const double* __restrict__ U,
                                                        const int32_t* __restrict__ flags, double* __restrict__ part) {
  __shared__ double s_um[DT_BS], s_td[DT_BS], s_pm[DT_BS], s_nt[DT_BS];
  const long long item = gtid();
  double um = 0.0, td = 0.0, pm = 1000000.0, nt = 0.0;
  if (item < (long long)K.nx * K.ny) {
    const int i = (int)(item % K.nx) + 1;
    const int j = (int)(item / K.nx) + 1;
    const long long c = i + (long long)K.nx2 * j;
    double m[NE][NP];
#pragma unroll
    for (int n = 0; n < NE; ++n)
#pragma unroll
      for (int d = 0; d < NP; ++d) m[n][d] = live_mode(n, d) ? U[c + K.plane * (d + 10 * n)] : 0.0;
    if (K.umax_all) {
#pragma unroll
      for (int n = 0; n < NE; ++n)
        if (fabs(m[n][0]) > um) um = fabs(m[n][0]);
    } else {
      um = fabs(m[0][0]);
    }
#pragma unroll 1
    for (int a = 0; a < NG; ++a)
#pragma unroll 1
      for (int b = 0; b < NG; ++b) {
        double gd = 0.0;
#pragma unroll
        for (int d = 0; d < NP; ++d) gd = gd + m[5][d] * K.phix[a][b][d] + m[6][d] * K.phiy[a][b][d];
        td = td + K.w[a] * K.w[b] * sq(gd);
        double q[NE];
#pragma unroll
        for (int n = 0; n < NE; ++n) {
          double acc = 0.0;
#pragma unroll
          for (int d = 0; d < NP; ++d)
            if (live_mode(n, d)) acc = acc + m[n][d] * K.phiG[a][b][d];
          q[n] = acc;
        }
        const double p1 = pressure(K.P.gamma, q);
        if (p1 < pm) pm = p1;
      }
    if (flags && flags[item] != 0) nt = 1.0;
  }
  s_um[threadIdx.x] = um; s_td[threadIdx.x] = td; s_pm[threadIdx.x] = pm; s_nt[threadIdx.x] = nt;
  __syncthreads();
  for (int s = DT_BS / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      s_um[threadIdx.x] = fmax(s_um[threadIdx.x], s_um[threadIdx.x + s]);
      s_td[threadIdx.x] = s_td[threadIdx.x] + s_td[threadIdx.x + s];
      s_pm[threadIdx.x] = fmin(s_pm[threadIdx.x], s_pm[threadIdx.x + s]);
      s_nt[threadIdx.x] = s_nt[threadIdx.x] + s_nt[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[4 * blockIdx.x] = s_um[0];
    part[4 * blockIdx.x + 1] = s_td[0];
    part[4 * blockIdx.x + 2] = s_pm[0];
    part[4 * blockIdx.x + 3] = s_nt[0];
  }
}

__global__ void k_diag_final(const __grid_constant__ Consts K, const double* __restrict__ part, int nblocks,
                             Scal* __restrict__ sc) {
  if (threadIdx.x != 0) return;
  double um = 0.0, td = 0.0, pm = 1000000.0, nt = 0.0;
  for (int b = 0; b < nblocks; ++b) {
    um = fmax(um, part[4 * b]);
    td = td + part[4 * b + 1];
    pm = fmin(pm, part[4 * b + 2]);
    nt = nt + part[4 * b + 3];
  }
  sc->umax = um;
  sc->totaldiv = sqrt(td * K.hx1 * K.hy1);
  sc->pmin = pm;
  sc->troubled = (long long)nt;
}

}  // namespace gdf

// =====================================================================
// Host side: handle, constants, C ABI.
// =====================================================================
using namespace gdf;

static thread_local std::string g_err;

static int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CK(call)                                                                       \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess) return fail(GDF_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
  } while (0)

struct GdfHandle {
  GdfConfig cfg{};
  Consts K{};
  cudaStream_t st = nullptr;
  double *U = nullptr, *U0 = nullptr, *UI = nullptr, *UT = nullptr;
  double *BX = nullptr, *BX0 = nullptr, *BXI = nullptr, *BY = nullptr, *BY0 = nullptr, *BYI = nullptr;
  double *Fxh = nullptr, *Fyh = nullptr, *EzRL = nullptr, *EzUD = nullptr, *EzV = nullptr;
  double *part = nullptr;
  float* QM = nullptr;       // learned-indicator feature modes (18 per cell)
  float* pnet = nullptr;     // learned-indicator probability per interior cell (this step)
  MlpDev* net = nullptr;     // learned-indicator network (device copy)
  float t_lo = 0.5f, t_hi = 0.5f;
  int32_t *flags = nullptr, *trouble = nullptr;
  int32_t *lim_list = nullptr, *lim_count = nullptr;  // cells the limiter's first pass deferred
  Scal* sc = nullptr;
  Scal* sc_host = nullptr;  // pinned mirror
  int uploaded = 0;
  int64_t launches = 0;
  int64_t step_launches = 0;
  int dt_blocks = 0;
  int sms = 0;  // SMs of the handle's device (grid of the resident inference blocks)
  cudaGraphExec_t graph = nullptr;
  // per-kernel timing (gdf_profile): events around every launch when set
  int prof = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double prof_ms[GDF_KERNEL_KINDS] = {0};
  int64_t prof_n[GDF_KERNEL_KINDS] = {0};
};

// Record a launch: when profiling, bracket it with events on the handle's
// stream and accumulate its device time under its kind.
template <class F>
static int run_kernel(GdfHandle* h, int kind, F&& launch) {
  if (h->prof) cudaEventRecord(h->ev0, h->st);
  launch();
  h->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(GDF_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  if (h->prof) {
    cudaEventRecord(h->ev1, h->st);
    cudaEventSynchronize(h->ev1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->prof_ms[kind] += ms;
    h->prof_n[kind] += 1;
  }
  return GDF_OK;
}

static void build_consts(const GdfConfig& c, Consts& K) {
  std::memset(&K, 0, sizeof(K));
  K.nx = c.nx; K.ny = c.ny; K.nx2 = c.nx + 2; K.ny2 = c.ny + 2;
  K.plane = (long long)K.nx2 * K.ny2;
  K.fxplane = (long long)(c.nx + 1) * c.ny;
  K.fyplane = (long long)c.nx * (c.ny + 1);
  K.vplane = (long long)(c.nx + 1) * (c.ny + 1);
  // init_data.f90:21-24
  K.hx = (c.xb - c.xa) / c.nx;
  K.hy = (c.yb - c.ya) / c.ny;
  K.hx1 = 0.5 * K.hx;
  K.hy1 = 0.5 * K.hy;
  K.cxs = 0.5 / K.hx;
  K.cys = 0.5 / K.hy;
  K.Mh2x = c.tvb_m * (K.hx * K.hx);
  K.Mh2y = c.tvb_m * (K.hy * K.hy);
  K.Mh2x_b = c.tvb_m * (K.hy * K.hy);
  K.Mh2y_b = c.tvb_m * (K.hx * K.hx);
  K.rxy = K.hx / K.hy;
  K.ryx = K.hy / K.hx;
  K.tvb_slope = c.tvb_slope;
  K.cfl = c.cfl;
  K.ck = c.kxrcf_ck;
  K.pow_hxhy = std::pow(K.hx * K.hy, 0.25 * (2 + 1));  // KXRCF_Detector.f90:98
  K.bc_r = c.bc_r; K.bc_l = c.bc_l; K.bc_u = c.bc_u; K.bc_d = c.bc_d;
  // TVB_Limiter_P1.f90:113-164 applies the face-B minmod whatever the switch
  K.pp = c.pp_limiter; K.faceb = (c.faceb_limiter || c.tvb_p1) ? 1 : 0; K.ez_fhat = c.ez_face_fhat;
  K.tvb_p1 = c.tvb_p1;
  K.eig_y_zero_w = c.eig_y_zero_w; K.detector = c.detector; K.sticky = c.kxrcf_sticky;
  K.dt_floor_stop = c.dt_floor_stop; K.umax_all = c.umax_all_vars;
  K.P.gamma = c.gamma;
  K.P.gamma1 = c.gamma - 1;
  K.P.gflux = c.gamma_flux;
  K.P.hlld_eps = c.hlld_eps;
  K.P.flux = c.flux_type;
  K.P.kml_w = c.kml_w_term;
  K.P.eig_p_typo = c.eig_p_typo;
  K.P.eig_identity = c.eig_identity;
  // get_GLP.f90:38-56 (5-point branch)
  const double lam[NG] = {-0.9061798459386639927976269, -0.5384693101056830910363144, 0,
                          0.5384693101056830910363144, 0.9061798459386639927976269};
  const double wt[NG] = {0.2369268850561890875142640, 0.4786286704993664680412915, 0.5688888888888888888888889,
                         0.4786286704993664680412915, 0.2369268850561890875142640};
  const double lamL[NG] = {-1, -0.6546536707079771437983, 0, 0.654653670707977143798, 1};
  const double hx1 = K.hx1, hy1 = K.hy1;
  const double c13 = 1.0 / 3.0, c23 = 2.0 / 3.0, c25 = 2.0 / 5.0, c35 = 3.0 / 5.0;
  for (int a = 0; a < NG; ++a) { K.w[a] = wt[a]; K.lam[a] = lam[a]; }
  // get_basis.f90: Legendre tensor basis values and derivatives
  auto P2 = [&](double x) { return x * x - c13; };
  auto P3 = [&](double x) { return x * x * x - 3.0 * x / 5.0; };
  for (int a = 0; a < NG; ++a)
    for (int b = 0; b < NG; ++b) {
      const double li = lam[a], lj = lam[b], Li = lamL[a], Lj = lamL[b];
      double* G = K.phiG[a][b];
      double* X = K.phix[a][b];
      double* Y = K.phiy[a][b];
      double* G1 = K.phiGLL[0][a][b];
      double* G2 = K.phiGLL[1][a][b];
      G[0] = 1; G1[0] = 1; G2[0] = 1; X[0] = 0; Y[0] = 0;
      G[1] = li; G1[1] = Li; G2[1] = li; X[1] = 1.0 / hx1; Y[1] = 0;
      G[2] = lj; G1[2] = lj; G2[2] = Lj; X[2] = 0; Y[2] = 1.0 / hy1;
      G[3] = P2(li); G1[3] = P2(Li); G2[3] = P2(li); X[3] = 2.0 * li / hx1; Y[3] = 0;
      G[4] = li * lj; G1[4] = Li * lj; G2[4] = li * Lj; X[4] = lj / hx1; Y[4] = li / hy1;
      G[5] = P2(lj); G1[5] = P2(lj); G2[5] = P2(Lj); X[5] = 0; Y[5] = 2.0 * lj / hy1;
      G[6] = P3(li); G1[6] = P3(Li); G2[6] = P3(li); X[6] = (3 * (li * li) - c35) / hx1; Y[6] = 0;
      G[7] = P2(li) * lj; G1[7] = P2(Li) * lj; G2[7] = P2(li) * Lj;
      X[7] = 2.0 * li * lj / hx1; Y[7] = P2(li) / hy1;
      G[8] = li * P2(lj); G1[8] = Li * P2(lj); G2[8] = li * P2(Lj);
      X[8] = P2(lj) / hx1; Y[8] = 2.0 * li * lj / hy1;
      G[9] = P3(lj); G1[9] = P3(lj); G2[9] = P3(Lj); X[9] = 0; Y[9] = (3 * (lj * lj) - c35) / hy1;
    }
  for (int d = 0; d < NP; ++d) {
    double mx = 0.0;
    for (int s2 = 0; s2 < 2; ++s2)
      for (int a = 0; a < NG; ++a)
        for (int b = 0; b < NG; ++b) mx = std::max(mx, std::fabs(K.phiGLL[s2][a][b][d]));
    K.ppM[d] = mx;
  }
  for (int g = 0; g < NG; ++g) {
    const double l = lam[g];
    const double R[NP] = {1, 1, l, c23, l, P2(l), c25, c23 * l, P2(l), P3(l)};
    const double Lf[NP] = {1, -1, l, c23, -l, P2(l), -c25, c23 * l, -P2(l), P3(l)};
    const double Uf[NP] = {1, l, 1, P2(l), l, c23, P3(l), P2(l), l * c23, c25};
    const double Df[NP] = {1, l, -1, P2(l), -l, c23, P3(l), -P2(l), l * c23, -c25};
    for (int d = 0; d < NP; ++d) {
      K.phiGR[g][d] = R[d]; K.phiGL[g][d] = Lf[d]; K.phiGU[g][d] = Uf[d]; K.phiGD[g][d] = Df[d];
    }
    K.EzxG[g][0] = 0; K.EzxG[g][1] = 1 / hx1; K.EzxG[g][2] = 2 * l / hx1;
    K.EzyG[g][0] = 0; K.EzyG[g][1] = 1 / hy1; K.EzyG[g][2] = 2 * l / hy1;
  }
  const double ru[NP] = {1, 1, 1, c23, 1, c23, c25, c23, c23, c25};
  const double lu[NP] = {1, -1, 1, c23, -1, c23, -c25, c23, -c23, c25};
  const double rd[NP] = {1, 1, -1, c23, -1, c23, c25, -c23, c23, -c25};
  const double ld[NP] = {1, -1, -1, c23, 1, c23, -c25, -c23, -c23, -c25};
  const double mm[NP] = {1, 1.0 / 3.0, 1.0 / 3.0, 4.0 / 45.0, 1.0 / 9.0, 4.0 / 45.0,
                         4.0 / 175.0, 4.0 / 135.0, 4.0 / 135.0, 4.0 / 175.0};
  for (int d = 0; d < NP; ++d) {
    K.phiRU[d] = ru[d]; K.phiLU[d] = lu[d]; K.phiRD[d] = rd[d]; K.phiLD[d] = ld[d]; K.mm[d] = mm[d];
  }
  K.mmE[0] = 1; K.mmE[1] = 1.0 / 3.0; K.mmE[2] = 4.0 / 45.0;
  K.EzR[0] = 1; K.EzR[1] = 1; K.EzR[2] = c23;
  K.EzL[0] = 1; K.EzL[1] = -1; K.EzL[2] = c23;
  for (int d = 0; d < 3; ++d) { K.EzU[d] = K.EzR[d]; K.EzD[d] = K.EzL[d]; }
}

static int check_config(const GdfConfig* c) {
  if (!c) return fail(GDF_ERR_ARG, "null config");
  if (c->nx < 2 || c->ny < 2) return fail(GDF_ERR_ARG, "nx and ny must be >= 2");
  if ((long long)c->nx * c->ny > (1LL << 31)) return fail(GDF_ERR_ARG, "grid too large");
  if (!(c->xb > c->xa) || !(c->yb > c->ya)) return fail(GDF_ERR_ARG, "empty domain");
  const int bcs[4] = {c->bc_r, c->bc_l, c->bc_u, c->bc_d};
  for (int b : bcs)
    if (b != GDF_BC_PERIODIC && b != GDF_BC_OUTFLOW) return fail(GDF_ERR_ARG, "boundary must be 1 or 2");
  if (c->flux_type < 1 || c->flux_type > 4) return fail(GDF_ERR_ARG, "flux_type must be 1..4");
  if (!(c->gamma > 1.0) || !(c->gamma_flux > 1.0)) return fail(GDF_ERR_ARG, "gamma must be > 1");
  if (!(c->cfl > 0.0)) return fail(GDF_ERR_ARG, "cfl must be > 0");
  if (c->detector != GDF_DETECT_ALL && c->detector != GDF_DETECT_KXRCF && c->detector != GDF_DETECT_LEARNED)
    return fail(GDF_ERR_ARG, "unknown detector");
  return GDF_OK;
}

namespace gdf {
// gdf_init.cu: the device projection of the initial data
int init_data_device(const GdfConfig& cfg, int problem, const double* params, double* U, double* BX, double* BY,
                     cudaStream_t st, std::string& err);
// the message gdf_last_error() returns, for the host-only parts of the ABI
int set_last_error(int code, const char* msg) { return fail(code, msg); }
void consts_for(const GdfConfig& c, Consts& K) { build_consts(c, K); }
void basis_of(const Consts& K, Basis& B) {
  std::memcpy(B.w, K.w, sizeof(B.w));
  std::memcpy(B.lam, K.lam, sizeof(B.lam));
  std::memcpy(B.phiG, K.phiG, sizeof(B.phiG));
  std::memcpy(B.phiGLL, K.phiGLL, sizeof(B.phiGLL));
  std::memcpy(B.ppM, K.ppM, sizeof(B.ppM));
  std::memcpy(B.phiGR, K.phiGR, sizeof(B.phiGR));
  std::memcpy(B.phiGL, K.phiGL, sizeof(B.phiGL));
  std::memcpy(B.phiGU, K.phiGU, sizeof(B.phiGU));
  std::memcpy(B.phiGD, K.phiGD, sizeof(B.phiGD));
  std::memcpy(B.phiRU, K.phiRU, sizeof(B.phiRU));
  std::memcpy(B.phiLU, K.phiLU, sizeof(B.phiLU));
  std::memcpy(B.phiRD, K.phiRD, sizeof(B.phiRD));
  std::memcpy(B.phiLD, K.phiLD, sizeof(B.phiLD));
  std::memcpy(B.mm, K.mm, sizeof(B.mm));
  std::memcpy(B.mmE, K.mmE, sizeof(B.mmE));
  std::memcpy(B.EzR, K.EzR, sizeof(B.EzR));
  std::memcpy(B.EzL, K.EzL, sizeof(B.EzL));
  std::memcpy(B.EzU, K.EzU, sizeof(B.EzU));
  std::memcpy(B.EzD, K.EzD, sizeof(B.EzD));
}
int config_error(const GdfConfig* c, std::string& msg) {
  const int rc = check_config(c);
  if (rc) msg = g_err;
  return rc;
}
}  // namespace gdf

static inline unsigned nblk(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

#define LAUNCH_CHECK(h)                                                                   \
  do {                                                                                    \
    cudaError_t e_ = cudaGetLastError();                                                  \
    if (e_ != cudaSuccess) return fail(GDF_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e_)); \
  } while (0)

static int launch_set_bc(GdfHandle* h, double* U, int zeroB, const Scal* sc) {
  const long long n = (2LL * (h->K.nx + 2) + 2LL * h->K.ny) * NLIVE;
  return run_kernel(h, GDF_K_SET_BC, [&] { k_set_bc<<<nblk(n, 256), 256, 0, h->st>>>(h->K, U, zeroB, sc); });
}

// Lh traces/Riemann (Fxhat, Fyhat, EzRL, EzUD) and LhEz vertex Ez on U
static int launch_faces(GdfHandle* h, const double* U, const Scal* sc) {
  const Consts& K = h->K;
  const long long nfx = (long long)(K.nx + 1) * NG * K.ny;
  const long long nfy = (long long)K.nx * NG * (K.ny + 1);
  int rc;
  if (GDF_FACE_STAGED && K.ny + 1 <= 65535) {
    const dim3 gx((unsigned)nblk(K.nx + 1, FACE_TILE), (unsigned)K.ny), gy((unsigned)nblk(K.nx, FACE_TILE), (unsigned)(K.ny + 1));
    rc = run_kernel(h, GDF_K_FACE_X, [&] { k_face_tile<0><<<gx, 128, 0, h->st>>>(K, U, h->Fxh, h->EzRL, sc); });
    if (!rc) rc = run_kernel(h, GDF_K_FACE_Y, [&] { k_face_tile<1><<<gy, 128, 0, h->st>>>(K, U, h->Fyh, h->EzUD, sc); });
  } else {
    rc = run_kernel(h, GDF_K_FACE_X, [&] { k_face<0><<<nblk(nfx, 128), 128, 0, h->st>>>(K, U, h->Fxh, h->EzRL, sc); });
    if (!rc) rc = run_kernel(h, GDF_K_FACE_Y, [&] { k_face<1><<<nblk(nfy, 128), 128, 0, h->st>>>(K, U, h->Fyh, h->EzUD, sc); });
  }
  if (!rc) rc = run_kernel(h, GDF_K_VERTEX, [&] { k_vertex<<<nblk(K.vplane, 128), 128, 0, h->st>>>(K, U, h->EzV, sc); });
  return rc;
}

static int launch_dt(GdfHandle* h, const double* U, int mode) {
  int rc = run_kernel(h, GDF_K_DT, [&] { k_dt_partial<<<h->dt_blocks, DT_BS, 0, h->st>>>(h->K, U, h->part, h->sc); });
  if (!rc) rc = run_kernel(h, GDF_K_DT, [&] { k_dt_final<<<1, DT_BS, 0, h->st>>>(h->K, h->part, h->dt_blocks, h->sc, mode); });
  return rc;
}

static int launch_limit(GdfHandle* h, const double* S, double* D, int stage, const Scal* sc_gate) {
  const Consts& K = h->K;
  const long long ncell = (long long)K.nx * K.ny;
  const int fused_divfree = K.faceb ? 0 : 1;
  size_t smem = 0;
  // the network runs at the first stage of a step (and at the start-up
  // limiting); stages 2 and 3 reuse its probabilities
  const int infer = stage <= 1 ? 1 : 0;
  if (K.detector == GDF_DETECT_LEARNED) {
    if (!h->net || !h->QM) return fail(GDF_ERR_STATE, "detector GDF_DETECT_LEARNED needs gdf_set_indicator first");
    if (infer) {
      int rq = run_kernel(h, GDF_K_LIMIT, [&] { k_qmodes<<<nblk(K.plane, 128), 128, 0, h->st>>>(K, S, h->QM); });
      if (!rq && GDF_INFER_APART) {
        const long long tiles = (long long)nblk(ncell, LIM_BS);
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_infer, LIM_BS, LIMIT_SMEM_LEARNED) !=
                cudaSuccess ||
            per_sm <= 0) {
          cudaGetLastError();
          per_sm = 1;
        }
        const unsigned nb = (unsigned)std::min<long long>(tiles, (long long)per_sm * h->sms);
        rq = run_kernel(h, GDF_K_LIMIT, [&] {
          k_infer<<<nb, LIM_BS, LIMIT_SMEM_LEARNED, h->st>>>(K, h->net, h->QM, h->pnet, sc_gate);
        });
      }
      if (rq) return rq;
      smem = LIMIT_SMEM_LEARNED;
    }
  }
  // KXRCF: the gated cells go to a second pass over full warps (the sticky
  // flags leave mixed warps for most of a run: the developed 512^2 rotor's
  // limiter 1.8x faster). The learned gate stays in one pass by default
  // (GDF_LEARNED_TWO_PASS): two passes are faster while few cells are gated
  // (learned blast 512^2, steps 1-1200, 5.41 against 5.67 ms per step;
  // blast 2048^2 45.4 against 45.6 ms) but slower once most are (the whole
  // 512^2 blast run to t = 0.01, 87% gated late: 7.86 against 7.13 ms per
  // step, two bench runs whose plain steps took 7.15 and 7.14 ms), same
  // values either way.
  const bool compact = K.detector == GDF_DETECT_KXRCF ||
                       (GDF_LEARNED_TWO_PASS && K.detector == GDF_DETECT_LEARNED && (GDF_INFER_APART || !infer));
  if (compact) CK(cudaMemsetAsync(h->lim_count, 0, sizeof(int32_t), h->st));
  int32_t *L = h->lim_list, *N = h->lim_count;
  int rc0 = run_kernel(h, GDF_K_LIMIT, [&] {
    const unsigned nb = nblk(ncell, LIM_BS);
    if (K.detector == GDF_DETECT_LEARNED && infer && !GDF_INFER_APART)
      k_limit<LIM_INFER, false><<<nb, LIM_BS, smem, h->st>>>(K, S, D, h->BX, h->BY, h->flags, h->trouble, stage,
                                                             fused_divfree, sc_gate, h->sc, h->net, h->QM, h->pnet,
                                                             h->t_lo, h->t_hi, nullptr, nullptr);
    else if (K.detector == GDF_DETECT_LEARNED && compact)
      k_limit<LIM_PNET, true><<<nb, LIM_BS, 0, h->st>>>(K, S, D, h->BX, h->BY, h->flags, h->trouble, stage,
                                                        fused_divfree, sc_gate, h->sc, h->net, h->QM, h->pnet,
                                                        h->t_lo, h->t_hi, L, N);
    else if (K.detector == GDF_DETECT_LEARNED)
      k_limit<LIM_PNET, false><<<nb, LIM_BS, 0, h->st>>>(K, S, D, h->BX, h->BY, h->flags, h->trouble, stage,
                                                         fused_divfree, sc_gate, h->sc, h->net, h->QM, h->pnet,
                                                         h->t_lo, h->t_hi, nullptr, nullptr);
    else if (compact)
      k_limit<LIM_PLAIN, true><<<nb, LIM_BS, 0, h->st>>>(K, S, D, h->BX, h->BY, h->flags, h->trouble, stage,
                                                         fused_divfree, sc_gate, h->sc, nullptr, nullptr, nullptr,
                                                         0.f, 0.f, L, N);
    else
      k_limit<LIM_PLAIN, false><<<nb, LIM_BS, 0, h->st>>>(K, S, D, h->BX, h->BY, h->flags, h->trouble, stage,
                                                          fused_divfree, sc_gate, h->sc, nullptr, nullptr, nullptr,
                                                          0.f, 0.f, nullptr, nullptr);
  });
  if (rc0) return rc0;
  if (compact) {
    rc0 = run_kernel(h, GDF_K_LIMIT_TVB, [&] {
      k_limit_tvb<<<nblk(ncell, LIM_BS), LIM_BS, 0, h->st>>>(K, S, D, h->BX, h->BY, h->flags, stage, fused_divfree,
                                                             sc_gate, h->sc, L, N);
    });
    if (rc0) return rc0;
  }
  if (K.faceb) {
    // TVB_Limiter_P2.f90:126-187 then div_free: set_bc on the limited state,
    // face-B minmod, div-free reconstruction
    int rc = launch_set_bc(h, D, 0, sc_gate);
    if (rc) return rc;
    rc = run_kernel(h, GDF_K_FACEB_LIMIT, [&] {
      k_faceb_limit<<<nblk(K.fxplane + K.fyplane, 128), 128, 0, h->st>>>(K, D, h->BX, h->BY, sc_gate);
    });
    if (!rc) rc = run_kernel(h, GDF_K_DIVFREE, [&] { k_divfree<<<nblk(ncell, 128), 128, 0, h->st>>>(K, D, h->BX, h->BY, sc_gate); });
    if (rc) return rc;
  }
  return GDF_OK;
}

// One RK3 stage on the resident state (stage = 1, 2, 3).
static int launch_stage(GdfHandle* h, int stage) {
  const Consts& K = h->K;
  int rc;
  if (stage == 1) {
    if ((rc = launch_set_bc(h, h->U, 0, h->sc))) return rc;  // RK3.f90:74
  }
  if ((rc = launch_faces(h, h->U, h->sc))) return rc;
  rc = run_kernel(h, GDF_K_CELL, [&] {
    k_cell<<<nblk(K.plane, CELL_BS), CELL_BS, 0, h->st>>>(K, h->U, h->U0, h->UI, h->Fxh, h->Fyh, nullptr, h->sc, stage);
  });
  if (!rc) rc = run_kernel(h, GDF_K_BFACE, [&] {
    k_bface<<<nblk(K.fxplane + K.fyplane, 128), 128, 0, h->st>>>(K, h->EzRL, h->EzUD, h->EzV, h->BX, h->BX0, h->BXI,
                                                                 h->BY, h->BY0, h->BYI, nullptr, nullptr, h->sc, stage);
  });
  if (rc) return rc;
  if ((rc = launch_limit(h, h->UI, h->U, stage, h->sc))) return rc;
  // RK3.f90:97 / :123 set_bc after stages 1 and 2; after stage 3 the ghosts
  // are TVB_Limiter_P2's set_bc with div_free's zeroed B modes
  return launch_set_bc(h, h->U, stage == 3 ? 1 : 0, h->sc);
}

static int launch_step(GdfHandle* h) {
  int rc = launch_dt(h, h->U, 1);
  if (rc) return rc;
  for (int s = 1; s <= 3; ++s)
    if ((rc = launch_stage(h, s))) return rc;
  return GDF_OK;
}

static int sync_scal(GdfHandle* h) {
  CK(cudaMemcpyAsync(h->sc_host, h->sc, sizeof(Scal), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return GDF_OK;
}

static size_t uh_bytes(const GdfConfig& c) { return (size_t)(c.nx + 2) * (c.ny + 2) * NP * NE * sizeof(double); }
static size_t bx_bytes(const GdfConfig& c) { return (size_t)(c.nx + 1) * c.ny * 3 * sizeof(double); }
static size_t by_bytes(const GdfConfig& c) { return (size_t)c.nx * (c.ny + 1) * 3 * sizeof(double); }

// dead (mode, variable) slots must be zero in an uploaded state. The 28
// dead planes are scanned by several host threads (a 2048^2 state has 940 MB
// of them; one thread took longer than the upload it overlaps); the error
// names the first failing slot in (variable, mode) order.
static int check_dead_slots(const GdfConfig& c, const double* uh) {
  const size_t plane = (size_t)(c.nx + 2) * (c.ny + 2);
  std::vector<int> dead;
  for (int n = 0; n < NE; ++n)
    for (int d = 0; d < NP; ++d)
      if (!live_mode(n, d)) dead.push_back(d + 10 * n);
  // +0 and -0 pass, anything else (NaN included) fails: OR of the bit
  // patterns without the sign bit, a loop the compiler vectorises
  auto bad_range = [&](int slot, size_t q0, size_t q1) {
    const uint64_t* w = reinterpret_cast<const uint64_t*>(uh + plane * slot);
    uint64_t acc = 0;
    for (size_t q = q0; q < q1; ++q) acc |= w[q] << 1;
    return acc != 0;
  };
  const size_t total = plane * dead.size();
  unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  if (total < ((size_t)1 << 22)) nt = 1;
  std::vector<char> bad(dead.size(), 0);
  auto work = [&](unsigned t) {
    // thread t scans a contiguous share of the concatenated dead planes
    const size_t a = total * t / nt, b = total * (t + 1) / nt;
    for (size_t k = a; k < b;) {
      const size_t s = k / plane, q0 = k - s * plane;
      const size_t q1 = std::min(plane, q0 + (b - k));
      if (bad_range(dead[s], q0, q1)) bad[s] = 1;
      k += q1 - q0;
    }
  };
  if (nt == 1) {
    work(0);
  } else {
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t) th.emplace_back(work, t);
    for (auto& x : th) x.join();
  }
  for (size_t s = 0; s < dead.size(); ++s)
    if (bad[s])
      return fail(GDF_ERR_ARG, "uh has a nonzero value in mode " + std::to_string(dead[s] % 10 + 1) + " of variable " +
                                   std::to_string(dead[s] / 10 + 1) + ", which the P2 scheme never populates");
  return GDF_OK;
}

// Copy of the 52 live slot planes of uh (the device copies' dead slots are
// zero from allocation and no kernel writes them).
static cudaError_t copy_live(double* dst, const double* uh, const GdfConfig& c, cudaStream_t st,
                             cudaMemcpyKind kind) {
  const size_t plane = (size_t)(c.nx + 2) * (c.ny + 2);
  for (int n = 0; n < NE; ++n) {
    // live slots of a variable are modes 0..5 plus (Bx) 6, 8 or (By) 7, 9
    const size_t o = plane * (10 * n);
    cudaError_t e = cudaMemcpyAsync(dst + o, uh + o, 6 * plane * sizeof(double), kind, st);
    if (e != cudaSuccess) return e;
    for (int d = 6; d < NP; ++d) {
      if (!live_mode(n, d)) continue;
      e = cudaMemcpyAsync(dst + o + plane * d, uh + o + plane * d, plane * sizeof(double), kind, st);
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

namespace gdf {
int dead_slot_error(const GdfConfig& c, const double* uh, std::string& msg) {
  const int rc = check_dead_slots(c, uh);
  if (rc) msg = g_err;
  return rc;
}
}  // namespace gdf

// ------------------------------------------------------------------------
// Scratch of gdf_lh_noalloc: the face fluxes (Fxhat, Fyhat) and face Ez that
// k_face writes and k_cell reads, for grids with at most NOALLOC_MAX_FACES
// faces per direction. The module holds this array on every device that
// loads the library, until the process exits. Host code must not use the
// symbol as a device address; gdf_lh_noalloc takes its address per device
// with cudaGetSymbolAddress.
constexpr long long NOALLOC_MAX_FACES = 16640;  // (nx+1)*ny and nx*(ny+1); 128 x 128 fits
constexpr long long NOALLOC_DOUBLES = 2 * NOALLOC_MAX_FACES * (NG * NE + NG);
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_DOUBLES];


// Capture one time step (RK3.f90:60-151) of the resident state as a CUDA
// graph; replays need no host work between steps.
static int ensure_graph(GdfHandle* h) {
  if (h->graph) return GDF_OK;
  cudaGraph_t g;
  CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
  const int64_t l0 = h->launches;
  int rc = launch_step(h);
  h->step_launches = h->launches - l0;
  h->launches = l0;
  cudaError_t e = cudaStreamEndCapture(h->st, &g);
  if (rc) return rc;
  if (e != cudaSuccess) return fail(GDF_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&h->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    h->graph = nullptr;
    return fail(GDF_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  }
  return GDF_OK;
}

static size_t state_bytes(const GdfConfig& c) { return (size_t)36 * c.nx * c.ny * sizeof(double); }

// A launch outside the step (state transfer): counted, its error reported.
template <class F>
static int run_plain(GdfHandle* h, F&& launch) {
  launch();
  h->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(GDF_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  return GDF_OK;
}

extern "C" {

const char* gdf_last_error(void) { return g_err.c_str(); }

int gdf_build_exact(void) { return GDF_EXACT; }

int64_t gdf_kernel_launches(GdfHandle* h) { return h ? h->launches : -1; }

int gdf_create(const GdfConfig* cfg, GdfHandle** out) {
  if (!out) return fail(GDF_ERR_ARG, "null handle pointer");
  *out = nullptr;
  int rc = check_config(cfg);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(GDF_ERR_CUDA, "no CUDA device available");
  }
  GdfHandle* h = new GdfHandle();
  h->cfg = *cfg;
  build_consts(*cfg, h->K);
  if (upload_basis_once(h->K, true) != cudaSuccess) {
    cudaGetLastError();
    delete h;
    return fail(GDF_ERR_CUDA, "uploading the basis tables failed");
  }
  const GdfConfig& c = *cfg;
  const size_t ub = uh_bytes(c), bxb = bx_bytes(c), byb = by_bytes(c);
  const size_t fxb = (size_t)h->K.fxplane * NG * NE * sizeof(double);
  const size_t fyb = (size_t)h->K.fyplane * NG * NE * sizeof(double);
  const long long ncell = (long long)c.nx * c.ny;
  h->dt_blocks = (int)nblk(ncell, DT_BS);
  {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || h->sms <= 0) {
      cudaGetLastError();
      delete h;
      return fail(GDF_ERR_CUDA, "querying the device's SM count failed");
    }
  }
  auto alloc = [&](void** p, size_t bytes) -> bool {
    if (cudaMalloc(p, bytes) != cudaSuccess) return false;
    return cudaMemset(*p, 0, bytes) == cudaSuccess;
  };
  bool ok = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && alloc((void**)&h->U, ub) && alloc((void**)&h->U0, ub) && alloc((void**)&h->UI, ub) &&
       alloc((void**)&h->UT, ub);
  ok = ok && alloc((void**)&h->BX, bxb) && alloc((void**)&h->BX0, bxb) && alloc((void**)&h->BXI, bxb);
  ok = ok && alloc((void**)&h->BY, byb) && alloc((void**)&h->BY0, byb) && alloc((void**)&h->BYI, byb);
  ok = ok && alloc((void**)&h->Fxh, fxb) && alloc((void**)&h->Fyh, fyb);
  ok = ok && alloc((void**)&h->EzRL, (size_t)h->K.fxplane * NG * sizeof(double)) &&
       alloc((void**)&h->EzUD, (size_t)h->K.fyplane * NG * sizeof(double)) &&
       alloc((void**)&h->EzV, (size_t)h->K.vplane * sizeof(double));
  ok = ok && alloc((void**)&h->part, (size_t)(h->dt_blocks + 1) * 4 * sizeof(double));
  ok = ok && alloc((void**)&h->flags, (size_t)ncell * sizeof(int32_t)) &&
       alloc((void**)&h->trouble, (size_t)ncell * sizeof(int32_t));
  ok = ok && alloc((void**)&h->lim_list, (size_t)ncell * sizeof(int32_t)) &&
       alloc((void**)&h->lim_count, sizeof(int32_t));
  ok = ok && alloc((void**)&h->sc, sizeof(Scal));
  ok = ok && cudaMallocHost((void**)&h->sc_host, sizeof(Scal)) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    gdf_destroy(h);
    return fail(GDF_ERR_NOMEM, "device allocation failed for a " + std::to_string(c.nx) + "x" +
                                   std::to_string(c.ny) + " grid");
  }
  std::memset(h->sc_host, 0, sizeof(Scal));
  h->sc_host->tend = 1e300;
  h->sc_host->active = 1;
  if (cudaMemcpy(h->sc, h->sc_host, sizeof(Scal), cudaMemcpyHostToDevice) != cudaSuccess) {
    gdf_destroy(h);
    return fail(GDF_ERR_CUDA, "initialising device scalars failed");
  }
  *out = h;
  return GDF_OK;
}

int gdf_destroy(GdfHandle* h) {
  if (!h) return GDF_OK;
  if (h->graph) cudaGraphExecDestroy(h->graph);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  double* bufs[] = {h->U, h->U0, h->UI, h->UT, h->BX, h->BX0, h->BXI, h->BY, h->BY0, h->BYI,
                    h->Fxh, h->Fyh, h->EzRL, h->EzUD, h->EzV, h->part};
  for (double* p : bufs)
    if (p) cudaFree(p);
  if (h->QM) cudaFree(h->QM);
  if (h->pnet) cudaFree(h->pnet);
  if (h->net) cudaFree(h->net);
  if (h->flags) cudaFree(h->flags);
  if (h->trouble) cudaFree(h->trouble);
  if (h->lim_list) cudaFree(h->lim_list);
  if (h->lim_count) cudaFree(h->lim_count);
  if (h->sc) cudaFree(h->sc);
  if (h->sc_host) cudaFreeHost(h->sc_host);
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
  return GDF_OK;
}

int gdf_upload(GdfHandle* h, const double* uh, const double* bx, const double* by) {
  if (!h || !uh || !bx || !by) return fail(GDF_ERR_ARG, "null argument");
  // the live planes travel to a staging buffer while the host checks the
  // dead ones; the resident state changes only once the check has passed
  CK(copy_live(h->UT, uh, h->cfg, h->st, cudaMemcpyHostToDevice));
  int rc = check_dead_slots(h->cfg, uh);
  if (rc) {
    cudaStreamSynchronize(h->st);
    return rc;
  }
  CK(copy_live(h->U, h->UT, h->cfg, h->st, cudaMemcpyDeviceToDevice));
  CK(cudaMemcpyAsync(h->BX, bx, bx_bytes(h->cfg), cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(h->BY, by, by_bytes(h->cfg), cudaMemcpyHostToDevice, h->st));
  CK(cudaStreamSynchronize(h->st));
  h->uploaded = 1;
  return GDF_OK;
}

int gdf_download(GdfHandle* h, double* uh, double* bx, double* by) {
  if (!h) return fail(GDF_ERR_ARG, "null handle");
  if (!h->uploaded) return fail(GDF_ERR_STATE, "no state uploaded");
  if (uh) CK(cudaMemcpyAsync(uh, h->U, uh_bytes(h->cfg), cudaMemcpyDeviceToHost, h->st));
  if (bx) CK(cudaMemcpyAsync(bx, h->BX, bx_bytes(h->cfg), cudaMemcpyDeviceToHost, h->st));
  if (by) CK(cudaMemcpyAsync(by, h->BY, by_bytes(h->cfg), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return GDF_OK;
}

int gdf_download_live(GdfHandle* h, double* uh, double* bx, double* by) {
  if (!h) return fail(GDF_ERR_ARG, "null handle");
  if (!h->uploaded) return fail(GDF_ERR_STATE, "no state uploaded");
  if (uh) CK(copy_live(uh, h->U, h->cfg, h->st, cudaMemcpyDeviceToHost));
  if (bx) CK(cudaMemcpyAsync(bx, h->BX, bx_bytes(h->cfg), cudaMemcpyDeviceToHost, h->st));
  if (by) CK(cudaMemcpyAsync(by, h->BY, by_bytes(h->cfg), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return GDF_OK;
}

int gdf_upload_state(GdfHandle* h, const double* cells, const double* bx, const double* by) {
  if (!h || !cells || !bx || !by) return fail(GDF_ERR_ARG, "null argument");
  const Consts& K = h->K;
  const long long n = 36LL * K.nx * K.ny;
  CK(cudaMemcpyAsync(h->UT, cells, state_bytes(h->cfg), cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(h->BX, bx, bx_bytes(h->cfg), cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(h->BY, by, by_bytes(h->cfg), cudaMemcpyHostToDevice, h->st));
  int rc = run_plain(h, [&] { k_unpack_state<<<nblk(n, 256), 256, 0, h->st>>>(K, h->UT, h->U); });
  // the cell B modes from the face fields (div_free_Balsara.f90:13-79), the
  // ghosts as the end of a stage leaves them (set_bc with the ghost B
  // modes cleared, div_free_Balsara.f90:11)
  if (!rc) rc = run_plain(h, [&] { k_divfree<<<nblk((long long)K.nx * K.ny, 128), 128, 0, h->st>>>(K, h->U, h->BX, h->BY, nullptr); });
  if (!rc) {
    const long long nb = (2LL * (K.nx + 2) + 2LL * K.ny) * NLIVE;
    rc = run_plain(h, [&] { k_set_bc<<<nblk(nb, 256), 256, 0, h->st>>>(K, h->U, 1, nullptr); });
  }
  if (rc) return rc;
  CK(cudaStreamSynchronize(h->st));
  h->uploaded = 1;
  return GDF_OK;
}

int gdf_download_state(GdfHandle* h, double* cells, double* bx, double* by) {
  if (!h) return fail(GDF_ERR_ARG, "null handle");
  if (!h->uploaded) return fail(GDF_ERR_STATE, "no state uploaded");
  if (cells) {
    const long long n = 36LL * h->K.nx * h->K.ny;
    int rc = run_plain(h, [&] { k_pack_state<<<nblk(n, 256), 256, 0, h->st>>>(h->K, h->U, h->UT); });
    if (rc) return rc;
    CK(cudaMemcpyAsync(cells, h->UT, state_bytes(h->cfg), cudaMemcpyDeviceToHost, h->st));
  }
  if (bx) CK(cudaMemcpyAsync(bx, h->BX, bx_bytes(h->cfg), cudaMemcpyDeviceToHost, h->st));
  if (by) CK(cudaMemcpyAsync(by, h->BY, by_bytes(h->cfg), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return GDF_OK;
}

int gdf_set_time(GdfHandle* h, double t) {
  if (!h) return fail(GDF_ERR_ARG, "null handle");
  int rc = sync_scal(h);
  if (rc) return rc;
  h->sc_host->t = t;
  CK(cudaMemcpyAsync(h->sc, h->sc_host, sizeof(Scal), cudaMemcpyHostToDevice, h->st));
  CK(cudaStreamSynchronize(h->st));
  return GDF_OK;
}

int gdf_get_time(GdfHandle* h, double* t, double* dt) {
  if (!h) return fail(GDF_ERR_ARG, "null handle");
  int rc = sync_scal(h);
  if (rc) return rc;
  if (t) *t = h->sc_host->t;
  if (dt) *dt = h->sc_host->dt;
  return GDF_OK;
}

static int set_scal(GdfHandle* h, double t, double tend, int active) {
  int rc = sync_scal(h);
  if (rc) return rc;
  h->sc_host->t = t;
  h->sc_host->tend = tend;
  h->sc_host->active = active;
  h->sc_host->status = 0;
  CK(cudaMemcpyAsync(h->sc, h->sc_host, sizeof(Scal), cudaMemcpyHostToDevice, h->st));
  return GDF_OK;
}

int gdf_prepare(GdfHandle* h, int32_t* flags) {
  if (!h) return fail(GDF_ERR_ARG, "null handle");
  if (!h->uploaded) return fail(GDF_ERR_STATE, "no state uploaded");
  int rc = set_scal(h, 0.0, h->sc_host->tend, 1);
  if (rc) return rc;
  // RK3.f90:8-12: set_bc, TVB_Limiter_P2, div_free_Balsara
  if ((rc = launch_set_bc(h, h->U, 0, nullptr))) return rc;
  CK(cudaMemcpyAsync(h->UI, h->U, uh_bytes(h->cfg), cudaMemcpyDeviceToDevice, h->st));
  if ((rc = launch_limit(h, h->UI, h->U, 1, nullptr))) return rc;
  if ((rc = launch_set_bc(h, h->U, 1, nullptr))) return rc;
  if (flags) {
    CK(cudaMemcpyAsync(flags, h->flags, (size_t)h->cfg.nx * h->cfg.ny * sizeof(int32_t), cudaMemcpyDeviceToHost,
                       h->st));
  }
  rc = sync_scal(h);
  if (rc) return rc;
  if (h->sc_host->status) return fail(GDF_ERR_NUMERIC, "non-positive density or non-finite energy after limiting");
  return GDF_OK;
}

int gdf_step(GdfHandle* h, double tend, double* t, double* dt_out, int32_t* flags) {
  if (!h || !t) return fail(GDF_ERR_ARG, "null argument");
  if (!h->uploaded) return fail(GDF_ERR_STATE, "no state uploaded");
  int rc = set_scal(h, *t, tend, 1);
  if (rc) return rc;
  if ((rc = launch_step(h))) return rc;
  if (flags) {
    CK(cudaMemcpyAsync(flags, h->flags, (size_t)h->cfg.nx * h->cfg.ny * sizeof(int32_t), cudaMemcpyDeviceToHost,
                       h->st));
  }
  if ((rc = sync_scal(h))) return rc;
  *t = h->sc_host->t;
  if (dt_out) *dt_out = h->sc_host->dt;
  if (h->sc_host->status) return fail(GDF_ERR_NUMERIC, "non-finite or non-positive state or dt in this step");
  return GDF_OK;
}

int gdf_advance(GdfHandle* h, double tend, int32_t max_steps, double* t, int32_t* steps) {
  if (!h || !t) return fail(GDF_ERR_ARG, "null argument");
  if (!h->uploaded) return fail(GDF_ERR_STATE, "no state uploaded");
  if (max_steps < 0) return fail(GDF_ERR_ARG, "max_steps < 0");
  int rc = set_scal(h, *t, tend, 1);
  if (rc) return rc;
  const long long s0 = h->sc_host->steps;
  if ((rc = ensure_graph(h))) return rc;
  const int chunk = 64;
  int done = 0;
  while (done < max_steps) {
    const int n = std::min(chunk, max_steps - done);
    for (int k = 0; k < n; ++k) {
      CK(cudaGraphLaunch(h->graph, h->st));
      h->launches += h->step_launches;
    }
    done += n;
    if ((rc = sync_scal(h))) return rc;
    if (h->sc_host->status) break;
    if (!(h->sc_host->t < tend)) break;
  }
  if ((rc = sync_scal(h))) return rc;
  *t = h->sc_host->t;
  if (steps) *steps = (int32_t)(h->sc_host->steps - s0);
  if (h->sc_host->status) return fail(GDF_ERR_NUMERIC, "non-finite or non-positive state or dt during advance");
  return GDF_OK;
}

// Lh of one grid on caller-owned device buffers, allocating nothing (the
// face-flux scratch is g_noalloc_scratch). Stream-ordered on `stream`;
// returns after enqueueing.
int gdf_lh_noalloc(const GdfConfig* cfg, const double* d_uh, double* d_du, void* stream) {
  int rc = check_config(cfg);
  if (rc) return rc;
  if (!d_uh || !d_du) return fail(GDF_ERR_ARG, "null device buffer");
  const long long fx = (long long)(cfg->nx + 1) * cfg->ny, fy = (long long)cfg->nx * (cfg->ny + 1);
  if (fx > NOALLOC_MAX_FACES || fy > NOALLOC_MAX_FACES)
    return fail(GDF_ERR_ARG, "gdf_lh_noalloc: grid " + std::to_string(cfg->nx) + "x" + std::to_string(cfg->ny) +
                                 " exceeds its fixed scratch: (nx+1)*ny and nx*(ny+1) must be at most " +
                                 std::to_string(NOALLOC_MAX_FACES) + " (128x128 fits); use gdf_lh");
  // The scratch's device address and the basis tables are set up on every
  // call rather than cached: a cudaDeviceReset between calls reloads the
  // module, which moves the array and clears the __constant__ tables.
  // cudaGetSymbolAddress is a host-side query; the tables (~10 KB, the same
  // bytes for every grid) are copied stream-ordered ahead of the kernels.
  void* base = nullptr;
  {
    cudaError_t e = cudaGetSymbolAddress(&base, g_noalloc_scratch);
    if (e != cudaSuccess)
      return fail(GDF_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  Consts K;
  build_consts(*cfg, K);
  {
    Basis B;
    basis_of(K, B);
    cudaError_t e = cudaMemcpyToSymbolAsync(c_basis, &B, sizeof(Basis), 0, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return fail(GDF_ERR_CUDA, std::string("basis tables: ") + cudaGetErrorString(e));
  }
  double* Fxh = static_cast<double*>(base);
  double* Fyh = Fxh + fx * NG * NE;
  double* ezx = Fyh + fy * NG * NE;
  double* ezy = ezx + fx * NG;
  // every face point of Fxh/Fyh/Ez is written before k_cell reads it, so
  // the scratch left by an earlier call needs no clearing; du's ghost and
  // dead slots must read 0
  CK(cudaMemsetAsync(d_du, 0, uh_bytes(*cfg), st));
  k_face<0><<<nblk(fx * NG, 128), 128, 0, st>>>(K, d_uh, Fxh, ezx, nullptr);
  k_face<1><<<nblk(fy * NG, 128), 128, 0, st>>>(K, d_uh, Fyh, ezy, nullptr);
  k_cell<<<nblk(K.plane, CELL_BS), CELL_BS, 0, st>>>(K, d_uh, nullptr, nullptr, Fxh, Fyh, d_du, nullptr, 0);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(GDF_ERR_CUDA, std::string("gdf_lh_noalloc launch: ") + cudaGetErrorString(e));
  return GDF_OK;
}

// init_data.f90 on the device, into the handle's resident state.
int gdf_init_data_device(GdfHandle* h, int32_t problem, const double* params) {
  if (!h) return fail(GDF_ERR_ARG, "null handle");
  if (problem < GDF_PROB_VORTEX || problem > GDF_PROB_CLOUD_SHOCK) return fail(GDF_ERR_ARG, "unknown problem");
  CK(cudaMemsetAsync(h->U, 0, uh_bytes(h->cfg), h->st));
  std::string err;
  int rc = gdf::init_data_device(h->cfg, problem, params, h->U, h->BX, h->BY, h->st, err);
  if (rc) {
    cudaStreamSynchronize(h->st);
    return fail(rc, err);
  }
  CK(cudaStreamSynchronize(h->st));
  h->uploaded = 1;
  return GDF_OK;
}

extern "C" const void* gdf_mlp_device_params(GdfMlp* m);

int gdf_set_indicator(GdfHandle* h, GdfMlp* m, float t_lo, float t_hi) {
  if (!h || !m) return fail(GDF_ERR_ARG, "null argument");
  if (!(t_lo <= t_hi)) return fail(GDF_ERR_ARG, "t_lo must not exceed t_hi");
  if (!h->net) CK(cudaMalloc((void**)&h->net, sizeof(MlpDev)));
  if (!h->QM) CK(cudaMalloc((void**)&h->QM, (size_t)QMODES * h->K.plane * sizeof(float)));
  if (!h->pnet) CK(cudaMalloc((void**)&h->pnet, (size_t)h->K.nx * h->K.ny * sizeof(float)));
  CK(cudaMemcpy(h->net, gdf_mlp_device_params(m), sizeof(MlpDev), cudaMemcpyDeviceToDevice));
  h->t_lo = t_lo;
  h->t_hi = t_hi;
  if (h->graph) {   // the captured step holds the old kernel arguments
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  return GDF_OK;
}

int gdf_features(GdfHandle* h, const double* uh, float* X) {
  if (!h || !uh || !X) return fail(GDF_ERR_ARG, "null argument");
  int rc = check_dead_slots(h->cfg, uh);
  if (rc) return rc;
  const long long ncell = (long long)h->cfg.nx * h->cfg.ny;
  if (!h->QM) CK(cudaMalloc((void**)&h->QM, (size_t)QMODES * h->K.plane * sizeof(float)));
  float* dX = nullptr;
  CK(cudaMallocAsync((void**)&dX, (size_t)ncell * NFEAT * sizeof(float), h->st));
  CK(cudaMemcpyAsync(h->UT, uh, uh_bytes(h->cfg), cudaMemcpyHostToDevice, h->st));
  rc = run_kernel(h, GDF_K_LIMIT, [&] { k_qmodes<<<nblk(h->K.plane, 128), 128, 0, h->st>>>(h->K, h->UT, h->QM); });
  if (!rc) rc = run_kernel(h, GDF_K_LIMIT, [&] { k_features<<<nblk(ncell, 128), 128, 0, h->st>>>(h->K, h->QM, dX); });
  if (!rc) {
    cudaError_t e = cudaMemcpyAsync(X, dX, (size_t)ncell * NFEAT * sizeof(float), cudaMemcpyDeviceToHost, h->st);
    if (e != cudaSuccess) rc = fail(GDF_ERR_CUDA, cudaGetErrorString(e));
  }
  cudaFreeAsync(dX, h->st);
  CK(cudaStreamSynchronize(h->st));
  return rc;
}

int gdf_config_of(GdfHandle* h, GdfConfig* out) {
  if (!h || !out) return fail(GDF_ERR_ARG, "null argument");
  *out = h->cfg;
  return GDF_OK;
}

// Is_Trouble_Cell (the sticky KXRCF flags), nx*ny int32 in (i-1)+nx*(j-1) order
int gdf_get_trouble(GdfHandle* h, int32_t* trouble) {
  if (!h || !trouble) return fail(GDF_ERR_ARG, "null argument");
  CK(cudaMemcpyAsync(trouble, h->trouble, (size_t)h->cfg.nx * h->cfg.ny * sizeof(int32_t), cudaMemcpyDeviceToHost,
                     h->st));
  CK(cudaStreamSynchronize(h->st));
  return GDF_OK;
}

int gdf_set_trouble(GdfHandle* h, const int32_t* trouble) {
  if (!h || !trouble) return fail(GDF_ERR_ARG, "null argument");
  CK(cudaMemcpyAsync(h->trouble, trouble, (size_t)h->cfg.nx * h->cfg.ny * sizeof(int32_t), cudaMemcpyHostToDevice,
                     h->st));
  CK(cudaStreamSynchronize(h->st));
  return GDF_OK;
}

int gdf_set_device(int32_t device) {
  CK(cudaSetDevice(device));
  return GDF_OK;
}

int gdf_advance_timed(GdfHandle* h, double tend, int32_t steps, double* t, int32_t* taken, double* device_ms) {
  if (!h || !t || !device_ms || steps < 1) return fail(GDF_ERR_ARG, "bad argument");
  if (!h->uploaded) return fail(GDF_ERR_STATE, "no state uploaded");
  int rc = set_scal(h, *t, tend, 1);
  if (rc) return rc;
  const long long s0 = h->sc_host->steps;
  if ((rc = ensure_graph(h))) return rc;
  if (!h->ev0) {
    CK(cudaEventCreate(&h->ev0));
    CK(cudaEventCreate(&h->ev1));
  }
  CK(cudaStreamSynchronize(h->st));
  CK(cudaEventRecord(h->ev0, h->st));
  for (int k = 0; k < steps; ++k) {
    CK(cudaGraphLaunch(h->graph, h->st));
    h->launches += h->step_launches;
  }
  CK(cudaEventRecord(h->ev1, h->st));
  CK(cudaEventSynchronize(h->ev1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  *device_ms = ms;
  if ((rc = sync_scal(h))) return rc;
  *t = h->sc_host->t;
  if (taken) *taken = (int32_t)(h->sc_host->steps - s0);
  if (h->sc_host->status) return fail(GDF_ERR_NUMERIC, "non-finite or non-positive state or dt during advance");
  return GDF_OK;
}

int gdf_lh(GdfHandle* h, const double* uh, double* du) {
  if (!h || !uh || !du) return fail(GDF_ERR_ARG, "null argument");
  int rc = check_dead_slots(h->cfg, uh);
  if (rc) return rc;
  const size_t ub = uh_bytes(h->cfg);
  CK(cudaMemcpyAsync(h->UT, uh, ub, cudaMemcpyHostToDevice, h->st));
  CK(cudaMemsetAsync(h->UI, 0, ub, h->st));  // du (ghost and dead entries stay 0)
  if ((rc = launch_faces(h, h->UT, nullptr))) return rc;
  rc = run_kernel(h, GDF_K_CELL, [&] {
    k_cell<<<nblk(h->K.plane, CELL_BS), CELL_BS, 0, h->st>>>(h->K, h->UT, nullptr, nullptr, h->Fxh, h->Fyh, h->UI,
                                                             nullptr, 0);
  });
  if (rc) return rc;
  CK(cudaMemcpyAsync(du, h->UI, ub, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return GDF_OK;
}

int gdf_lhez(GdfHandle* h, const double* uh, double* dez1, double* dez2) {
  if (!h || !uh || !dez1 || !dez2) return fail(GDF_ERR_ARG, "null argument");
  int rc = check_dead_slots(h->cfg, uh);
  if (rc) return rc;
  CK(cudaMemcpyAsync(h->UT, uh, uh_bytes(h->cfg), cudaMemcpyHostToDevice, h->st));
  if ((rc = launch_faces(h, h->UT, nullptr))) return rc;
  double *d1 = h->BX0, *d2 = h->BY0;
  rc = run_kernel(h, GDF_K_BFACE, [&] {
    k_bface<<<nblk(h->K.fxplane + h->K.fyplane, 128), 128, 0, h->st>>>(
        h->K, h->EzRL, h->EzUD, h->EzV, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, d1, d2, nullptr, 0);
  });
  if (rc) return rc;
  CK(cudaMemcpyAsync(dez1, d1, bx_bytes(h->cfg), cudaMemcpyDeviceToHost, h->st));
  CK(cudaMemcpyAsync(dez2, d2, by_bytes(h->cfg), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return GDF_OK;
}

int gdf_limit(GdfHandle* h, double* uh, double* bx, double* by, int32_t* flags) {
  if (!h || !uh || !bx || !by) return fail(GDF_ERR_ARG, "null argument");
  int rc = check_dead_slots(h->cfg, uh);
  if (rc) return rc;
  const size_t ub = uh_bytes(h->cfg);
  // the limiter works on the resident buffers; save and restore them
  CK(cudaMemcpyAsync(h->UT, uh, ub, cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(h->U0, h->UT, ub, cudaMemcpyDeviceToDevice, h->st));
  CK(cudaMemcpyAsync(h->BX0, bx, bx_bytes(h->cfg), cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(h->BY0, by, by_bytes(h->cfg), cudaMemcpyHostToDevice, h->st));
  double* sBX = h->BX;
  double* sBY = h->BY;
  h->BX = h->BX0;
  h->BY = h->BY0;
  rc = launch_limit(h, h->UT, h->U0, 1, nullptr);
  if (!rc) rc = launch_set_bc(h, h->U0, 1, nullptr);
  h->BX = sBX;
  h->BY = sBY;
  if (rc) return rc;
  CK(cudaMemcpyAsync(uh, h->U0, ub, cudaMemcpyDeviceToHost, h->st));
  CK(cudaMemcpyAsync(bx, h->BX0, bx_bytes(h->cfg), cudaMemcpyDeviceToHost, h->st));
  CK(cudaMemcpyAsync(by, h->BY0, by_bytes(h->cfg), cudaMemcpyDeviceToHost, h->st));
  if (flags)
    CK(cudaMemcpyAsync(flags, h->flags, (size_t)h->cfg.nx * h->cfg.ny * sizeof(int32_t), cudaMemcpyDeviceToHost,
                       h->st));
  CK(cudaStreamSynchronize(h->st));
  return GDF_OK;
}

int gdf_dt(GdfHandle* h, const double* uh, double* dt) {
  if (!h || !uh || !dt) return fail(GDF_ERR_ARG, "null argument");
  CK(cudaMemcpyAsync(h->UT, uh, uh_bytes(h->cfg), cudaMemcpyHostToDevice, h->st));
  int rc = launch_dt(h, h->UT, 0);
  if (rc) return rc;
  if ((rc = sync_scal(h))) return rc;
  *dt = h->sc_host->dt;
  return GDF_OK;
}

void* gdf_stream(GdfHandle* h) { return h ? (void*)h->st : nullptr; }

int gdf_profile(GdfHandle* h, int32_t steps, double* ms_per_launch, int64_t* launches_per_kind, int32_t nkinds) {
  if (!h || !ms_per_launch || steps < 1) return fail(GDF_ERR_ARG, "bad argument");
  if (!h->uploaded) return fail(GDF_ERR_STATE, "no state uploaded");
  if (!h->ev0) {
    CK(cudaEventCreate(&h->ev0));
    CK(cudaEventCreate(&h->ev1));
  }
  for (int k = 0; k < GDF_KERNEL_KINDS; ++k) { h->prof_ms[k] = 0; h->prof_n[k] = 0; }
  int rc = sync_scal(h);
  if (rc) return rc;
  const double t0 = h->sc_host->t;
  if ((rc = set_scal(h, t0, 1e300, 1))) return rc;
  h->prof = 1;
  for (int s = 0; s < steps && !rc; ++s) rc = launch_step(h);
  h->prof = 0;
  if (rc) return rc;
  CK(cudaStreamSynchronize(h->st));
  for (int k = 0; k < nkinds && k < GDF_KERNEL_KINDS; ++k) {
    ms_per_launch[k] = h->prof_n[k] ? h->prof_ms[k] / (double)h->prof_n[k] : 0.0;
    if (launches_per_kind) launches_per_kind[k] = h->prof_n[k] / steps;
  }
  return GDF_OK;
}

int gdf_diagnostics(GdfHandle* h, double* umax, double* totaldiv, double* pmin, int64_t* n_troubled) {
  if (!h) return fail(GDF_ERR_ARG, "null handle");
  if (!h->uploaded) return fail(GDF_ERR_STATE, "no state uploaded");
  const long long ncell = (long long)h->cfg.nx * h->cfg.ny;
  const int nb = (int)nblk(ncell, DT_BS);
  double* part = nullptr;
  CK(cudaMallocAsync((void**)&part, (size_t)nb * 4 * sizeof(double), h->st));
  int rc0 = run_kernel(h, GDF_K_DIAG, [&] { k_diag_partial<<<nb, DT_BS, 0, h->st>>>(h->K, h->U, h->flags, part); });
  if (!rc0) rc0 = run_kernel(h, GDF_K_DIAG, [&] { k_diag_final<<<1, 32, 0, h->st>>>(h->K, part, nb, h->sc); });
  if (rc0) return rc0;
  CK(cudaFreeAsync(part, h->st));
  int rc = sync_scal(h);
  if (rc) return rc;
  if (umax) *umax = h->sc_host->umax;
  if (totaldiv) *totaldiv = h->sc_host->totaldiv;
  if (pmin) *pmin = h->sc_host->pmin;
  if (n_troubled) *n_troubled = h->sc_host->troubled;
  return GDF_OK;
}

}  // extern "C"
