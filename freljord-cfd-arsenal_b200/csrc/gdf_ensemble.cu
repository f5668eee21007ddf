// gdf_ensemble.cu -- an ensemble of independent GDF P2 problems of different
// grid sizes advanced together: one persistent cooperative kernel per RK
// stage, the three stages of a step captured as one CUDA graph.
//
// Work of a stage is a sequence of phases (set_bc; face and vertex Riemann
// solves; residual + combine and face-B update; indicator modes; limiter;
// face-B limiter and div-free reconstruction), the same per-item device code
// as the single-problem kernels (gdf_device.cuh). Each phase is a flat list of
// tiles over all instances (prefix sums per kind); the resident blocks take
// tiles round-robin, and a grid barrier separates dependent phases. Every
// item is computed exactly as the single-problem path computes it and the
// per-instance dt reduction is a maximum, so each instance follows the
// trajectory it has when run alone, value for value.
//
// Per instance, a step runs while t < tend (its own dt, its own end time);
// an instance that has arrived stays idle while the others go on.
//
// The grid barrier spins with a time limit (EnsArgs::timeout_ns: 2 s, or
// 200 ns per cell of the ensemble if longer): a block that waits longer
// records an error, every block returns, and the host reports
// GDF_ERR_TIMEOUT.

#include <cuda/atomic>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gdf.h"
#include "gdf_device.cuh"

extern "C" const void* gdf_mlp_device_params(GdfMlp* m);

namespace gdf {
namespace {

constexpr int ENS_BS = 64;   // threads per block: one limiter / cell tile row

enum EnsKind {
  EK_DT,     // interior cells: wave-speed maxima (calculate_dt)
  EK_BC,     // ghost items (set_bc)
  EK_BCF,    // ghost items of face-B-limited instances (TVB_Limiter_P2's set_bc)
  EK_FX,     // x-face quadrature points
  EK_FY,     // y-face quadrature points
  EK_VX,     // vertices
  EK_CELL,   // cells incl. ghosts (residual + combine)
  EK_BF,     // faces (dEz + face-B combine)
  EK_QM,     // cells incl. ghosts (indicator modes)
  EK_LIM,    // interior cells (limiter), one ENS_BS tile at a time
  EK_FB,     // faces of face-B-limited instances
  EK_DF,     // interior cells of face-B-limited instances (div-free)
  EK_COPY,   // live slots of every cell (prepare: U -> UI)
  EK_N
};

struct EnsInst {
  const Consts* K;
  Scal* sc;
  double *U, *U0, *UI, *BX, *BX0, *BXI, *BY, *BY0, *BYI;
  double *Fxh, *Fyh, *EzRL, *EzUD, *EzV;
  int32_t *flags, *trouble;
  float* QM;
  float* pnet;
};

struct EnsSync {
  unsigned int count;
  unsigned int gen;
  int err;   // bit 0: a grid barrier timed out
  int pad;
};

struct EnsArgs {
  const EnsInst* inst;
  const int* off;                 // [EK_N][n + 1] tile prefix sums
  unsigned long long* amax;       // [2n] bit patterns of the x / y speed maxima
  EnsSync* sync;
  const MlpDev* net;
  unsigned long long timeout_ns;
  int n;
  int any_faceb;
  float t_lo, t_hi;
  int per_tile[EK_N];             // items per tile
  int total[EK_N];                // tiles
};

// The per-item bodies are called, not inlined, from the persistent kernel:
// inlined into one kernel their live ranges add up to a 1.4 KB stack frame
// whose spills went to DRAM; as calls each keeps the register allocation it
// has in its own single-problem kernel.
__device__ __noinline__ void call_face_x(const Consts& K, const double* U, double* F, double* Ez, long long item) {
  face_item<0>(K, U, F, Ez, item);
}
__device__ __noinline__ void call_face_y(const Consts& K, const double* U, double* F, double* Ez, long long item) {
  face_item<1>(K, U, F, Ez, item);
}
__device__ __noinline__ void call_vertex(const Consts& K, const double* U, double* EzV, long long item) {
  vertex_item(K, U, EzV, item);
}
extern __shared__ __align__(16) unsigned char ens_sm[];   // the stage kernel's dynamic shared memory
__device__ __noinline__ void call_cell(const Consts& K, const double* U, double* U0, double* UI, const double* Fxh,
                                       const double* Fyh, const Scal* sc, int stage, long long item) {
  cell_item<false, GDF_CELL_PAIRS != 0>(K, U, U0, UI, Fxh, Fyh, nullptr, sc, stage, item,
                                        reinterpret_cast<double*>(ens_sm));
}
__device__ __noinline__ void call_bface(const Consts& K, const double* EzRL, const double* EzUD, const double* EzV,
                                        double* BX, double* BX0, double* BXI, double* BY, double* BY0, double* BYI,
                                        const Scal* sc, int stage, long long item) {
  bface_item(K, EzRL, EzUD, EzV, BX, BX0, BXI, BY, BY0, BYI, nullptr, nullptr, sc, stage, item);
}
__device__ __noinline__ void call_qmodes(const Consts& K, const double* S, float* QM, long long item) {
  qmodes_item(K, S, QM, item);
}
template <int LM>
__device__ __noinline__ void call_limit(const Consts& K, const double* S, double* D, const double* BX, const double* BY,
                                        int32_t* flags, int32_t* trouble, int stage, int divfree, Scal* sc,
                                        const MlpDev* net, const float* QM, float* pnet, float t_lo, float t_hi,
                                        long long item) {
  limit_item<LM>(K, S, D, BX, BY, flags, trouble, stage, divfree, sc, net, QM, pnet, t_lo, t_hi, item, ens_sm);
}
__device__ __noinline__ void call_dt(const Consts& K, const double* U, long long item, double& ax, double& ay,
                                     Scal* sc) {
  dt_cell_speeds(K, U, item, ax, ay, sc);
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid-wide barrier over the co-resident blocks of a cooperative launch.
// Returns false (in every thread of the block) once any block has timed out.
__device__ bool ens_barrier(const EnsArgs& A, int* s_ok) {
  __syncthreads();
  if (threadIdx.x == 0) {
    cuda::atomic_ref<unsigned int, cuda::thread_scope_device> cnt(A.sync->count);
    cuda::atomic_ref<unsigned int, cuda::thread_scope_device> gen(A.sync->gen);
    cuda::atomic_ref<int, cuda::thread_scope_device> err(A.sync->err);
    const unsigned int g = gen.load(cuda::memory_order_acquire);
    __threadfence();
    if (cnt.fetch_add(1u, cuda::memory_order_acq_rel) == gridDim.x - 1) {
      cnt.store(0u, cuda::memory_order_relaxed);
      gen.fetch_add(1u, cuda::memory_order_release);
    } else {
      const unsigned long long t0 = global_ns();
      while (gen.load(cuda::memory_order_acquire) == g) {
        if (err.load(cuda::memory_order_relaxed) != 0) break;
        if (global_ns() - t0 > A.timeout_ns) {
          err.fetch_or(1, cuda::memory_order_relaxed);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    *s_ok = err.load(cuda::memory_order_relaxed) == 0;
  }
  __syncthreads();
  return *s_ok != 0;
}

// Self-test of the bounded grid barrier: every block but `skip` arrives at
// one barrier; with skip >= 0 the others wait out the limit and record the
// error (nothing else is done, so the device stays usable).
__global__ void __launch_bounds__(ENS_BS) k_barrier_selftest(const __grid_constant__ EnsArgs A, int skip) {
  __shared__ int s_ok;
  if ((int)blockIdx.x == skip) return;
  ens_barrier(A, &s_ok);
}

__device__ __forceinline__ int tile_instance(const int* off, int n, int t) {
  int lo = 0, hi = n;   // off[lo] <= t < off[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= t) lo = mid; else hi = mid;
  }
  return lo;
}

// f(instance index, instance, its constants, first item of the tile, items
// per tile) for the block's tiles of `kind`; GATED skips instances whose step
// has stopped.
template <bool GATED, class F>
__device__ __forceinline__ void for_tiles(const EnsArgs& A, int kind, F&& f) {
  const int* off = A.off + kind * (A.n + 1);
  const int per = A.per_tile[kind];
  for (int t = blockIdx.x; t < A.total[kind]; t += gridDim.x) {
    const int i = tile_instance(off, A.n, t);
    const EnsInst& I = A.inst[i];
    if (GATED && !I.sc->active) continue;
    f(i, I, *I.K, (long long)(t - off[i]) * per, per);
  }
}

__device__ __forceinline__ void phase_bc(const EnsArgs& A, int kind, int zeroB) {
  for_tiles<true>(A, kind, [&](int, const EnsInst& I, const Consts& K, long long base, int per) {
    const long long n = set_bc_items(K);
    for (int k = threadIdx.x; k < per; k += ENS_BS) {
      const long long item = base + k;
      if (item < n) set_bc_item(K, I.U, zeroB, item);
    }
  });
}

template <int LM>
__device__ __forceinline__ void phase_limit(const EnsArgs& A, int stage) {
  for_tiles<true>(A, EK_LIM, [&](int, const EnsInst& I, const Consts& K, long long base, int) {
    call_limit<LM>(K, I.UI, I.U, I.BX, I.BY, I.flags, I.trouble, stage, K.faceb ? 0 : 1, I.sc, A.net, I.QM, I.pnet,
                   A.t_lo, A.t_hi, base + threadIdx.x);
    if (LM == LIM_INFER) __syncthreads();
  });
}

// TVB_Limiter_P2.f90:126-187 + div_free_Balsara for the face-B-limited
// instances: set_bc on the limited state, face-B minmod, div-free.
__device__ __forceinline__ bool phase_faceb(const EnsArgs& A, int* s_ok) {
  phase_bc(A, EK_BCF, 0);
  if (!ens_barrier(A, s_ok)) return false;
  for_tiles<true>(A, EK_FB, [&](int, const EnsInst& I, const Consts& K, long long base, int per) {
    for (int k = threadIdx.x; k < per; k += ENS_BS) faceb_item(K, I.U, I.BX, I.BY, base + k);
  });
  if (!ens_barrier(A, s_ok)) return false;
  for_tiles<true>(A, EK_DF, [&](int, const EnsInst& I, const Consts& K, long long base, int per) {
    const long long n = (long long)K.nx * K.ny;
    for (int k = threadIdx.x; k < per; k += ENS_BS) {
      const long long item = base + k;
      if (item < n) divfree_item(K, I.U, I.BX, I.BY, item);
    }
  });
  return ens_barrier(A, s_ok);
}

// stage 1..3: one RK3 stage of every active instance (stage 1 starts with
// the dt reduction and the time update); stage 0: the start-up limiting of
// RK3.f90:8-12.
template <bool LEARNED>
__global__ void __launch_bounds__(ENS_BS) k_ens_stage(const __grid_constant__ EnsArgs A, int stage) {
  __shared__ int s_ok;
  __shared__ double s_x[ENS_BS], s_y[ENS_BS];
  if (A.sync->err) return;
  if (stage == 0) {
    phase_bc(A, EK_BC, 0);
    if (!ens_barrier(A, &s_ok)) return;
    for_tiles<true>(A, EK_COPY, [&](int, const EnsInst& I, const Consts& K, long long base, int per) {
      const long long n = K.plane * NLIVE;
      for (int k = threadIdx.x; k < per; k += ENS_BS) {
        const long long item = base + k;
        if (item >= n) break;
        const int s = (int)(item / K.plane);
        const long long c = (item - (long long)s * K.plane) + K.plane * (c_live_d[s] + 10 * c_live_n[s]);
        I.UI[c] = I.U[c];
      }
    });
    if (!ens_barrier(A, &s_ok)) return;
  } else if (stage == 1) {
    // calculate_dt: per-instance maxima (exact whatever the order)
    for_tiles<false>(A, EK_DT, [&](int i, const EnsInst& I, const Consts& K, long long base, int per) {
      const long long n = (long long)K.nx * K.ny;
      double ax = 0.0, ay = 0.0;
      for (int k = threadIdx.x; k < per; k += ENS_BS) {
        const long long item = base + k;
        if (item < n) call_dt(K, I.U, item, ax, ay, I.sc);
      }
      __syncthreads();
      s_x[threadIdx.x] = ax;
      s_y[threadIdx.x] = ay;
      __syncthreads();
      for (int s = ENS_BS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
          s_x[threadIdx.x] = max_ign_nan(s_x[threadIdx.x], s_x[threadIdx.x + s]);
          s_y[threadIdx.x] = max_ign_nan(s_y[threadIdx.x], s_y[threadIdx.x + s]);
        }
        __syncthreads();
      }
      if (threadIdx.x == 0) {
        // non-negative doubles order as their bit patterns
        atomicMax(&A.amax[2 * i], (unsigned long long)__double_as_longlong(s_x[0]));
        atomicMax(&A.amax[2 * i + 1], (unsigned long long)__double_as_longlong(s_y[0]));
      }
    });
    if (!ens_barrier(A, &s_ok)) return;
    if (blockIdx.x == 0) {
      for (int i = threadIdx.x; i < A.n; i += ENS_BS) {
        const EnsInst& I = A.inst[i];
        const double ax = __longlong_as_double((long long)A.amax[2 * i]);
        const double ay = __longlong_as_double((long long)A.amax[2 * i + 1]);
        A.amax[2 * i] = 0ull;
        A.amax[2 * i + 1] = 0ull;
        dt_advance(*I.K, ax, ay, I.sc, 1);
      }
    }
    if (!ens_barrier(A, &s_ok)) return;
    phase_bc(A, EK_BC, 0);   // RK3.f90:74
    if (!ens_barrier(A, &s_ok)) return;
  }
  if (stage >= 1) {
    // Lh traces + Riemann, LhEz face and vertex Ez
    for_tiles<true>(A, EK_FX, [&](int, const EnsInst& I, const Consts& K, long long base, int per) {
      const long long n = face_items<0>(K);
      for (int k = threadIdx.x; k < per; k += ENS_BS) {
        const long long item = base + k;
        if (item < n) call_face_x(K, I.U, I.Fxh, I.EzRL, item);
      }
    });
    for_tiles<true>(A, EK_FY, [&](int, const EnsInst& I, const Consts& K, long long base, int per) {
      const long long n = face_items<1>(K);
      for (int k = threadIdx.x; k < per; k += ENS_BS) {
        const long long item = base + k;
        if (item < n) call_face_y(K, I.U, I.Fyh, I.EzUD, item);
      }
    });
    for_tiles<true>(A, EK_VX, [&](int, const EnsInst& I, const Consts& K, long long base, int per) {
      for (int k = threadIdx.x; k < per; k += ENS_BS) {
        const long long item = base + k;
        if (item < K.vplane) call_vertex(K, I.U, I.EzV, item);
      }
    });
    if (!ens_barrier(A, &s_ok)) return;
    // residual + RK combine; dEz + face-B combine
    for_tiles<true>(A, EK_CELL, [&](int, const EnsInst& I, const Consts& K, long long base, int per) {
      for (int k = threadIdx.x; k < per; k += ENS_BS) {
        const long long item = base + k;
        if (item < K.plane)
          call_cell(K, I.U, I.U0, I.UI, I.Fxh, I.Fyh, I.sc, stage, item);
      }
    });
    for_tiles<true>(A, EK_BF, [&](int, const EnsInst& I, const Consts& K, long long base, int per) {
      const long long n = K.fxplane + K.fyplane;
      for (int k = threadIdx.x; k < per; k += ENS_BS) {
        const long long item = base + k;
        if (item < n)
          call_bface(K, I.EzRL, I.EzUD, I.EzV, I.BX, I.BX0, I.BXI, I.BY, I.BY0, I.BYI, I.sc, stage, item);
      }
    });
    if (!ens_barrier(A, &s_ok)) return;
  }
  if (LEARNED && stage <= 1) {   // the network sees the stage-1 pre-limit state
    for_tiles<true>(A, EK_QM, [&](int, const EnsInst& I, const Consts& K, long long base, int per) {
      for (int k = threadIdx.x; k < per; k += ENS_BS) {
        const long long item = base + k;
        if (item < K.plane) call_qmodes(K, I.UI, I.QM, item);
      }
    });
    if (!ens_barrier(A, &s_ok)) return;
  }
  if (!LEARNED) phase_limit<LIM_PLAIN>(A, stage == 0 ? 1 : stage);
  else if (stage <= 1) phase_limit<LIM_INFER>(A, stage == 0 ? 1 : stage);
  else phase_limit<LIM_PNET>(A, stage);
  if (!ens_barrier(A, &s_ok)) return;
  if (A.any_faceb && !phase_faceb(A, &s_ok)) return;
  // RK3.f90:97 / :123 set_bc after stages 1 and 2; after stage 3 (and the
  // start-up limiting) TVB_Limiter_P2's set_bc with div_free's zeroed B modes
  phase_bc(A, EK_BC, (stage == 3 || stage == 0) ? 1 : 0);
}

// ---------------------------------------------------------------------
// Per-phase mode: the same phases as batched launches over all instances,
// one kernel per phase, each with its own register allocation (the item
// bodies inlined as in the single-problem kernels) and the hardware block
// scheduler balancing the tiles; graph-captured like the persistent mode.
__global__ void __launch_bounds__(ENS_BS) k_ep_copy(const __grid_constant__ EnsArgs A) {
  for_tiles<true>(A, EK_COPY, [&](int, const EnsInst& I, const Consts& K, long long base, int per) {
    const long long n = K.plane * NLIVE;
    for (int k = threadIdx.x; k < per; k += ENS_BS) {
      const long long item = base + k;
      if (item >= n) break;
      const int s = (int)(item / K.plane);
      const long long c = (item - (long long)s * K.plane) + K.plane * (c_live_d[s] + 10 * c_live_n[s]);
      I.UI[c] = I.U[c];
    }
  });
}

__global__ void __launch_bounds__(ENS_BS) k_ep_dt(const __grid_constant__ EnsArgs A) {
  __shared__ double s_x[ENS_BS], s_y[ENS_BS];
  for_tiles<false>(A, EK_DT, [&](int i, const EnsInst& I, const Consts& K, long long base, int per) {
    const long long n = (long long)K.nx * K.ny;
    double ax = 0.0, ay = 0.0;
    for (int k = threadIdx.x; k < per; k += ENS_BS) {
      const long long item = base + k;
      if (item < n) dt_cell_speeds(K, I.U, item, ax, ay, I.sc);
    }
    __syncthreads();
    s_x[threadIdx.x] = ax;
    s_y[threadIdx.x] = ay;
    __syncthreads();
    for (int s = ENS_BS / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) {
        s_x[threadIdx.x] = max_ign_nan(s_x[threadIdx.x], s_x[threadIdx.x + s]);
        s_y[threadIdx.x] = max_ign_nan(s_y[threadIdx.x], s_y[threadIdx.x + s]);
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      atomicMax(&A.amax[2 * i], (unsigned long long)__double_as_longlong(s_x[0]));
      atomicMax(&A.amax[2 * i + 1], (unsigned long long)__double_as_longlong(s_y[0]));
    }
  });
}

__global__ void k_ep_dt_final(const __grid_constant__ EnsArgs A) {
  for (int i = threadIdx.x; i < A.n; i += blockDim.x) {
    const EnsInst& I = A.inst[i];
    const double ax = __longlong_as_double((long long)A.amax[2 * i]);
    const double ay = __longlong_as_double((long long)A.amax[2 * i + 1]);
    A.amax[2 * i] = 0ull;
    A.amax[2 * i + 1] = 0ull;
    dt_advance(*I.K, ax, ay, I.sc, 1);
  }
}

__global__ void __launch_bounds__(ENS_BS) k_ep_bc(const __grid_constant__ EnsArgs A, int kind, int zeroB) {
  phase_bc(A, kind, zeroB);
}

__global__ void __launch_bounds__(ENS_BS, 8) k_ep_faces(const __grid_constant__ EnsArgs A) {
  for_tiles<true>(A, EK_FX, [&](int, const EnsInst& I, const Consts& K, long long base, int per) {
    const long long n = face_items<0>(K);
    for (int k = threadIdx.x; k < per; k += ENS_BS) {
      const long long item = base + k;
      if (item < n) face_item<0>(K, I.U, I.Fxh, I.EzRL, item);
    }
  });
  for_tiles<true>(A, EK_FY, [&](int, const EnsInst& I, const Consts& K, long long base, int per) {
    const long long n = face_items<1>(K);
    for (int k = threadIdx.x; k < per; k += ENS_BS) {
      const long long item = base + k;
      if (item < n) face_item<1>(K, I.U, I.Fyh, I.EzUD, item);
    }
  });
  for_tiles<true>(A, EK_VX, [&](int, const EnsInst& I, const Consts& K, long long base, int per) {
    for (int k = threadIdx.x; k < per; k += ENS_BS) {
      const long long item = base + k;
      if (item < K.vplane) vertex_item(K, I.U, I.EzV, item);
    }
  });
}

__global__ void __launch_bounds__(ENS_BS) k_ep_cell(const __grid_constant__ EnsArgs A, int stage) {
  static_assert(ENS_BS == CELL_BS, "cell_item's staging stride is CELL_BS");
  __shared__ __align__(16) double ms[NLIVE * ENS_BS];
  for_tiles<true>(A, EK_CELL, [&](int, const EnsInst& I, const Consts& K, long long base, int per) {
    for (int k = threadIdx.x; k < per; k += ENS_BS) {
      const long long item = base + k;
      if (item < K.plane)
        cell_item<false, GDF_CELL_PAIRS != 0>(K, I.U, I.U0, I.UI, I.Fxh, I.Fyh, nullptr, I.sc, stage, item, ms);
    }
  });
}

__global__ void __launch_bounds__(ENS_BS) k_ep_bface(const __grid_constant__ EnsArgs A, int stage) {
  for_tiles<true>(A, EK_BF, [&](int, const EnsInst& I, const Consts& K, long long base, int per) {
    const long long n = K.fxplane + K.fyplane;
    for (int k = threadIdx.x; k < per; k += ENS_BS) {
      const long long item = base + k;
      if (item < n)
        bface_item(K, I.EzRL, I.EzUD, I.EzV, I.BX, I.BX0, I.BXI, I.BY, I.BY0, I.BYI, nullptr, nullptr, I.sc, stage,
                   item);
    }
  });
}

__global__ void __launch_bounds__(ENS_BS) k_ep_qmodes(const __grid_constant__ EnsArgs A) {
  for_tiles<true>(A, EK_QM, [&](int, const EnsInst& I, const Consts& K, long long base, int per) {
    for (int k = threadIdx.x; k < per; k += ENS_BS) {
      const long long item = base + k;
      if (item < K.plane) qmodes_item(K, I.UI, I.QM, item);
    }
  });
}

template <int LM>
__global__ void __launch_bounds__(ENS_BS) k_ep_limit(const __grid_constant__ EnsArgs A, int stage) {
  extern __shared__ __align__(16) unsigned char lsm[];
  for_tiles<true>(A, EK_LIM, [&](int, const EnsInst& I, const Consts& K, long long base, int) {
    limit_item<LM>(K, I.UI, I.U, I.BX, I.BY, I.flags, I.trouble, stage, K.faceb ? 0 : 1, I.sc, A.net, I.QM, I.pnet,
                   A.t_lo, A.t_hi, base + threadIdx.x, lsm);
    if (LM == LIM_INFER) __syncthreads();
  });
}

__global__ void __launch_bounds__(ENS_BS) k_ep_faceb(const __grid_constant__ EnsArgs A) {
  for_tiles<true>(A, EK_FB, [&](int, const EnsInst& I, const Consts& K, long long base, int per) {
    for (int k = threadIdx.x; k < per; k += ENS_BS) faceb_item(K, I.U, I.BX, I.BY, base + k);
  });
}

__global__ void __launch_bounds__(ENS_BS) k_ep_divfree(const __grid_constant__ EnsArgs A) {
  for_tiles<true>(A, EK_DF, [&](int, const EnsInst& I, const Consts& K, long long base, int per) {
    const long long n = (long long)K.nx * K.ny;
    for (int k = threadIdx.x; k < per; k += ENS_BS) {
      const long long item = base + k;
      if (item < n) divfree_item(K, I.U, I.BX, I.BY, item);
    }
  });
}

thread_local std::string g_ens_err;
int efail(int code, const std::string& m) {
  g_ens_err = m;
  return code;
}
#define ECK(call)                                                                          \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) return efail(GDF_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
  } while (0)

struct InstBufs {
  GdfConfig cfg{};
  Consts K{};
  EnsInst d{};
  double *BXs = nullptr, *BYs = nullptr, *Us = nullptr;   // tuner snapshots
  int32_t* Ts = nullptr;
};

}  // namespace
}  // namespace gdf

using namespace gdf;

struct GdfEnsemble {
  int n = 0;
  std::vector<InstBufs> in;
  cudaStream_t st = nullptr;
  Consts* dK = nullptr;
  EnsInst* dInst = nullptr;
  Scal* sc = nullptr;          // [n]
  Scal* sc_host = nullptr;     // pinned [n]
  Scal* sc_save = nullptr;     // tuner snapshot [n]
  unsigned long long* amax = nullptr;
  EnsSync* sync = nullptr;
  int* off = nullptr;          // [EK_N][n+1]
  MlpDev* net = nullptr;
  int learned = 0;
  float t_lo = 0.5f, t_hi = 0.5f;
  int any_faceb = 0;
  int uploaded = 0;
  // tile shape
  int ctas_per_sm = 0;         // 0: the occupancy limit
  int face_per_thread = 1;     // items per thread of the face/vertex/face-B/set_bc/modes tiles
  int cell_per_thread = 1;     // cells per thread of the residual tiles
  int grid = 0;
  int sms = 0;
  int mode = 1;                // 0: one persistent kernel per stage; 1: one launch per phase (faster here)
  EnsArgs args{};
  cudaGraphExec_t graph = nullptr;
  int graph_ok = 1;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int64_t launches = 0;
  int64_t step_launches = 3;
};

namespace {

size_t uh_sz(const GdfConfig& c) { return (size_t)(c.nx + 2) * (c.ny + 2) * NP * NE * sizeof(double); }
size_t bx_sz(const GdfConfig& c) { return (size_t)(c.nx + 1) * c.ny * 3 * sizeof(double); }
size_t by_sz(const GdfConfig& c) { return (size_t)c.nx * (c.ny + 1) * 3 * sizeof(double); }

size_t ens_smem(int learned) {
  const size_t cell = (size_t)NLIVE * ENS_BS * sizeof(double);
  return learned ? std::max(cell, LIMIT_SMEM_LEARNED) : cell;
}

const void* stage_kernel(int learned) {
  return learned ? (const void*)k_ens_stage<true> : (const void*)k_ens_stage<false>;
}

// tile tables and launch shape for the current tile choice
int ens_layout(GdfEnsemble* e) {
  const int n = e->n;
  EnsArgs& A = e->args;
  const int f = e->face_per_thread, c = e->cell_per_thread;
  const int per[EK_N] = {ENS_BS * f, ENS_BS * f, ENS_BS * f, ENS_BS * f, ENS_BS * f, ENS_BS * f, ENS_BS * c,
                         ENS_BS * f, ENS_BS * f, ENS_BS,     ENS_BS * f, ENS_BS * f, ENS_BS * f * 4};
  std::vector<int> off((size_t)EK_N * (n + 1), 0);
  for (int k = 0; k < EK_N; ++k) {
    A.per_tile[k] = per[k];
    long long acc = 0;
    for (int i = 0; i < n; ++i) {
      const Consts& K = e->in[i].K;
      const long long cells = (long long)K.nx * K.ny;
      long long items = 0;
      switch (k) {
        case EK_DT: items = cells; break;
        case EK_BC: items = set_bc_items(K); break;
        case EK_BCF: items = K.faceb ? set_bc_items(K) : 0; break;
        case EK_FX: items = face_items<0>(K); break;
        case EK_FY: items = face_items<1>(K); break;
        case EK_VX: items = K.vplane; break;
        case EK_CELL: items = K.plane; break;
        case EK_BF: items = K.fxplane + K.fyplane; break;
        case EK_QM: items = K.plane; break;
        case EK_LIM: items = cells; break;
        case EK_FB: items = K.faceb ? K.fxplane + K.fyplane : 0; break;
        case EK_DF: items = K.faceb ? cells : 0; break;
        default: items = K.plane * NLIVE; break;
      }
      off[(size_t)k * (n + 1) + i] = (int)acc;
      acc += (items + per[k] - 1) / per[k];
      if (acc > (1LL << 30)) return efail(GDF_ERR_ARG, "ensemble too large for the tile tables");
    }
    off[(size_t)k * (n + 1) + n] = (int)acc;
    A.total[k] = (int)acc;
  }
  ECK(cudaMemcpyAsync(e->off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice, e->st));
  int occ = 0;
  const size_t smem = ens_smem(e->learned);
  ECK(cudaFuncSetAttribute(stage_kernel(e->learned), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  ECK(cudaFuncSetAttribute(k_ep_limit<LIM_INFER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)LIMIT_SMEM_LEARNED));
  ECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, stage_kernel(e->learned), ENS_BS, smem));
  if (occ < 1) return efail(GDF_ERR_CUDA, "the ensemble stage kernel cannot be resident");
  const int per_sm = e->ctas_per_sm > 0 ? std::min(e->ctas_per_sm, occ) : occ;
  e->grid = per_sm * e->sms;
  A.inst = e->dInst;
  A.off = e->off;
  A.amax = e->amax;
  A.sync = e->sync;
  A.net = e->net;
  // a phase of a large ensemble may legitimately run for a while: 2 s, or
  // 200 ns per cell of the whole ensemble if that is longer
  unsigned long long cells = 0;
  for (const auto& b : e->in) cells += (unsigned long long)b.K.nx * b.K.ny;
  A.timeout_ns = std::max(2000000000ull, 200ull * cells);
  A.n = n;
  A.any_faceb = e->any_faceb;
  A.t_lo = e->t_lo;
  A.t_hi = e->t_hi;
  if (e->graph) {
    cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
  }
  return GDF_OK;
}

int launch_stage_persistent(GdfEnsemble* e, int stage) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)e->grid);
  cfg.blockDim = dim3(ENS_BS);
  cfg.dynamicSmemBytes = ens_smem(e->learned);
  cfg.stream = e->st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaError_t err = e->learned ? cudaLaunchKernelEx(&cfg, k_ens_stage<true>, e->args, stage)
                               : cudaLaunchKernelEx(&cfg, k_ens_stage<false>, e->args, stage);
  e->launches++;
  if (err != cudaSuccess) return efail(GDF_ERR_CUDA, std::string("ensemble stage launch: ") + cudaGetErrorString(err));
  return GDF_OK;
}

// grid of a phase launch: one block per tile (at least one block)
unsigned tiles_of(const EnsArgs& A, int kind) { return (unsigned)std::max(A.total[kind], 1); }

int launch_stage_phases(GdfEnsemble* e, int stage) {
  const EnsArgs& A = e->args;
  cudaStream_t st = e->st;
  int n = 0;
  auto bc = [&](int kind, int zeroB) {
    k_ep_bc<<<tiles_of(A, kind), ENS_BS, 0, st>>>(A, kind, zeroB);
    ++n;
  };
  if (stage == 0) {
    bc(EK_BC, 0);
    k_ep_copy<<<tiles_of(A, EK_COPY), ENS_BS, 0, st>>>(A);
    ++n;
  } else {
    if (stage == 1) {
      k_ep_dt<<<tiles_of(A, EK_DT), ENS_BS, 0, st>>>(A);
      k_ep_dt_final<<<1, 128, 0, st>>>(A);
      n += 2;
      bc(EK_BC, 0);
    }
    const unsigned gf = std::max(tiles_of(A, EK_FX), std::max(tiles_of(A, EK_FY), tiles_of(A, EK_VX)));
    k_ep_faces<<<gf, ENS_BS, 0, st>>>(A);
    k_ep_cell<<<tiles_of(A, EK_CELL), ENS_BS, 0, st>>>(A, stage);
    k_ep_bface<<<tiles_of(A, EK_BF), ENS_BS, 0, st>>>(A, stage);
    n += 3;
  }
  const int ls = stage == 0 ? 1 : stage;
  if (e->learned && stage <= 1) {
    k_ep_qmodes<<<tiles_of(A, EK_QM), ENS_BS, 0, st>>>(A);
    k_ep_limit<LIM_INFER><<<tiles_of(A, EK_LIM), ENS_BS, LIMIT_SMEM_LEARNED, st>>>(A, ls);
    n += 2;
  } else if (e->learned) {
    k_ep_limit<LIM_PNET><<<tiles_of(A, EK_LIM), ENS_BS, 0, st>>>(A, ls);
    ++n;
  } else {
    k_ep_limit<LIM_PLAIN><<<tiles_of(A, EK_LIM), ENS_BS, 0, st>>>(A, ls);
    ++n;
  }
  if (A.any_faceb) {
    bc(EK_BCF, 0);
    k_ep_faceb<<<tiles_of(A, EK_FB), ENS_BS, 0, st>>>(A);
    k_ep_divfree<<<tiles_of(A, EK_DF), ENS_BS, 0, st>>>(A);
    n += 2;
  }
  bc(EK_BC, (stage == 3 || stage == 0) ? 1 : 0);
  e->launches += n;
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return efail(GDF_ERR_CUDA, std::string("ensemble phase launch: ") + cudaGetErrorString(err));
  return GDF_OK;
}

int launch_stage_ens(GdfEnsemble* e, int stage) {
  return e->mode == 1 ? launch_stage_phases(e, stage) : launch_stage_persistent(e, stage);
}

int launch_step_ens(GdfEnsemble* e) {
  for (int s = 1; s <= 3; ++s) {
    int rc = launch_stage_ens(e, s);
    if (rc) return rc;
  }
  return GDF_OK;
}

// One step as a graph of three cooperative kernel nodes; where the runtime
// does not capture cooperative launches, steps are launched directly.
int ensure_graph_ens(GdfEnsemble* e) {
  if (e->graph || !e->graph_ok) return GDF_OK;
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    e->graph_ok = 0;
    return GDF_OK;
  }
  const int64_t l0 = e->launches;
  int rc = launch_step_ens(e);
  e->step_launches = e->launches - l0;
  e->launches = l0;
  cudaError_t ce = cudaStreamEndCapture(e->st, &g);
  if (rc || ce != cudaSuccess || !g) {
    cudaGetLastError();
    if (g) cudaGraphDestroy(g);
    e->graph_ok = 0;
    return GDF_OK;
  }
  ce = cudaGraphInstantiate(&e->graph, g, 0);
  cudaGraphDestroy(g);
  if (ce != cudaSuccess) {
    cudaGetLastError();
    e->graph = nullptr;
    e->graph_ok = 0;
  }
  return GDF_OK;
}

int run_steps(GdfEnsemble* e, int steps) {
  int rc = ensure_graph_ens(e);
  if (rc) return rc;
  for (int k = 0; k < steps; ++k) {
    if (e->graph) {
      ECK(cudaGraphLaunch(e->graph, e->st));
      e->launches += e->step_launches;
    } else if ((rc = launch_step_ens(e))) {
      return rc;
    }
  }
  return GDF_OK;
}

int pull_scal(GdfEnsemble* e) {
  ECK(cudaMemcpyAsync(e->sc_host, e->sc, (size_t)e->n * sizeof(Scal), cudaMemcpyDeviceToHost, e->st));
  ECK(cudaStreamSynchronize(e->st));
  return GDF_OK;
}

int check_health(GdfEnsemble* e) {
  EnsSync s{};
  ECK(cudaMemcpyAsync(&s, e->sync, sizeof(EnsSync), cudaMemcpyDeviceToHost, e->st));
  int rc = pull_scal(e);
  if (rc) return rc;
  if (s.err) return efail(GDF_ERR_TIMEOUT, "an ensemble grid barrier timed out");
  for (int i = 0; i < e->n; ++i)
    if (e->sc_host[i].status)
      return efail(GDF_ERR_NUMERIC, "instance " + std::to_string(i) + ": non-finite or non-positive state or dt");
  return GDF_OK;
}

}  // namespace

extern "C" {

const char* gdf_ens_last_error(void) { return g_ens_err.c_str(); }

int gdf_ens_destroy(GdfEnsemble* e) {
  if (!e) return GDF_OK;
  if (e->st) cudaStreamSynchronize(e->st);
  if (e->graph) cudaGraphExecDestroy(e->graph);
  for (auto& b : e->in) {
    EnsInst& d = b.d;
    void* bufs[] = {d.U, d.U0, d.UI, d.BX, d.BX0, d.BXI, d.BY, d.BY0, d.BYI, d.Fxh, d.Fyh, d.EzRL, d.EzUD,
                    d.EzV, d.flags, d.trouble, d.QM, d.pnet, b.Us, b.BXs, b.BYs, b.Ts};
    for (void* p : bufs)
      if (p) cudaFree(p);
  }
  void* bufs[] = {e->dK, e->dInst, e->sc, e->amax, e->sync, e->off, e->net, e->sc_save};
  for (void* p : bufs)
    if (p) cudaFree(p);
  if (e->sc_host) cudaFreeHost(e->sc_host);
  if (e->ev0) cudaEventDestroy(e->ev0);
  if (e->ev1) cudaEventDestroy(e->ev1);
  if (e->st) cudaStreamDestroy(e->st);
  delete e;
  return GDF_OK;
}

int gdf_ens_create(const GdfConfig* cfgs, int32_t n, GdfEnsemble** out) {
  if (!out || !cfgs || n < 1) return efail(GDF_ERR_ARG, "bad argument");
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    std::string msg;
    int rc = config_error(&cfgs[i], msg);
    if (rc) return efail(rc, "instance " + std::to_string(i) + ": " + msg);
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return efail(GDF_ERR_CUDA, "no CUDA device available");
  }
  GdfEnsemble* e = new GdfEnsemble();
  e->n = n;
  e->in.resize(n);
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&e->sms, cudaDevAttrMultiProcessorCount, dev);
  auto alloc = [&](void** p, size_t bytes) -> bool {
    if (cudaMalloc(p, bytes) != cudaSuccess) return false;
    return cudaMemset(*p, 0, bytes) == cudaSuccess;
  };
  bool ok = cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && alloc((void**)&e->dK, (size_t)n * sizeof(Consts)) && alloc((void**)&e->dInst, (size_t)n * sizeof(EnsInst));
  ok = ok && alloc((void**)&e->sc, (size_t)n * sizeof(Scal)) && alloc((void**)&e->amax, (size_t)2 * n * 8);
  ok = ok && alloc((void**)&e->sync, sizeof(EnsSync)) && alloc((void**)&e->off, (size_t)EK_N * (n + 1) * sizeof(int));
  ok = ok && cudaMallocHost((void**)&e->sc_host, (size_t)n * sizeof(Scal)) == cudaSuccess;
  std::vector<EnsInst> hi(n);
  for (int i = 0; ok && i < n; ++i) {
    InstBufs& b = e->in[i];
    b.cfg = cfgs[i];
    consts_for(cfgs[i], b.K);
    if (i == 0) ok = ok && upload_basis_once(b.K, true) == cudaSuccess;
    if (b.K.faceb) e->any_faceb = 1;
    const Consts& K = b.K;
    const GdfConfig& c = cfgs[i];
    EnsInst& d = b.d;
    const size_t ub = uh_sz(c), bxb = bx_sz(c), byb = by_sz(c);
    ok = ok && alloc((void**)&d.U, ub) && alloc((void**)&d.U0, ub) && alloc((void**)&d.UI, ub);
    ok = ok && alloc((void**)&d.BX, bxb) && alloc((void**)&d.BX0, bxb) && alloc((void**)&d.BXI, bxb);
    ok = ok && alloc((void**)&d.BY, byb) && alloc((void**)&d.BY0, byb) && alloc((void**)&d.BYI, byb);
    ok = ok && alloc((void**)&d.Fxh, (size_t)K.fxplane * NG * NE * 8) && alloc((void**)&d.Fyh, (size_t)K.fyplane * NG * NE * 8);
    ok = ok && alloc((void**)&d.EzRL, (size_t)K.fxplane * NG * 8) && alloc((void**)&d.EzUD, (size_t)K.fyplane * NG * 8) &&
         alloc((void**)&d.EzV, (size_t)K.vplane * 8);
    ok = ok && alloc((void**)&d.flags, (size_t)c.nx * c.ny * 4) && alloc((void**)&d.trouble, (size_t)c.nx * c.ny * 4);
    d.K = e->dK + i;
    d.sc = e->sc + i;
    hi[i] = d;
    if (ok) ok = cudaMemcpy(e->dK + i, &b.K, sizeof(Consts), cudaMemcpyHostToDevice) == cudaSuccess;
  }
  if (!ok) {
    cudaGetLastError();
    gdf_ens_destroy(e);
    return efail(GDF_ERR_NOMEM, "device allocation failed for the ensemble");
  }
  for (int i = 0; i < n; ++i) {
    std::memset(&e->sc_host[i], 0, sizeof(Scal));
    e->sc_host[i].tend = 1e300;
    e->sc_host[i].active = 1;
  }
  ok = cudaMemcpy(e->sc, e->sc_host, (size_t)n * sizeof(Scal), cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(e->dInst, hi.data(), (size_t)n * sizeof(EnsInst), cudaMemcpyHostToDevice) == cudaSuccess;
  if (!ok) {
    gdf_ens_destroy(e);
    return efail(GDF_ERR_CUDA, "initialising the ensemble failed");
  }
  int rc = ens_layout(e);
  if (rc) {
    gdf_ens_destroy(e);
    return rc;
  }
  *out = e;
  return GDF_OK;
}

int gdf_ens_upload(GdfEnsemble* e, int32_t i, const double* uh, const double* bx, const double* by) {
  if (!e || i < 0 || i >= e->n || !uh || !bx || !by) return efail(GDF_ERR_ARG, "bad argument");
  InstBufs& b = e->in[i];
  std::string msg;
  int rc = dead_slot_error(b.cfg, uh, msg);
  if (rc) return efail(rc, msg);
  ECK(cudaMemcpyAsync(b.d.U, uh, uh_sz(b.cfg), cudaMemcpyHostToDevice, e->st));
  ECK(cudaMemcpyAsync(b.d.BX, bx, bx_sz(b.cfg), cudaMemcpyHostToDevice, e->st));
  ECK(cudaMemcpyAsync(b.d.BY, by, by_sz(b.cfg), cudaMemcpyHostToDevice, e->st));
  ECK(cudaStreamSynchronize(e->st));
  e->uploaded = 1;
  return GDF_OK;
}

int gdf_ens_download(GdfEnsemble* e, int32_t i, double* uh, double* bx, double* by) {
  if (!e || i < 0 || i >= e->n) return efail(GDF_ERR_ARG, "bad argument");
  InstBufs& b = e->in[i];
  if (uh) ECK(cudaMemcpyAsync(uh, b.d.U, uh_sz(b.cfg), cudaMemcpyDeviceToHost, e->st));
  if (bx) ECK(cudaMemcpyAsync(bx, b.d.BX, bx_sz(b.cfg), cudaMemcpyDeviceToHost, e->st));
  if (by) ECK(cudaMemcpyAsync(by, b.d.BY, by_sz(b.cfg), cudaMemcpyDeviceToHost, e->st));
  ECK(cudaStreamSynchronize(e->st));
  return GDF_OK;
}

int gdf_ens_set_indicator(GdfEnsemble* e, GdfMlp* m, float t_lo, float t_hi) {
  if (!e || !m) return efail(GDF_ERR_ARG, "null argument");
  if (!(t_lo <= t_hi)) return efail(GDF_ERR_ARG, "t_lo must not exceed t_hi");
  for (int i = 0; i < e->n; ++i)
    if (e->in[i].cfg.detector != GDF_DETECT_LEARNED)
      return efail(GDF_ERR_STATE, "every instance needs detector GDF_DETECT_LEARNED for the learned indicator");
  if (!e->net) ECK(cudaMalloc((void**)&e->net, sizeof(MlpDev)));
  ECK(cudaMemcpy(e->net, gdf_mlp_device_params(m), sizeof(MlpDev), cudaMemcpyDeviceToDevice));
  std::vector<EnsInst> hi(e->n);
  for (int i = 0; i < e->n; ++i) {
    EnsInst& d = e->in[i].d;
    if (!d.QM) ECK(cudaMalloc((void**)&d.QM, (size_t)QMODES * e->in[i].K.plane * sizeof(float)));
    if (!d.pnet) ECK(cudaMalloc((void**)&d.pnet, (size_t)e->in[i].K.nx * e->in[i].K.ny * sizeof(float)));
    hi[i] = d;
  }
  ECK(cudaMemcpy(e->dInst, hi.data(), (size_t)e->n * sizeof(EnsInst), cudaMemcpyHostToDevice));
  e->learned = 1;
  e->t_lo = t_lo;
  e->t_hi = t_hi;
  return ens_layout(e);
}

static int ens_ready(GdfEnsemble* e) {
  if (!e) return efail(GDF_ERR_ARG, "null handle");
  if (!e->uploaded) return efail(GDF_ERR_STATE, "no state uploaded");
  bool any_learned = false;
  for (auto& b : e->in) any_learned = any_learned || b.cfg.detector == GDF_DETECT_LEARNED;
  if (any_learned && !e->learned) return efail(GDF_ERR_STATE, "detector GDF_DETECT_LEARNED needs gdf_ens_set_indicator first");
  return GDF_OK;
}

int gdf_ens_set_time(GdfEnsemble* e, int32_t i, double t, double tend) {
  if (!e || i < -1 || i >= e->n) return efail(GDF_ERR_ARG, "bad argument");
  int rc = pull_scal(e);
  if (rc) return rc;
  for (int k = 0; k < e->n; ++k) {
    if (i >= 0 && k != i) continue;
    e->sc_host[k].t = t;
    e->sc_host[k].tend = tend;
    e->sc_host[k].active = 1;
    e->sc_host[k].status = 0;
  }
  ECK(cudaMemcpyAsync(e->sc, e->sc_host, (size_t)e->n * sizeof(Scal), cudaMemcpyHostToDevice, e->st));
  ECK(cudaStreamSynchronize(e->st));
  return GDF_OK;
}

int gdf_ens_get_time(GdfEnsemble* e, int32_t i, double* t, double* dt, int64_t* steps) {
  if (!e || i < 0 || i >= e->n) return efail(GDF_ERR_ARG, "bad argument");
  int rc = pull_scal(e);
  if (rc) return rc;
  if (t) *t = e->sc_host[i].t;
  if (dt) *dt = e->sc_host[i].dt;
  if (steps) *steps = e->sc_host[i].steps;
  return GDF_OK;
}

int gdf_ens_prepare(GdfEnsemble* e) {
  int rc = ens_ready(e);
  if (rc) return rc;
  if ((rc = gdf_ens_set_time(e, -1, 0.0, 1e300))) return rc;
  if ((rc = launch_stage_ens(e, 0))) return rc;
  return check_health(e);
}

int gdf_ens_advance(GdfEnsemble* e, int32_t steps, int64_t* cell_updates, int32_t* n_active, double* device_ms) {
  int rc = ens_ready(e);
  if (rc) return rc;
  if (steps < 1) return efail(GDF_ERR_ARG, "steps must be positive");
  if ((rc = pull_scal(e))) return rc;
  std::vector<long long> s0(e->n);
  for (int i = 0; i < e->n; ++i) s0[i] = e->sc_host[i].steps;
  if (!e->ev0) {
    ECK(cudaEventCreate(&e->ev0));
    ECK(cudaEventCreate(&e->ev1));
  }
  if ((rc = ensure_graph_ens(e))) return rc;
  ECK(cudaEventRecord(e->ev0, e->st));
  if ((rc = run_steps(e, steps))) return rc;
  ECK(cudaEventRecord(e->ev1, e->st));
  ECK(cudaEventSynchronize(e->ev1));
  float ms = 0.f;
  ECK(cudaEventElapsedTime(&ms, e->ev0, e->ev1));
  if (device_ms) *device_ms = ms;
  rc = check_health(e);
  long long cu = 0;
  int act = 0;
  for (int i = 0; i < e->n; ++i) {
    cu += (e->sc_host[i].steps - s0[i]) * (long long)e->in[i].cfg.nx * e->in[i].cfg.ny;
    if (e->sc_host[i].t < e->sc_host[i].tend) ++act;
  }
  if (cell_updates) *cell_updates = cu;
  if (n_active) *n_active = act;
  return rc;
}

int gdf_ens_set_tiles(GdfEnsemble* e, int32_t ctas_per_sm, int32_t face_per_thread, int32_t cell_per_thread) {
  if (!e || ctas_per_sm < 0 || face_per_thread < 1 || face_per_thread > 64 || cell_per_thread < 1 ||
      cell_per_thread > 64)
    return efail(GDF_ERR_ARG, "bad tile shape");
  e->ctas_per_sm = ctas_per_sm;
  e->face_per_thread = face_per_thread;
  e->cell_per_thread = cell_per_thread;
  return ens_layout(e);
}

int gdf_ens_set_mode(GdfEnsemble* e, int32_t mode) {
  if (!e || (mode != 0 && mode != 1)) return efail(GDF_ERR_ARG, "mode must be 0 (persistent) or 1 (per phase)");
  e->mode = mode;
  if (e->graph) {
    cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
  }
  return GDF_OK;
}

int gdf_ens_get_tiles(GdfEnsemble* e, int32_t* ctas_per_sm, int32_t* face_per_thread, int32_t* cell_per_thread,
                      int32_t* grid, int32_t* graph, int32_t* mode) {
  if (!e) return efail(GDF_ERR_ARG, "null handle");
  if (mode) *mode = e->mode;
  if (ctas_per_sm) *ctas_per_sm = e->grid / std::max(e->sms, 1);
  if (face_per_thread) *face_per_thread = e->face_per_thread;
  if (cell_per_thread) *cell_per_thread = e->cell_per_thread;
  if (grid) *grid = e->grid;
  if (graph) *graph = e->graph ? 1 : 0;
  return GDF_OK;
}

// Times `steps` steps for every candidate (execution mode x tile shape)
// from the same state (saved before, restored after each trial, so the
// ensemble's trajectory is unchanged) and keeps the fastest. ms_out
// (optional, GDF_ENS_TUNE_CANDIDATES entries) receives the candidates' ms per
// step, -1 where not resident: first the persistent mode (blocks per SM 1..4
// x face items 1, 2, 4 x cells 1, 2, 4), then the per-phase mode (face items
// x cells).
int gdf_ens_tune(GdfEnsemble* e, int32_t steps, float* ms_out) {
  int rc = ens_ready(e);
  if (rc) return rc;
  if (steps < 1) return efail(GDF_ERR_ARG, "steps must be positive");
  const int n = e->n;
  for (auto& b : e->in) {
    if (!b.Us) ECK(cudaMalloc((void**)&b.Us, uh_sz(b.cfg)));
    if (!b.BXs) ECK(cudaMalloc((void**)&b.BXs, bx_sz(b.cfg)));
    if (!b.BYs) ECK(cudaMalloc((void**)&b.BYs, by_sz(b.cfg)));
    if (!b.Ts) ECK(cudaMalloc((void**)&b.Ts, (size_t)b.cfg.nx * b.cfg.ny * 4));
  }
  if (!e->sc_save) ECK(cudaMalloc((void**)&e->sc_save, (size_t)n * sizeof(Scal)));
  auto copy_state = [&](bool save) -> int {
    for (auto& b : e->in) {
      const EnsInst& d = b.d;
      ECK(cudaMemcpyAsync(save ? b.Us : d.U, save ? d.U : b.Us, uh_sz(b.cfg), cudaMemcpyDeviceToDevice, e->st));
      ECK(cudaMemcpyAsync(save ? b.BXs : d.BX, save ? d.BX : b.BXs, bx_sz(b.cfg), cudaMemcpyDeviceToDevice, e->st));
      ECK(cudaMemcpyAsync(save ? b.BYs : d.BY, save ? d.BY : b.BYs, by_sz(b.cfg), cudaMemcpyDeviceToDevice, e->st));
      ECK(cudaMemcpyAsync(save ? b.Ts : d.trouble, save ? d.trouble : b.Ts, (size_t)b.cfg.nx * b.cfg.ny * 4,
                          cudaMemcpyDeviceToDevice, e->st));
    }
    ECK(cudaMemcpyAsync(save ? e->sc_save : e->sc, save ? e->sc : e->sc_save, (size_t)n * sizeof(Scal),
                        cudaMemcpyDeviceToDevice, e->st));
    return GDF_OK;
  };
  if ((rc = copy_state(true))) return rc;
  if (!e->ev0) {
    ECK(cudaEventCreate(&e->ev0));
    ECK(cudaEventCreate(&e->ev1));
  }
  int occ = 0;
  ECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, stage_kernel(e->learned), ENS_BS, ens_smem(e->learned)));
  const int faces[3] = {1, 2, 4}, cells[3] = {1, 2, 4};
  float best = 1e30f;
  int bmode = 0, bc = 0, bf = 1, bcell = 1, k = 0;
  for (int mode = 0; mode <= 1; ++mode)
    for (int cps = 1; cps <= (mode == 0 ? 4 : 1); ++cps)
      for (int fi = 0; fi < 3; ++fi)
        for (int ci = 0; ci < 3; ++ci, ++k) {
          if (mode == 0 && cps > occ) {
            if (ms_out) ms_out[k] = -1.f;
            continue;
          }
          if ((rc = gdf_ens_set_mode(e, mode))) return rc;
          if ((rc = gdf_ens_set_tiles(e, mode == 0 ? cps : 0, faces[fi], cells[ci]))) return rc;
          if ((rc = run_steps(e, 1))) return rc;   // warm-up (and graph capture)
          if ((rc = copy_state(false))) return rc;
          ECK(cudaEventRecord(e->ev0, e->st));
          if ((rc = run_steps(e, steps))) return rc;
          ECK(cudaEventRecord(e->ev1, e->st));
          ECK(cudaEventSynchronize(e->ev1));
          float ms = 0.f;
          ECK(cudaEventElapsedTime(&ms, e->ev0, e->ev1));
          ms /= (float)steps;
          if (ms_out) ms_out[k] = ms;
          if ((rc = check_health(e))) return rc;
          if ((rc = copy_state(false))) return rc;
          if (ms < best) {
            best = ms;
            bmode = mode; bc = mode == 0 ? cps : 0; bf = faces[fi]; bcell = cells[ci];
          }
        }
  if ((rc = gdf_ens_set_mode(e, bmode))) return rc;
  if ((rc = gdf_ens_set_tiles(e, bc, bf, bcell))) return rc;
  ECK(cudaStreamSynchronize(e->st));
  return GDF_OK;
}

int64_t gdf_ens_kernel_launches(GdfEnsemble* e) { return e ? e->launches : -1; }

// Runs k_barrier_selftest on `blocks` co-resident blocks with the barrier's
// time limit set to limit_ns: *timed_out receives 1 when some block gave up
// waiting (expected when skip_block names one of them), else 0.
int gdf_ens_barrier_selftest(int32_t blocks, int32_t skip_block, uint64_t limit_ns, int32_t* timed_out) {
  if (blocks < 1 || blocks > 1024 || !timed_out || limit_ns == 0) return efail(GDF_ERR_ARG, "bad argument");
  EnsSync* sy = nullptr;
  ECK(cudaMalloc((void**)&sy, sizeof(EnsSync)));
  ECK(cudaMemset(sy, 0, sizeof(EnsSync)));
  EnsArgs A{};
  A.sync = sy;
  A.timeout_ns = limit_ns;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)blocks);
  cfg.blockDim = dim3(ENS_BS);
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaError_t err = cudaLaunchKernelEx(&cfg, k_barrier_selftest, A, (int)skip_block);
  if (err == cudaSuccess) err = cudaDeviceSynchronize();
  EnsSync h{};
  if (err == cudaSuccess) err = cudaMemcpy(&h, sy, sizeof(EnsSync), cudaMemcpyDeviceToHost);
  cudaFree(sy);
  if (err != cudaSuccess) return efail(GDF_ERR_CUDA, std::string("barrier self-test: ") + cudaGetErrorString(err));
  *timed_out = h.err ? 1 : 0;
  return GDF_OK;
}

}  // extern "C"
