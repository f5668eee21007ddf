// gdf_init.cu -- initial data on the device (init_data.f90:21-121 with the
// problem includes), so a large grid or an ensemble starts without a host
// projection and a host-to-device copy of the whole state.
//
// The values equal gdf_init_data's (gdf_host.cpp) bit for bit: every
// operation is written with the _rn intrinsics in the host code's order, so
// no contraction can change a rounding in either library build, and the
// only transcendental function of the benchmark problems (Orszag-Tang's
// sine) is read from tables the host fills with its own libm at the
// quadrature coordinates, which are computed by the same expressions on
// both sides. The vortex of init1.txt uses exp of a two-dimensional
// argument and runs on the device's exp (within one or two units in the
// last place of the host's).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gdf.h"

namespace gdf {

namespace {

constexpr int NGI = 5, NEI = 8;

__constant__ double c_lam[NGI] = {-0.9061798459386639927976269, -0.5384693101056830910363144, 0,
                                  0.5384693101056830910363144, 0.9061798459386639927976269};
__constant__ double c_wt[NGI] = {0.2369268850561890875142640, 0.4786286704993664680412915,
                                 0.5688888888888888888888889, 0.4786286704993664680412915,
                                 0.2369268850561890875142640};

__device__ __forceinline__ double M(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double A(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double S(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double D(double a, double b) { return __ddiv_rn(a, b); }

struct InitArgs {
  int problem, nx, ny;
  double g, xa, ya, hx, hy, hx1, hy1;
  double prm[8];
  double c13, mm[6], mmE[3];   // 1/3 and the mass diagonals, as the host computes them
  const double* sx;    // Orszag-Tang: sin(x) at the Gauss x-coordinates, [i-1][a]
  const double* s2x;   // sin(2x) at the same points
  const double* sy;    // sin(y) at the Gauss y-coordinates, [j-1][b]
};

// Point values of the conserved variables (gdf_host.cpp Init::conserved).
// For Orszag-Tang the caller passes sin(x), sin(2x), sin(y) of the point.
__device__ void conserved_at(const InitArgs& P, double x, double y, double snx, double sn2x, double sny, double* U) {
  double rho = 0, v1 = 0, v2 = 0, v3 = 0, p = 0, B1 = 0, B2 = 0, B3 = 0;
  const double* prm = P.prm;
  switch (P.problem) {
    case GDF_PROB_VORTEX: {
      const double pi = 3.141592653589793115997963468544185161590576171875;   // 4 atan(1) in FP64
      const double r2 = A(M(x, x), M(y, y));
      const double e = exp(M(0.5, S(1.0, r2)));
      p = S(1.0, M(D(r2, M(8.0, M(pi, pi))), exp(S(1.0, r2))));
      rho = 1;
      const double c = D(1.0, M(2.0, pi));
      v1 = S(1.0, M(M(c, y), e));
      v2 = A(1.0, M(M(c, x), e));
      B1 = M(M(-c, y), e);
      B2 = M(M(c, x), e);
      break;
    }
    case GDF_PROB_ORSZAG_TANG:
      p = P.g;
      rho = M(P.g, P.g);
      v1 = -sny;
      v2 = snx;
      B1 = -sny;
      B2 = sn2x;
      break;
    case GDF_PROB_ROTOR: {
      const double cx = prm[0], cy = prm[1], r0 = prm[2], r1 = prm[3], rin = prm[4], u0 = prm[5];
      const double dx = S(x, cx), dy = S(y, cy);
      const double r = __dsqrt_rn(A(M(dx, dx), M(dy, dy)));
      const double f = D(S(r1, r), S(r1, r0));
      if (r < r0) {
        rho = rin;
        v1 = D(M(-u0, dy), r0);
        v2 = D(M(u0, dx), r0);
      } else if (r < r1) {
        rho = A(1.0, M(S(rin, 1.0), f));
        v1 = D(M(M(-f, u0), dy), r);
        v2 = D(M(M(f, u0), dx), r);
      } else {
        rho = 1.0;
      }
      p = prm[6];
      B1 = prm[7];
      break;
    }
    case GDF_PROB_BLAST: {
      const double dx = S(x, prm[0]), dy = S(y, prm[1]);
      const double r = __dsqrt_rn(A(M(dx, dx), M(dy, dy)));
      p = (r <= prm[2]) ? prm[3] : prm[4];
      rho = prm[5];
      B1 = prm[6];
      B2 = prm[7];
      break;
    }
    default: {   // cloud shock
      const double ex = S(x, 1.4), ey = S(y, 0.5);
      const double r = __dsqrt_rn(A(M(ex, ex), M(ey, ey)));
      if (x <= 1.2) {
        rho = 3.88968; v3 = -0.05234; p = 14.2641; B1 = 1; B3 = 3.9353;
      } else {
        rho = (r >= 0.18) ? 1.0 : 5.0; v1 = -3.3156; p = 0.04; B1 = 1; B3 = 1;
      }
      break;
    }
  }
  const double g1 = S(P.g, 1.0);
  U[0] = rho;
  U[1] = M(rho, v1);
  U[2] = M(rho, v2);
  U[3] = M(rho, v3);
  if (P.problem == GDF_PROB_CLOUD_SHOCK)
    U[4] = A(A(D(p, g1), M(M(0.5, rho), A(A(M(v1, v1), M(v2, v2)), M(v3, v3)))),
             M(0.5, A(A(M(B1, B1), M(B2, B2)), M(B3, B3))));
  else
    U[4] = A(A(D(p, g1), M(M(0.5, rho), A(M(v1, v1), M(v2, v2)))), M(0.5, A(M(B1, B1), M(B2, B2))));
  U[5] = B1;
  U[6] = B2;
  U[7] = B3;
}

__device__ __forceinline__ double phi6(const InitArgs& P, int a, int b, int d) {
  const double c13 = P.c13;
  const double li = c_lam[a], lj = c_lam[b];
  switch (d) {
    case 0: return 1.0;
    case 1: return li;
    case 2: return lj;
    case 3: return S(M(li, li), c13);
    case 4: return M(li, lj);
    default: return S(M(lj, lj), c13);
  }
}

// One interior cell: the L2 projection of init_data.f90:37-63 (modes 1..6,
// the projection mask of :43), or the point value at the centre for the
// piecewise-constant start of :92-121.
__global__ void k_init_cells(const InitArgs P, int shock, double* __restrict__ U) {
  const long long item = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (item >= (long long)P.nx * P.ny) return;
  const int i = (int)(item % P.nx) + 1, j = (int)(item / P.nx) + 1;
  const long long nx2 = P.nx + 2, plane = nx2 * (P.ny + 2);
  const long long c = i + nx2 * j;
  const double xc = A(P.xa, M(S((double)i, 0.5), P.hx));
  const double yc = A(P.ya, M(S((double)j, 0.5), P.hy));
  if (shock) {
    double Uv[NEI];
    conserved_at(P, xc, yc, 0, 0, 0, Uv);
#pragma unroll
    for (int n = 0; n < NEI; ++n) U[c + plane * (10 * n)] = Uv[n];
    return;
  }
  double acc[6][NEI];
#pragma unroll
  for (int d = 0; d < 6; ++d)
#pragma unroll
    for (int n = 0; n < NEI; ++n) acc[d][n] = 0.0;
  // the reference's order: d outermost, then the 5x5 points; the point
  // values are evaluated once per point (they do not depend on d)
  double Up[NGI * NGI][NEI];
#pragma unroll 1
  for (int a = 0; a < NGI; ++a)
#pragma unroll 1
    for (int b = 0; b < NGI; ++b) {
      const double x = A(xc, M(P.hx1, c_lam[a])), y = A(yc, M(P.hy1, c_lam[b]));
      double snx = 0, sn2x = 0, sny = 0;
      if (P.problem == GDF_PROB_ORSZAG_TANG) {
        snx = P.sx[(i - 1) * NGI + a];
        sn2x = P.s2x[(i - 1) * NGI + a];
        sny = P.sy[(j - 1) * NGI + b];
      }
      conserved_at(P, x, y, snx, sn2x, sny, Up[a * NGI + b]);
    }
#pragma unroll
  for (int d = 0; d < 6; ++d)
#pragma unroll 1
    for (int a = 0; a < NGI; ++a)
#pragma unroll 1
      for (int b = 0; b < NGI; ++b) {
        const double f = M(M(c_wt[a], c_wt[b]), phi6(P, a, b, d));
#pragma unroll
        for (int n = 0; n < NEI; ++n) acc[d][n] = A(acc[d][n], M(f, Up[a * NGI + b][n]));
      }
#pragma unroll
  for (int d = 0; d < 6; ++d)
#pragma unroll
    for (int n = 0; n < NEI; ++n) U[c + plane * (d + 10 * n)] = D(M(0.25, acc[d][n]), P.mm[d]);
}

// Face B: x faces (i = 0..Nx, j = 1..Ny) then y faces (i = 1..Nx,
// j = 0..Ny), init_data.f90:65-90 (three Legendre modes) or :92-121.
__global__ void k_init_faces(const InitArgs P, int shock, double* __restrict__ BX, double* __restrict__ BY) {
  const long long item = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nfx = (long long)(P.nx + 1) * P.ny, nfy = (long long)P.nx * (P.ny + 1);
  if (item >= nfx + nfy) return;
  const double c13 = P.c13;
  const bool xf = item < nfx;
  int i, j;
  if (xf) {
    i = (int)(item % (P.nx + 1));
    j = (int)(item / (P.nx + 1)) + 1;
  } else {
    const long long k = item - nfx;
    i = (int)(k % P.nx) + 1;
    j = (int)(k / P.nx);
  }
  double* out = xf ? BX : BY;
  const long long o = xf ? item : item - nfx;
  const long long fp = xf ? nfx : nfy;
  double Uv[NEI];
  if (shock) {
    if (xf) {
      const double x = A(P.xa, M((double)i, P.hx)), y = A(P.ya, M(S((double)j, 0.5), P.hy));
      conserved_at(P, x, y, 0, 0, 0, Uv);
      out[o] = Uv[5];
    } else {
      const double x = A(P.xa, M(S((double)i, 0.5), P.hx)), y = A(P.ya, M((double)j, P.hy));
      conserved_at(P, x, y, 0, 0, 0, Uv);
      out[o] = Uv[6];
    }
    out[o + fp] = 0.0;
    out[o + 2 * fp] = 0.0;
    return;
  }
  double Bq[NGI];
#pragma unroll 1
  for (int q = 0; q < NGI; ++q) {
    double snx = 0, sn2x = 0, sny = 0;
    if (xf) {
      const double yc = A(P.ya, M(S((double)j, 0.5), P.hy));
      const double x = A(P.xa, M((double)i, P.hx)), y = A(yc, M(P.hy1, c_lam[q]));
      if (P.problem == GDF_PROB_ORSZAG_TANG) sny = P.sy[(j - 1) * NGI + q];
      conserved_at(P, x, y, snx, sn2x, sny, Uv);
      Bq[q] = Uv[5];
    } else {
      const double xc = A(P.xa, M(S((double)i, 0.5), P.hx));
      const double x = A(xc, M(P.hx1, c_lam[q])), y = A(P.ya, M((double)j, P.hy));
      if (P.problem == GDF_PROB_ORSZAG_TANG) sn2x = P.s2x[(i - 1) * NGI + q];
      conserved_at(P, x, y, snx, sn2x, sny, Uv);
      Bq[q] = Uv[6];
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double acc = 0.0;
#pragma unroll
    for (int q = 0; q < NGI; ++q) {
      const double l = c_lam[q];
      const double e = d == 0 ? 1.0 : d == 1 ? l : S(M(l, l), c13);
      acc = A(acc, M(M(M(0.5, c_wt[q]), e), Bq[q]));
    }
    out[o + fp * d] = D(acc, P.mmE[d]);
  }
}

}  // namespace

// Host part: parameters as gdf_init_data takes them (default_params of
// gdf_host.cpp when params is null), the Orszag-Tang sine tables, the two
// launches on `st`. U must hold the config's uh extents and be zero
// outside the slots the kernels write (ghosts, modes 7..10): the caller
// clears it first.
int init_data_device(const GdfConfig& cfg, int problem, const double* params, double* U, double* BX, double* BY,
                     cudaStream_t st, std::string& err) {
  InitArgs P{};
  P.problem = problem;
  P.nx = cfg.nx;
  P.ny = cfg.ny;
  P.g = cfg.gamma;
  P.xa = cfg.xa;
  P.ya = cfg.ya;
  P.hx = (cfg.xb - cfg.xa) / cfg.nx;
  P.hy = (cfg.yb - cfg.ya) / cfg.ny;
  P.hx1 = 0.5 * P.hx;
  P.hy1 = 0.5 * P.hy;
  P.c13 = 1.0 / 3.0;
  const double mm[6] = {1, 1.0 / 3.0, 1.0 / 3.0, 4.0 / 45.0, 1.0 / 9.0, 4.0 / 45.0};
  const double mmE[3] = {1, 1.0 / 3.0, 4.0 / 45.0};
  std::memcpy(P.mm, mm, sizeof(mm));
  std::memcpy(P.mmE, mmE, sizeof(mmE));
  if (params) {
    std::memcpy(P.prm, params, sizeof(P.prm));
  } else {
    const double pi = 4 * std::atan(1.0);
    if (problem == GDF_PROB_ROTOR) {
      const double v[8] = {0.5, 0.5, 0.1, 0.115, 10.0, 2.0, 1.0, 5.0 / std::sqrt(4 * pi)};
      std::memcpy(P.prm, v, sizeof(v));
    } else if (problem == GDF_PROB_BLAST) {
      const double v[8] = {0, 0, 0.1, 1000, 0.1, 1.0, 100.0 / std::sqrt(8 * pi), 100.0 / std::sqrt(8 * pi)};
      std::memcpy(P.prm, v, sizeof(v));
    }
  }
  const int shock = (problem == GDF_PROB_BLAST || problem == GDF_PROB_CLOUD_SHOCK) ? 1 : 0;
  double* tab = nullptr;
  if (problem == GDF_PROB_ORSZAG_TANG) {
    // sin at the quadrature coordinates, evaluated as gdf_host.cpp does
    const double lam[NGI] = {-0.9061798459386639927976269, -0.5384693101056830910363144, 0,
                             0.5384693101056830910363144, 0.9061798459386639927976269};
    std::vector<double> h((size_t)(2 * cfg.nx + cfg.ny) * NGI);
    double* sx = h.data();
    double* s2x = sx + (size_t)cfg.nx * NGI;
    double* sy = s2x + (size_t)cfg.nx * NGI;
    for (int i = 1; i <= cfg.nx; ++i) {
      const double Xc = cfg.xa + (i - 0.5) * P.hx;
      for (int a = 0; a < NGI; ++a) {
        const double x = Xc + P.hx1 * lam[a];
        sx[(i - 1) * NGI + a] = std::sin(x);
        s2x[(i - 1) * NGI + a] = std::sin(2.0 * x);
      }
    }
    for (int j = 1; j <= cfg.ny; ++j) {
      const double Yc = cfg.ya + (j - 0.5) * P.hy;
      for (int b = 0; b < NGI; ++b) sy[(j - 1) * NGI + b] = std::sin(Yc + P.hy1 * lam[b]);
    }
    cudaError_t e = cudaMallocAsync((void**)&tab, h.size() * sizeof(double), st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(tab, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);   // h leaves scope
    if (e != cudaSuccess) {
      if (tab) cudaFreeAsync(tab, st);
      err = std::string("init tables: ") + cudaGetErrorString(e);
      return GDF_ERR_CUDA;
    }
    P.sx = tab;
    P.s2x = tab + (size_t)cfg.nx * NGI;
    P.sy = tab + (size_t)2 * cfg.nx * NGI;
  }
  const long long ncell = (long long)cfg.nx * cfg.ny;
  const long long nface = (long long)(cfg.nx + 1) * cfg.ny + (long long)cfg.nx * (cfg.ny + 1);
  k_init_cells<<<(unsigned)((ncell + 127) / 128), 128, 0, st>>>(P, shock, U);
  k_init_faces<<<(unsigned)((nface + 127) / 128), 128, 0, st>>>(P, shock, BX, BY);
  cudaError_t e = cudaGetLastError();
  if (tab) cudaFreeAsync(tab, st);
  if (e != cudaSuccess) {
    err = std::string("init launch: ") + cudaGetErrorString(e);
    return GDF_ERR_CUDA;
  }
  return GDF_OK;
}

}  // namespace gdf
