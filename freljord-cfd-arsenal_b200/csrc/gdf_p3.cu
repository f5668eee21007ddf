// gdf_p3.cu -- the k = 3 variant of the GDF MHD method (MPI_BalsaraP3/main.f90)
// on sm_100a: P3 modal solution in 15 slots (84 of them live), four-mode
// face B, the ten-stage SSP Runge-Kutta of RK4 (main.f90:1315-1431), the
// characteristic TVB limiter with the P3 reconstruction on every cell and
// Balsara's divergence-free reconstruction, behind the C ABI of
// include/gdf_p3.h.
//
// One item per thread, in the reference's operation order (the product
// build has no FMA contraction), so every value equals the reference
// arithmetic. Per stage:
//   k3_set_bc          set_bc (main.f90:1574-1867) on one block
//   k3_face<0>, <1>    face traces, fluxes, eigenvalueMm, Riemann solve
//                      (main.f90:2006-2230) -> Fxh, Fyh
//   k3_vertex          corner traces, 2-D vertex solver (:2271-2307) -> EzV
//   k3_cell<KIND>      volume + surface integrals, mass matrix (:1913-2002,
//                      :2234-2264), fused with the stage's RK combination
//   k3_bface<KIND>     dBx, dBy (:2309-2335) fused with the combination
//   k3_faceb_limit     face-B limiting of TVB_Limiter (:3427-3478)
//   k3_limit           TVB_Limiter's cell part (:3298-3424) fused with
//                      div_free_Balsara (:3108-3233)
// and per step k3_dt_partial + k3_dt_final (calculate_dt, :1469-1541, and
// the clamp to tend, :1338-1343). A step is captured once as a CUDA graph.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gdf_p3.h"
#include "gdf_p3_basis.h"
#include "gdf_physics.cuh"

namespace gdf {
int set_last_error(int code, const char* msg);
}

namespace gdf3 {

using gdf::fmax2;
using gdf::fmin2;
using gdf::Phys;
using gdf::sgn1;
using gdf::Side;
using gdf::sq;

// ------------------------------------------------------------ live slots ---
// 84 slots per cell: modes 1-10 of every variable, plus modes 11 and 14 of
// the cell Bx (a40, a13) and 12 and 15 of the cell By (b31, b04) that
// div_free_Balsara writes (main.f90:3199-3226). Every other slot is zero
// throughout the method and is not stored.
constexpr int NS3 = 84;
__host__ __device__ constexpr int slot3(int n, int d) {
  return d < NQ3 ? (n < 5 ? NQ3 * n + d : n == 5 ? 50 + d : n == 6 ? 62 + d : 74 + d)
                 : (n == 5 ? (d == 10 ? 60 : d == 13 ? 61 : -1) : n == 6 ? (d == 11 ? 72 : d == 14 ? 73 : -1) : -1);
}

// stage kinds of k3_cell / k3_bface (the combinations of RK4, main.f90:1353-1419)
constexpr int KIND_LH = 0;     // du only (gdf_p3_lh)
constexpr int KIND_FIRST = 1;  // stage 1: T = U + dt/6 du, UII = U
constexpr int KIND_STAGE = 2;  // stages 2-4, 6-9: T = U + dt/6 du
constexpr int KIND_FIVE = 3;   // stage 5: UII = 0.04 UII + 0.36 (U + dt/6 du); U = 15 UII - 5 (U + dt/6 du)
constexpr int KIND_LAST = 4;   // stage 10: T = UII + 0.6 T + dt/10 du

struct K3 {
  int nx, ny, nx2, ny2;
  long long plane, fxplane, fyplane, vplane, bxplane, byplane;
  double hx, hy, cxs, cys, rxy, ryx, Mh2x, Mh2y, beta, change_tol, cfl;
  int bc_r, bc_l, bc_u, bc_d;
  Phys P;
  BasisP3 B;
};

struct Scal3 {
  double t, dt, tend, c6, c10;
  double ax, ay;       // the block's largest |u_n +- c_f| (gdf_p3_step_speeds)
  int active;          // 0 once t has reached tend: the step's kernels return at once
  int status;          // bit 0: non-positive density or non-finite energy / dt seen
  long long steps;
};

__device__ __forceinline__ long long gtid() { return (long long)blockIdx.x * blockDim.x + threadIdx.x; }

// ------------------------------------------------------------- physics -----
// Lh's point flux (main.f90:1942-1969, 2021-2164): the first component is
// rho*u (rho*v), not the momentum itself; K carries the w term on every side.
template <int DIR>
__device__ __forceinline__ void flux3(const Side& s, double* F) {
  const double S = s.p + 0.5 * s.BB;
  const double T = s.E + S;
  const double K = s.u * s.B1 + s.v * s.B2 + s.w * s.B3;
  if (DIR == 0) {
    F[0] = s.rho * s.u;
    F[1] = s.rho * sq(s.u) + S - sq(s.B1);
    F[2] = s.rho * s.u * s.v - s.B1 * s.B2;
    F[3] = s.rho * s.u * s.w - s.B1 * s.B3;
    F[4] = T * s.u - K * s.B1;
    F[5] = 0.0;
    F[6] = s.u * s.B2 - s.v * s.B1;
    F[7] = s.u * s.B3 - s.w * s.B1;
  } else {
    F[0] = s.rho * s.v;
    F[1] = s.rho * s.u * s.v - s.B1 * s.B2;
    F[2] = s.rho * sq(s.v) + S - sq(s.B2);
    F[3] = s.rho * s.v * s.w - s.B2 * s.B3;
    F[4] = T * s.v - K * s.B2;
    F[5] = s.v * s.B1 - s.u * s.B2;
    F[6] = 0.0;
    F[7] = s.v * s.B3 - s.w * s.B2;
  }
}

// one face point: uL = trace of the cell on the -normal side (the
// reference's UL1), uR = the +normal side (UR1); Fh = Fhat1
template <int DIR>
__device__ __forceinline__ void face_flux3(const Phys& P, const double* uL, const double* uR, double* Fh) {
  Side L, R;
  gdf::make_side(P, uL, L);
  gdf::make_side(P, uR, R);
  double fL[NE], fR[NE];
  flux3<DIR>(L, fL);
  flux3<DIR>(R, fR);
  double a1, a2, b1, b2;
  gdf::side_speeds(P, L, DIR, a1, a2);   // SRmax, SRmin (from the left cell's trace)
  gdf::side_speeds(P, R, DIR, b1, b2);   // SLmax, SLmin
  const double SR = fmax2(a1, b1);
  const double SL = fmin2(a2, b2);
  if (P.flux == 1) {
    const double a = fmax2(fabs(SR), fabs(SL));
#pragma unroll
    for (int n = 0; n < NE; ++n) Fh[n] = 0.5 * (fR[n] + fL[n] - a * (R.U[n] - L.U[n]));
  } else if (P.flux == 2) {
    if (SR < 0) {
#pragma unroll
      for (int n = 0; n < NE; ++n) Fh[n] = fR[n];
    } else if (SL > 0) {
#pragma unroll
      for (int n = 0; n < NE; ++n) Fh[n] = fL[n];
    } else {
      const double den = SR - SL, sls = SL * SR;
#pragma unroll
      for (int n = 0; n < NE; ++n) Fh[n] = (SR * fL[n] - SL * fR[n] + sls * (R.U[n] - L.U[n])) / den;
    }
  } else {
    double Ust[NE];
    if (P.flux == 3)
      gdf::hllcd_flux<false>(P, R, L, fR, fL, SR, SL, DIR, Fh, Ust);
    else
      gdf::hllcd_flux<true>(P, R, L, fR, fL, SR, SL, DIR, Fh, Ust);
  }
}

// the eight values of cell c at a point with basis values phi[15]:
// sum over the modes from zero in mode order (dead slots add nothing)
__device__ __forceinline__ void trace3(const K3& K, const double* __restrict__ U, long long c, const double* phi,
                                       double* out) {
#pragma unroll
  for (int n = 0; n < NE; ++n) {
    double acc = 0.0;
#pragma unroll
    for (int d = 0; d < NP3; ++d) {
      const int s = slot3(n, d);
      if (s >= 0) acc = acc + __ldg(&U[c + K.plane * s]) * phi[d];
    }
    out[n] = acc;
  }
}

// the same from a thread's copy of its cell's 84 slots in shared memory
// (slot s at sm[s * 64])
__device__ __forceinline__ void trace3s(const double* sm, const double* phi, double* out) {
#pragma unroll
  for (int n = 0; n < NE; ++n) {
    double acc = 0.0;
#pragma unroll
    for (int d = 0; d < NP3; ++d) {
      const int s = slot3(n, d);
      if (s >= 0) acc = acc + sm[s * 64] * phi[d];
    }
    out[n] = acc;
  }
}

// column-major 8x8 times vector, summed from zero in column order (MATMUL)
__device__ __forceinline__ void mv8(const double* A, const double* x, double* y) {
#pragma unroll
  for (int r = 0; r < NE; ++r) {
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < NE; ++k) acc = acc + A[r + 8 * k] * x[k];
    y[r] = acc;
  }
}

// minmod / minmodB with beta (main.f90:3952-3979, 3983-4001)
__device__ __forceinline__ double minmod3(double a, double b, double c, double Mh2, double beta) {
  if (fabs(a) <= Mh2) return a;
  const double s = (sgn1(a) + sgn1(b) + sgn1(c)) / 3.0;
  if (fabs(s) == 1) return s * fmin2(fmin2(fabs(a), beta * fabs(b)), beta * fabs(c));
  return 0.0;
}

// --------------------------------------------------------------- set_bc ----
// Ghost cells: the x ghosts over every row, then the y ghosts over every
// column (corners from the y pass), i.e. ghost (i, j) takes cell (si, sj)
// with si, sj the x and y sources. One thread per (slot, ghost cell); then
// the face fields' ghost rows (Bx) and columns (By), one thread per mode.
__global__ void __launch_bounds__(128) k3_set_bc(const __grid_constant__ K3 K, double* __restrict__ U,
                                                 double* __restrict__ BX, double* __restrict__ BY,
                                                 const Scal3* __restrict__ sc) {
  if (sc && !sc->active) return;
  const long long t = gtid();
  const long long nring = 2LL * K.ny2 + 2LL * K.nx;
  const long long nbx = 2LL * (K.nx + 1), nby = 2LL * (K.ny + 1);
  if (t < nring * NS3) {
    const int s = (int)(t / nring);
    const long long g = t - (long long)s * nring;
    int i, j;
    if (g < 2LL * K.ny2) {
      j = (int)(g >> 1);
      i = (g & 1) ? K.nx + 1 : 0;
    } else {
      const long long r = g - 2LL * K.ny2;
      i = (int)(r >> 1) + 1;
      j = (r & 1) ? K.ny + 1 : 0;
    }
    auto src = [](int q, int n, bool lo_periodic, bool hi_periodic) {
      if (q == 0) return lo_periodic ? n : 1;
      if (q == n + 1) return hi_periodic ? 1 : n;
      return q;
    };
    const int si = src(i, K.nx, K.bc_l == GDF_BC_PERIODIC, K.bc_r == GDF_BC_PERIODIC);
    const int sj = src(j, K.ny, K.bc_d == GDF_BC_PERIODIC, K.bc_u == GDF_BC_PERIODIC);
    U[i + (long long)K.nx2 * j + K.plane * s] = U[si + (long long)K.nx2 * sj + K.plane * s];
    return;
  }
  long long r = t - nring * NS3;
  if (r < nbx * NB3) {
    const int d = (int)(r / nbx);
    r -= (long long)d * nbx;
    const int i = (int)(r >> 1);
    const bool up = r & 1;
    const int j = up ? K.ny + 1 : 0;
    const int sj = up ? (K.bc_u == GDF_BC_PERIODIC ? 1 : K.ny) : (K.bc_d == GDF_BC_PERIODIC ? K.ny : 1);
    BX[i + (long long)(K.nx + 1) * j + K.bxplane * d] = BX[i + (long long)(K.nx + 1) * sj + K.bxplane * d];
    return;
  }
  r -= nbx * NB3;
  if (r < nby * NB3) {
    const int d = (int)(r / nby);
    r -= (long long)d * nby;
    const int j = (int)(r >> 1);
    const bool right = r & 1;
    const int i = right ? K.nx + 1 : 0;
    const int si = right ? (K.bc_r == GDF_BC_PERIODIC ? 1 : K.nx) : (K.bc_l == GDF_BC_PERIODIC ? K.nx : 1);
    BY[i + (long long)K.nx2 * j + K.byplane * d] = BY[si + (long long)K.nx2 * j + K.byplane * d];
  }
}

// ---------------------------------------------------------------- faces ----
// item = g * (faces) + face: a warp covers consecutive faces at one point.
template <int DIR>
__global__ void __launch_bounds__(128) k3_face(const __grid_constant__ K3 K, const double* __restrict__ U,
                                               double* __restrict__ Fh, const Scal3* __restrict__ sc) {
  if (sc && !sc->active) return;
  const long long nf = DIR == 0 ? K.fxplane : K.fyplane;
  const long long item = gtid();
  if (item >= nf * NG) return;
  const int g = (int)(item / nf);
  const long long f = item - (long long)g * nf;
  long long cl, cr;
  if (DIR == 0) {
    const int i = (int)(f % (K.nx + 1)), j = (int)(f / (K.nx + 1)) + 1;
    cl = i + (long long)K.nx2 * j;
    cr = cl + 1;
  } else {
    const int i = (int)(f % K.nx) + 1, j = (int)(f / K.nx);
    cl = i + (long long)K.nx2 * j;
    cr = cl + K.nx2;
  }
  double uL[NE], uR[NE], F[NE];
  trace3(K, U, cl, DIR == 0 ? K.B.phiGR[g] : K.B.phiGU[g], uL);
  trace3(K, U, cr, DIR == 0 ? K.B.phiGL[g] : K.B.phiGD[g], uR);
  face_flux3<DIR>(K.P, uL, uR, F);
#pragma unroll
  for (int n = 0; n < NE; ++n) Fh[(long long)(g * NE + n) * nf + f] = F[n];
}

// -------------------------------------------------------------- vertices ---
__global__ void __launch_bounds__(128) k3_vertex(const __grid_constant__ K3 K, const double* __restrict__ U,
                                                 double* __restrict__ EzV, const Scal3* __restrict__ sc) {
  if (sc && !sc->active) return;
  const long long v = gtid();
  if (v >= K.vplane) return;
  const int i = (int)(v % (K.nx + 1)), j = (int)(v / (K.nx + 1));
  const long long c = i + (long long)K.nx2 * j;
  double URU[NE], ULU[NE], URD[NE], ULD[NE];
  trace3(K, U, c + K.nx2 + 1, K.B.phiLD, URU);   // ULD of cell (i+1, j+1)
  trace3(K, U, c + K.nx2, K.B.phiRD, ULU);       // URD of cell (i, j+1)
  trace3(K, U, c + 1, K.B.phiLU, URD);           // ULU of cell (i+1, j)
  trace3(K, U, c, K.B.phiRU, ULD);               // URU of cell (i, j)
  EzV[v] = gdf::vertex_ez(K.P, URU, ULU, URD, ULD);
}

// ------------------------------------------------------------------ cells --
// du of one interior cell: each du(d, n) is one chain of additions in the
// reference's order (volume points i1 then j1, x faces, y faces, then the
// mass matrix), held in registers; then the stage's combination.
// GDF_P3_CELL_SMEM: each thread first copies its cell's 84 slots to shared
// memory and evaluates the 25 points from there (same values)
#ifndef GDF_P3_CELL_SMEM
#define GDF_P3_CELL_SMEM 0
#endif
constexpr size_t CELL_SMEM = GDF_P3_CELL_SMEM ? (size_t)NS3 * 64 * sizeof(double) : 0;

template <int KIND>
__global__ void __launch_bounds__(64) k3_cell(const __grid_constant__ K3 K, double* __restrict__ U,
                                              double* __restrict__ T, double* __restrict__ UII,
                                              const double* __restrict__ Fxh, const double* __restrict__ Fyh,
                                              const Scal3* __restrict__ sc) {
  if (sc && !sc->active) return;
  const long long item = gtid();
  if (item >= (long long)K.nx * K.ny) return;
  const int i = (int)(item % K.nx) + 1, j = (int)(item / K.nx) + 1;
  const long long c = i + (long long)K.nx2 * j;
#if GDF_P3_CELL_SMEM
  extern __shared__ double cell_sm[];
  double* my = cell_sm + threadIdx.x;
#pragma unroll 4
  for (int q = 0; q < NS3; ++q) my[q * 64] = U[c + K.plane * q];
#endif
  double du[NQ3][NE];
#pragma unroll
  for (int d = 0; d < NQ3; ++d)
#pragma unroll
    for (int n = 0; n < NE; ++n) du[d][n] = 0.0;
  // volume integral (main.f90:1924-2003)
#pragma unroll 1
  for (int a = 0; a < NG; ++a)
#pragma unroll 1
    for (int b = 0; b < NG; ++b) {
      double uG[NE];
#if GDF_P3_CELL_SMEM
      trace3s(my, K.B.phiG[a][b], uG);
#else
      trace3(K, U, c, K.B.phiG[a][b], uG);
#endif
      Side s;
      gdf::make_side(K.P, uG, s);
      double Fx[NE], Fy[NE];
      flux3<0>(s, Fx);
      flux3<1>(s, Fy);
      const double wab = 0.25 * K.B.weight[a] * K.B.weight[b];
#pragma unroll
      for (int d = 1; d < NQ3; ++d) {
        const double px = K.B.phixG[a][b][d], py = K.B.phiyG[a][b][d];
#pragma unroll
        for (int n = 0; n < NE; ++n) du[d][n] = du[d][n] + wab * (Fx[n] * px + Fy[n] * py);
      }
    }
  // surface integrals (main.f90:2232-2258): x faces of the cell, then y faces
  {
    const long long fr = i + (long long)(K.nx + 1) * (j - 1), fl = fr - 1;
#pragma unroll 1
    for (int g = 0; g < NG; ++g) {
      const double cw = K.cxs * K.B.weight[g];
      double Fr[NE], Fl[NE];
#pragma unroll
      for (int n = 0; n < NE; ++n) {
        Fr[n] = Fxh[(long long)(g * NE + n) * K.fxplane + fr];
        Fl[n] = Fxh[(long long)(g * NE + n) * K.fxplane + fl];
      }
#pragma unroll
      for (int d = 0; d < NQ3; ++d) {
        const double pr = K.B.phiGR[g][d], pl = K.B.phiGL[g][d];
#pragma unroll
        for (int n = 0; n < NE; ++n) du[d][n] = du[d][n] - cw * (Fr[n] * pr - Fl[n] * pl);
      }
    }
  }
  {
    const long long fu = (i - 1) + (long long)K.nx * j, fd = fu - K.nx;
#pragma unroll 1
    for (int g = 0; g < NG; ++g) {
      const double cw = K.cys * K.B.weight[g];
      double Fu[NE], Fd[NE];
#pragma unroll
      for (int n = 0; n < NE; ++n) {
        Fu[n] = Fyh[(long long)(g * NE + n) * K.fyplane + fu];
        Fd[n] = Fyh[(long long)(g * NE + n) * K.fyplane + fd];
      }
#pragma unroll
      for (int d = 0; d < NQ3; ++d) {
        const double pu = K.B.phiGU[g][d], pd = K.B.phiGD[g][d];
#pragma unroll
        for (int n = 0; n < NE; ++n) du[d][n] = du[d][n] - cw * (Fu[n] * pu - Fd[n] * pd);
      }
    }
  }
#pragma unroll
  for (int d = 0; d < NQ3; ++d)
#pragma unroll
    for (int n = 0; n < NE; ++n) du[d][n] = du[d][n] / K.B.mm[d];
  // the stage's combination over the 84 live slots (du = 0 beyond mode 10)
  const double c6 = KIND == KIND_LH ? 0.0 : sc->c6;
  const double c10 = KIND == KIND_LAST ? sc->c10 : 0.0;
#pragma unroll
  for (int n = 0; n < NE; ++n)
#pragma unroll
    for (int d = 0; d < NP3; ++d) {
      const int s = slot3(n, d);
      if (s < 0) continue;
      const double dd = d < NQ3 ? du[d][n] : 0.0;
      const long long q = c + K.plane * s;
      if (KIND == KIND_LH) {
        T[q] = dd;
      } else if (KIND == KIND_FIRST) {
        const double u = U[q];
        UII[q] = u;
        T[q] = u + c6 * dd;
      } else if (KIND == KIND_STAGE) {
        T[q] = U[q] + c6 * dd;
      } else if (KIND == KIND_FIVE) {
        const double uI = U[q] + c6 * dd;
        const double uII = 0.04 * UII[q] + 0.36 * uI;
        UII[q] = uII;
        U[q] = 15 * uII - 5 * uI;
      } else {
        T[q] = UII[q] + 0.6 * T[q] + c10 * dd;
      }
    }
}

// ------------------------------------------------------------- face B ------
// dBx on x faces (i 0..nx, j 1..ny), dBy on y faces (i 1..nx, j 0..ny) from
// EzRL = -Fxhat(7), EzUD = Fyhat(6) and the vertex Ez; then the combination
// of the face arrays (same kinds as k3_cell).
template <int KIND>
__global__ void __launch_bounds__(128) k3_bface(const __grid_constant__ K3 K, const double* __restrict__ Fxh,
                                                const double* __restrict__ Fyh, const double* __restrict__ EzV,
                                                double* __restrict__ BX, double* __restrict__ BXT,
                                                double* __restrict__ BXII, double* __restrict__ BY,
                                                double* __restrict__ BYT, double* __restrict__ BYII,
                                                const Scal3* __restrict__ sc) {
  if (sc && !sc->active) return;
  long long t = gtid();
  double db[NB3];
  double *A, *AT, *AII;
  long long q, pl;
  if (t < K.fxplane) {
    const int i = (int)(t % (K.nx + 1)), j = (int)(t / (K.nx + 1)) + 1;
    const double e1 = EzV[i + (long long)(K.nx + 1) * j], e0 = EzV[i + (long long)(K.nx + 1) * (j - 1)];
#pragma unroll
    for (int d = 0; d < NB3; ++d) {
      double acc = 0.0;
#pragma unroll
      for (int g = 0; g < NG; ++g)
        acc = acc + 0.5 * K.B.weight[g] * (-Fxh[(long long)(g * NE + 6) * K.fxplane + t]) * K.B.EzyG[g][d];
      db[d] = (acc - e1 * K.B.EzR[d] / K.hy + e0 * K.B.EzL[d] / K.hy) / K.B.mmE[d];
    }
    A = BX; AT = BXT; AII = BXII;
    q = i + (long long)(K.nx + 1) * j;
    pl = K.bxplane;
  } else {
    t -= K.fxplane;
    if (t >= K.fyplane) return;
    const int i = (int)(t % K.nx) + 1, j = (int)(t / K.nx);
    const double e1 = EzV[i + (long long)(K.nx + 1) * j], e0 = EzV[(i - 1) + (long long)(K.nx + 1) * j];
#pragma unroll
    for (int d = 0; d < NB3; ++d) {
      double acc = 0.0;
#pragma unroll
      for (int g = 0; g < NG; ++g)
        acc = acc - 0.5 * K.B.weight[g] * Fyh[(long long)(g * NE + 5) * K.fyplane + t] * K.B.EzxG[g][d];
      db[d] = (acc + e1 * K.B.EzR[d] / K.hx - e0 * K.B.EzL[d] / K.hx) / K.B.mmE[d];
    }
    A = BY; AT = BYT; AII = BYII;
    q = i + (long long)K.nx2 * j;
    pl = K.byplane;
  }
  const double c6 = KIND == KIND_LH ? 0.0 : sc->c6;
  const double c10 = KIND == KIND_LAST ? sc->c10 : 0.0;
#pragma unroll
  for (int d = 0; d < NB3; ++d) {
    const long long r = q + pl * d;
    if (KIND == KIND_LH) {
      AT[r] = db[d];
    } else if (KIND == KIND_FIRST) {
      const double u = A[r];
      AII[r] = u;
      AT[r] = u + c6 * db[d];
    } else if (KIND == KIND_STAGE) {
      AT[r] = A[r] + c6 * db[d];
    } else if (KIND == KIND_FIVE) {
      const double uI = A[r] + c6 * db[d];
      const double uII = 0.04 * AII[r] + 0.36 * uI;
      AII[r] = uII;
      A[r] = 15 * uII - 5 * uI;
    } else {
      AT[r] = AII[r] + 0.6 * AT[r] + c10 * db[d];
    }
  }
}

// ------------------------------------------------------- face-B limiting ---
// main.f90:3430-3478: modes 2-4 of every face rebuilt from the TVB-limited
// end differences; mode 1 kept. Reads Fin (ghost rows/columns set), writes Fout.
__global__ void __launch_bounds__(128) k3_faceb_limit(const __grid_constant__ K3 K, const double* __restrict__ BXin,
                                                      const double* __restrict__ BYin, double* __restrict__ BXout,
                                                      double* __restrict__ BYout, const Scal3* __restrict__ sc) {
  if (sc && !sc->active) return;
  long long t = gtid();
  const double* Fin;
  double* Fout;
  long long q, step, pl;
  double Mh2;
  if (t < K.fxplane) {
    const int i = (int)(t % (K.nx + 1)), j = (int)(t / (K.nx + 1)) + 1;
    q = i + (long long)(K.nx + 1) * j;
    step = K.nx + 1;
    pl = K.bxplane;
    Fin = BXin;
    Fout = BXout;
    Mh2 = K.Mh2y;
  } else {
    t -= K.fxplane;
    if (t >= K.fyplane) return;
    const int i = (int)(t % K.nx) + 1, j = (int)(t / K.nx);
    q = i + (long long)K.nx2 * j;
    step = 1;
    pl = K.byplane;
    Fin = BYin;
    Fout = BYout;
    Mh2 = K.Mh2x;
  }
  const double a0 = Fin[q];
  const double dRM = Fin[q + step] - a0;
  const double dLM = a0 - Fin[q - step];
  const double b2 = Fin[q + pl], b3 = Fin[q + 2 * pl], b4 = Fin[q + 3 * pl];
  const double dR = b2 + (2.0 / 3.0) * b3 + (2.0 / 5.0) * b4;
  const double dL = b2 - (2.0 / 3.0) * b3 + (2.0 / 5.0) * b4;
  const double R1 = minmod3(dR, dRM, dLM, Mh2, K.beta);
  const double L1 = minmod3(dL, dRM, dLM, Mh2, K.beta);
  Fout[q] = a0;
  Fout[q + pl] = 7.0 / 10.0 * b2 - 3.0 / 25.0 * b4 + 3.0 / 20.0 * (R1 + L1);
  Fout[q + 2 * pl] = 0.75 * (R1 - L1);
  Fout[q + 3 * pl] = -(7.0 / 4.0) * b2 + 3.0 / 10.0 * b4 + 7.0 / 8.0 * (R1 + L1);
}

// ------------------------------------------------------------- limiter -----
// One direction of TVB_Limiter's characteristic part: the face slopes X1
// (mean to + face) and X2 (- face to mean) limited against the mean
// differences DR, DL in the characteristic variables of the cell mean,
// back in conserved variables as Y1, Y2. The left eigenvectors are built
// and used in the four products with L (main.f90:3319-3321, 3337), then
// the right ones for the two products with R: one 8x8 matrix live at a
// time, the same products and sums as with both (this eigenmatrix has no
// identity fallback that would tie R to L).
__device__ __forceinline__ void char_limit(const Phys& P, int dir, double rho, double u1, double u2, double u3,
                                           const double* m0, const double* DR, const double* DL, const double* X1,
                                           const double* X2, double Mh2, double beta, double* Y1, double* Y2) {
  gdf::EigFrame f;
  gdf::eigen_frame(P, dir, rho, u1, u2, u3, m0[4], m0[5], m0[6], m0[7], f);
  double mod1[NE], mod2[NE];
  {
    double L[64], t1[NE], t2[NE], tu1[NE], tu2[NE];
    gdf::eigen_left(dir, f, rho, u1, u2, u3, m0[5], m0[6], m0[7], L);
    mv8(L, DR, t1);
    mv8(L, DL, t2);
    mv8(L, X1, tu1);
    mv8(L, X2, tu2);
#pragma unroll
    for (int k = 0; k < NE; ++k) {
      mod1[k] = minmod3(tu1[k], t1[k], t2[k], Mh2, beta);
      mod2[k] = minmod3(tu2[k], t1[k], t2[k], Mh2, beta);
    }
  }
  double R[64];
  gdf::eigen_right(dir, f, rho, u1, u2, u3, m0[5], m0[6], m0[7], R);
  mv8(R, mod1, Y1);
  mv8(R, mod2, Y2);
}

// TVB_Limiter's cell part (main.f90:3295-3428) on the pre-limit state S
// (ghosts set) for one interior cell, then div_free_Balsara for it from the
// limited face fields; writes the cell's 84 slots of D. flags (may be NULL):
// bits 0-7 changed variables, 8-15 those rebuilt with the P3 reconstruction.
__global__ void __launch_bounds__(64) k3_limit(const __grid_constant__ K3 K, const double* __restrict__ S,
                                               double* __restrict__ D, const double* __restrict__ BX,
                                               const double* __restrict__ BY, int32_t* __restrict__ flags,
                                               const Scal3* __restrict__ sc) {
  if (sc && !sc->active) return;
  const long long item = gtid();
  if (item >= (long long)K.nx * K.ny) return;
  const int i = (int)(item % K.nx) + 1, j = (int)(item / K.nx) + 1;
  const long long c = i + (long long)K.nx2 * j, pl = K.plane;
  auto at = [&](long long cc, int n, int d) { return S[cc + pl * slot3(n, d)]; };
  double m0[NE];
#pragma unroll
  for (int n = 0; n < NE; ++n) m0[n] = at(c, n, 0);
  const double rhoij = m0[0];
  const double u1 = m0[1] / rhoij, u2 = m0[2] / rhoij, u3 = m0[3] / rhoij;
  double DR[NE], DL[NE], X1[NE], X2[NE];
  double Rm[NE], Lm[NE], Um[NE], Dm[NE];
  unsigned change = 0;
  // x direction (main.f90:3312-3345)
#pragma unroll
  for (int n = 0; n < NE; ++n) {
    DR[n] = at(c + 1, n, 0) - m0[n];
    DL[n] = m0[n] - at(c - 1, n, 0);
    const double a2 = at(c, n, 1), a4 = at(c, n, 3), a7 = at(c, n, 6);
    X1[n] = a2 + (2.0 / 3.0) * a4 + (2.0 / 5.0) * a7;
    X2[n] = a2 - (2.0 / 3.0) * a4 + (2.0 / 5.0) * a7;
  }
  char_limit(K.P, 0, rhoij, u1, u2, u3, m0, DR, DL, X1, X2, K.Mh2x, K.beta, Rm, Lm);
#pragma unroll
  for (int n = 0; n < NE; ++n)
    if (fabs(Rm[n] - X1[n]) > K.change_tol || fabs(Lm[n] - X2[n]) > K.change_tol) change |= 1u << n;
  // y direction (main.f90:3347-3380)
#pragma unroll
  for (int n = 0; n < NE; ++n) {
    DR[n] = at(c + K.nx2, n, 0) - m0[n];
    DL[n] = m0[n] - at(c - K.nx2, n, 0);
    const double a3 = at(c, n, 2), a6 = at(c, n, 5), a10 = at(c, n, 9);
    X1[n] = a3 + (2.0 / 3.0) * a6 + (2.0 / 5.0) * a10;
    X2[n] = a3 - (2.0 / 3.0) * a6 + (2.0 / 5.0) * a10;
  }
  char_limit(K.P, 1, rhoij, u1, u2, u3, m0, DR, DL, X1, X2, K.Mh2y, K.beta, Um, Dm);
#pragma unroll
  for (int n = 0; n < NE; ++n)
    if (fabs(Um[n] - X1[n]) > K.change_tol || fabs(Dm[n] - X2[n]) > K.change_tol) change |= 1u << n;
  // reconstruction (main.f90:3382-3425); the cell B's modes 2 and 3 only
  // feed omega of the divergence-free rebuild below
  unsigned p3 = 0;
  double om_by2 = at(c, 6, 1), om_bx3 = at(c, 5, 2);
#pragma unroll
  for (int n = 0; n < NE; ++n) {
    if (!(change & (1u << n))) {
      if (n != 5 && n != 6) {
#pragma unroll
        for (int d = 0; d < NQ3; ++d) D[c + pl * slot3(n, d)] = at(c, n, d);
      }
      continue;
    }
    const double a2 = at(c, n, 1), a3 = at(c, n, 2), a7 = at(c, n, 6), a10 = at(c, n, 9);
    const double m2 = 7.0 / 10.0 * a2 - 3.0 / 25.0 * a7 + 3.0 / 20.0 * (Rm[n] + Lm[n]);
    const double m3 = 7.0 / 10.0 * a3 - 3.0 / 25.0 * a10 + 3.0 / 20.0 * (Um[n] + Dm[n]);
    const double u0 = m0[n];
    const bool keep = fabs(m2) < fabs(at(c + 1, n, 0) - u0) && fabs(m2) < fabs(u0 - at(c - 1, n, 0)) &&
                      fabs(m3) < fabs(at(c + K.nx2, n, 0) - u0) && fabs(m3) < fabs(u0 - at(c - K.nx2, n, 0));
    double out[NQ3];
#pragma unroll
    for (int d = 0; d < NQ3; ++d) out[d] = 0.0;
    out[0] = u0;
    if (keep) {
      p3 |= 1u << n;
      out[1] = m2;
      out[2] = m3;
      out[3] = 3.0 / 4.0 * (Rm[n] - Lm[n]);
      out[6] = -(7.0 / 4.0) * a2 + 3.0 / 10.0 * a7 + 7.0 / 8.0 * (Rm[n] + Lm[n]);
      out[5] = 3.0 / 4.0 * (Um[n] - Dm[n]);
      out[9] = -(7.0 / 4.0) * a3 + 3.0 / 10.0 * a10 + 7.0 / 8.0 * (Um[n] + Dm[n]);
    } else {
      out[1] = 0.5 * (Rm[n] + Lm[n]);
      out[2] = 0.5 * (Um[n] + Dm[n]);
    }
    if (n == 6) om_by2 = out[1];
    if (n == 5) om_bx3 = out[2];
    if (n != 5 && n != 6) {
#pragma unroll
      for (int d = 0; d < NQ3; ++d) D[c + pl * slot3(n, d)] = out[d];
    }
  }
  if (flags) flags[item] = (int32_t)(change | (p3 << 8));
  // div_free_Balsara (main.f90:3119-3225)
  const double omega = om_by2 - om_bx3;
  const long long bxr = i + (long long)(K.nx + 1) * j, bxl = bxr - 1;
  const long long byu = i + (long long)K.nx2 * j, byd = byu - K.nx2;
  const long long px = K.bxplane, py = K.byplane;
  const double a0R = BX[bxr], a1R = BX[bxr + px], a2R = BX[bxr + 2 * px], a3R = BX[bxr + 3 * px];
  const double a0L = BX[bxl], a1L = BX[bxl + px], a2L = BX[bxl + 2 * px], a3L = BX[bxl + 3 * px];
  const double b0U = BY[byu], b1U = BY[byu + py], b2U = BY[byu + 2 * py], b3U = BY[byu + 3 * py];
  const double b0D = BY[byd], b1D = BY[byd + py], b2D = BY[byd + 2 * py], b3D = BY[byd + 3 * py];
  const double rxy = K.rxy, ryx = K.ryx;
  const double S1 = (1.0 / 2.0) * (a1R + a1L);
  const double S2 = (1.0 / 2.0) * (b1U + b1D);
  const double a03 = (1.0 / 2.0) * (a3R + a3L);
  const double b30 = (1.0 / 2.0) * (b3U + b3D);
  const double a13 = (1.0 / 2.0) * (a3R - a3L);
  const double b31 = (1.0 / 2.0) * (b3U - b3D);
  const double a02 = (1.0 / 2.0) * (a2R + a2L);
  const double b20 = (1.0 / 2.0) * (b2U + b2D);
  const double a12 = (1.0 / 2.0) * (a2R - a2L);
  const double b21 = (1.0 / 2.0) * (b2U - b2D);
  const double a11 = (1.0 / 2.0) * (a1R - a1L);
  const double b11 = (1.0 / 2.0) * (b1U - b1D);
  const double a40 = -((1.0 / 4.0) * rxy * b31);
  const double b04 = -((1.0 / 4.0) * ryx * a13);
  const double a30 = -((1.0 / 3.0) * rxy * b21);
  const double b03 = -((1.0 / 3.0) * ryx * a12);
  const double a10 = (1.0 / 2.0) * (a0R - a0L) - (2.0 / 5.0) * a30;
  const double b01 = (1.0 / 2.0) * (b0U - b0D) - (2.0 / 5.0) * b03;
  const double a20 = -((1.0 / 2.0) * rxy * (b11 - 3.0 / 5.0 * b31)) + (6.0 / 7.0) * a40;
  const double b02 = -((1.0 / 2.0) * ryx * (a11 - 3.0 / 5.0 * a13)) + (6.0 / 7.0) * b04;
  const double a00 = (1.0 / 2.0) * (a0R + a0L) - (2.0 / 3.0) * a20 - (8.0 / 35.0) * a40;
  const double b00 = (1.0 / 2.0) * (b0U + b0D) - (2.0 / 3.0) * b02 - (8.0 / 35.0) * b04;
  const double a01 = (S1 * ryx + S2 - omega) / (1 + ryx);
  const double b10 = a01 + omega;
  const double a21 = (3.0 / 2.0) * (S1 - a01);
  const double b12 = (3.0 / 2.0) * (S2 - b10);
  const double A[12] = {a00, a10, a01, a20, a11, a02, a30, a21, a12, a03, a40, a13};
  const double Bv[12] = {b00, b10, b01, b20, b11, b02, b30, b21, b12, b03, b31, b04};
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    D[c + pl * (50 + k)] = A[k];
    D[c + pl * (62 + k)] = Bv[k];
  }
}

// ---------------------------------------------------------------- dt -------
constexpr int DT_BS = 256;

__device__ __forceinline__ double max_skip_nan(double a, double b) { return b > a ? b : a; }

// calculate_dt (main.f90:1475-1490) for the interior cells of one block:
// the largest |u_n +- c_f| of the cell averages in x and y (NaN-skipping,
// as the reference's comparisons); non-positive density or non-finite
// energy flags sc->status.
__global__ void __launch_bounds__(DT_BS) k3_dt_partial(const __grid_constant__ K3 K, const double* __restrict__ U,
                                                       double* __restrict__ part, Scal3* __restrict__ sc, int step) {
  if (step == 1 && !sc->active) return;
  __shared__ double sx[DT_BS], sy[DT_BS];
  const long long item = gtid();
  double ax = 0.0, ay = 0.0;
  if (item < (long long)K.nx * K.ny) {
    const int i = (int)(item % K.nx) + 1, j = (int)(item / K.nx) + 1;
    const long long c = i + (long long)K.nx2 * j;
    double Uv[NE];
#pragma unroll
    for (int n = 0; n < NE; ++n) Uv[n] = U[c + K.plane * slot3(n, 0)];
    double a1, a2;
    gdf::fast_speeds(K.P, Uv, 0, a1, a2);
    ax = max_skip_nan(max_skip_nan(ax, fabs(a1)), fabs(a2));
    gdf::fast_speeds(K.P, Uv, 1, a1, a2);
    ay = max_skip_nan(max_skip_nan(ay, fabs(a1)), fabs(a2));
    if (!(Uv[0] > 0.0) || !isfinite(Uv[4])) atomicOr(&sc->status, 1);
  }
  sx[threadIdx.x] = ax;
  sy[threadIdx.x] = ay;
  __syncthreads();
  for (int s = DT_BS / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      sx[threadIdx.x] = max_skip_nan(sx[threadIdx.x], sx[threadIdx.x + s]);
      sy[threadIdx.x] = max_skip_nan(sy[threadIdx.x], sy[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = sx[0];
    part[2 * blockIdx.x + 1] = sy[0];
  }
}

// dt from the grid's largest speeds, RK4's clamp and t update
// (main.f90:1338-1343) and the stage coefficients dt/6, dt/10
__device__ __forceinline__ void advance_t(const K3& K, double ax, double ay, Scal3* __restrict__ sc) {
  double dt = K.cfl / (ax / K.hx + ay / K.hy);
  double t = sc->t;
  if (t + dt > sc->tend) {
    dt = sc->tend - t;
    t = sc->tend;
  } else {
    t = t + dt;
  }
  if (!(dt > 0.0) || !isfinite(dt)) sc->status |= 1;
  sc->dt = dt;
  sc->t = t;
  sc->c6 = dt / 6.0;
  sc->c10 = dt / 10.0;
  sc->active = 1;
  sc->steps += 1;
}

// step 0: dt only (gdf_p3_dt); 1: a time step (advance_t); 2: the block's
// speeds only (gdf_p3_step_speeds, for a maximum over the blocks of a grid)
__global__ void __launch_bounds__(DT_BS) k3_dt_final(const __grid_constant__ K3 K, const double* __restrict__ part,
                                                     int nblocks, Scal3* __restrict__ sc, int step) {
  __shared__ double sx[DT_BS], sy[DT_BS];
  if (step == 1 && !(sc->t < sc->tend)) {
    if (threadIdx.x == 0) sc->active = 0;
    return;
  }
  double ax = 0.0, ay = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += DT_BS) {
    ax = max_skip_nan(ax, part[2 * b]);
    ay = max_skip_nan(ay, part[2 * b + 1]);
  }
  sx[threadIdx.x] = ax;
  sy[threadIdx.x] = ay;
  __syncthreads();
  for (int s = DT_BS / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      sx[threadIdx.x] = max_skip_nan(sx[threadIdx.x], sx[threadIdx.x + s]);
      sy[threadIdx.x] = max_skip_nan(sy[threadIdx.x], sy[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  if (step == 2) {
    sc->ax = sx[0];
    sc->ay = sy[0];
    return;
  }
  if (!step) {
    sc->dt = K.cfl / (sx[0] / K.hx + sy[0] / K.hy);
    return;
  }
  advance_t(K, sx[0], sy[0], sc);
}

// a step of a block from the speeds of the whole grid (gdf_p3_step_begin)
__global__ void k3_dt_set(const __grid_constant__ K3 K, double ax, double ay, Scal3* __restrict__ sc) {
  if (!(sc->t < sc->tend)) {
    sc->active = 0;
    return;
  }
  advance_t(K, ax, ay, sc);
}

// calculate_umax and calculate_totaldiv's per-cell terms (main.f90:1433-1465,
// 3235-3279): |rho mean| and the cell's sum of 0.25 w w |div B| over its
// Gauss points; the host folds them in the reference's cell order.
__global__ void __launch_bounds__(128) k3_diag(const __grid_constant__ K3 K, const double* __restrict__ U,
                                               double* __restrict__ rho_abs, double* __restrict__ div_cell) {
  const long long item = gtid();
  if (item >= (long long)K.nx * K.ny) return;
  const int i = (int)(item % K.nx) + 1, j = (int)(item / K.nx) + 1;
  const long long c = i + (long long)K.nx2 * j;
  rho_abs[item] = fabs(U[c]);
  double td = 0.0;
#pragma unroll 1
  for (int a = 0; a < NG; ++a)
#pragma unroll 1
    for (int b = 0; b < NG; ++b) {
      double g = 0.0;
#pragma unroll
      for (int d = 0; d < NP3; ++d) {
        const int sx = slot3(5, d), sy = slot3(6, d);
        const double bxv = sx >= 0 ? U[c + K.plane * sx] : 0.0;
        const double byv = sy >= 0 ? U[c + K.plane * sy] : 0.0;
        g = g + bxv * K.B.phixG[a][b][d] + byv * K.B.phiyG[a][b][d];
      }
      td = td + 0.25 * K.B.weight[a] * K.B.weight[b] * fabs(g);
    }
  div_cell[item] = td;
}

}  // namespace gdf3

// =================================================================== host ==
using namespace gdf3;

struct GdfP3Handle {
  GdfP3Config cfg{};
  K3 K{};
  cudaStream_t st = nullptr;
  double *U = nullptr, *T = nullptr, *UII = nullptr;
  double *BX = nullptr, *BXT = nullptr, *BXII = nullptr, *BY = nullptr, *BYT = nullptr, *BYII = nullptr;
  double *Fxh = nullptr, *Fyh = nullptr, *EzV = nullptr, *part = nullptr, *diag = nullptr;
  int32_t* flags = nullptr;
  Scal3* sc = nullptr;
  Scal3* sc_host = nullptr;
  int dt_blocks = 0;
  int uploaded = 0;
  int64_t launches = 0;
  int64_t step_launches = 0;
  cudaGraphExec_t graph = nullptr;
};

namespace {

int fail(int code, const std::string& msg) { return gdf::set_last_error(code, msg.c_str()); }

#define CK3(x)                                                                  \
  do {                                                                          \
    cudaError_t e_ = (x);                                                       \
    if (e_ != cudaSuccess) return fail(GDF_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
  } while (0)

unsigned nblk(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

int check_config(const GdfP3Config* c) {
  if (!c) return fail(GDF_ERR_ARG, "null configuration");
  if (c->nx < 2 || c->ny < 2) return fail(GDF_ERR_ARG, "the grid needs at least 2 x 2 cells");
  if ((long long)(c->nx + 2) * (c->ny + 2) > (1LL << 31) / 84)
    return fail(GDF_ERR_ARG, "grid too large for one device");
  const int32_t bcs[4] = {c->bc_r, c->bc_l, c->bc_u, c->bc_d};
  for (int32_t b : bcs)
    if (b != GDF_BC_PERIODIC && b != GDF_BC_OUTFLOW) return fail(GDF_ERR_ARG, "boundary condition must be 1 or 2");
  if (c->flux_type < 1 || c->flux_type > 4) return fail(GDF_ERR_ARG, "flux_type must be 1..4");
  if (!(c->xb > c->xa) || !(c->yb > c->ya)) return fail(GDF_ERR_ARG, "empty domain");
  if ((c->nx_global != 0 && c->nx_global < c->nx) || (c->ny_global != 0 && c->ny_global < c->ny))
    return fail(GDF_ERR_ARG, "a block cannot be larger than its grid (nx_global, ny_global)");
  if (!(c->gamma > 1.0) || !(c->cfl > 0.0) || !(c->tvb_m >= 0.0) || !(c->tvb_beta > 0.0) ||
      !(c->change_tol >= 0.0) || !(c->hlld_eps >= 0.0))
    return fail(GDF_ERR_ARG, "gamma > 1, cfl > 0, tvb_m >= 0, tvb_beta > 0, change_tol >= 0, hlld_eps >= 0");
  return GDF_OK;
}

void build_k3(const GdfP3Config& c, K3& K) {
  std::memset(&K, 0, sizeof(K));
  K.nx = c.nx;
  K.ny = c.ny;
  K.nx2 = c.nx + 2;
  K.ny2 = c.ny + 2;
  K.plane = (long long)K.nx2 * K.ny2;
  K.fxplane = (long long)(c.nx + 1) * c.ny;
  K.fyplane = (long long)c.nx * (c.ny + 1);
  K.vplane = (long long)(c.nx + 1) * (c.ny + 1);
  K.bxplane = (long long)(c.nx + 1) * K.ny2;
  K.byplane = (long long)K.nx2 * (c.ny + 1);
  // main.f90:565-568
  K.hx = (c.xb - c.xa) / (c.nx_global > 0 ? c.nx_global : c.nx);
  K.hy = (c.yb - c.ya) / (c.ny_global > 0 ? c.ny_global : c.ny);
  const double hx1 = 0.5 * K.hx, hy1 = 0.5 * K.hy;
  K.cxs = 0.5 / K.hx;
  K.cys = 0.5 / K.hy;
  K.rxy = K.hx / K.hy;
  K.ryx = K.hy / K.hx;
  K.Mh2x = c.tvb_m * (K.hx * K.hx);
  K.Mh2y = c.tvb_m * (K.hy * K.hy);
  K.beta = c.tvb_beta;
  K.change_tol = c.change_tol;
  K.cfl = c.cfl;
  K.bc_r = c.bc_r;
  K.bc_l = c.bc_l;
  K.bc_u = c.bc_u;
  K.bc_d = c.bc_d;
  K.P.gamma = c.gamma;
  K.P.gamma1 = c.gamma - 1;
  K.P.gflux = c.gamma;       // MHD_flux (main.f90:2786) and eigenmatrix (:3500) use the module's 5/3
  K.P.hlld_eps = c.hlld_eps;
  K.P.flux = c.flux_type;
  K.P.kml_w = 1;
  K.P.eig_p_typo = 0;
  K.P.eig_identity = 0;      // this eigenmatrix has no identity fallback
  build_basis_p3(hx1, hy1, &K.B);
}

template <class F>
int run(GdfP3Handle* h, F&& launch) {
  launch();
  h->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(GDF_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  return GDF_OK;
}

// set_bc of (S, SX, SY)
int launch_set_bc(GdfP3Handle* h, double* S, double* SX, double* SY, const Scal3* sc) {
  const K3& K = h->K;
  const long long n = (2LL * K.ny2 + 2LL * K.nx) * NS3 + (2LL * (K.nx + 1) + 2LL * (K.ny + 1)) * NB3;
  return run(h, [&] { k3_set_bc<<<nblk(n, 128), 128, 0, h->st>>>(K, S, SX, SY, sc); });
}

// Lh of U (ghosts as they are) into the stage's outputs (kind)
int launch_lh_body(GdfP3Handle* h, int kind, const Scal3* sc) {
  const K3& K = h->K;
  int rc = run(h, [&] { k3_face<0><<<nblk(K.fxplane * NG, 128), 128, 0, h->st>>>(K, h->U, h->Fxh, sc); });
  if (!rc) rc = run(h, [&] { k3_face<1><<<nblk(K.fyplane * NG, 128), 128, 0, h->st>>>(K, h->U, h->Fyh, sc); });
  if (!rc) rc = run(h, [&] { k3_vertex<<<nblk(K.vplane, 128), 128, 0, h->st>>>(K, h->U, h->EzV, sc); });
  if (rc) return rc;
  const unsigned nc = nblk((long long)K.nx * K.ny, 64), nf = nblk(K.fxplane + K.fyplane, 128);
  h->launches++;  // the pair below is two launches
  return run(h, [&] {
    switch (kind) {
      case KIND_LH:
        k3_cell<KIND_LH><<<nc, 64, CELL_SMEM, h->st>>>(K, h->U, h->T, h->UII, h->Fxh, h->Fyh, sc);
        k3_bface<KIND_LH><<<nf, 128, 0, h->st>>>(K, h->Fxh, h->Fyh, h->EzV, h->BX, h->BXT, h->BXII, h->BY, h->BYT,
                                                  h->BYII, sc);
        break;
      case KIND_FIRST:
        k3_cell<KIND_FIRST><<<nc, 64, CELL_SMEM, h->st>>>(K, h->U, h->T, h->UII, h->Fxh, h->Fyh, sc);
        k3_bface<KIND_FIRST><<<nf, 128, 0, h->st>>>(K, h->Fxh, h->Fyh, h->EzV, h->BX, h->BXT, h->BXII, h->BY,
                                                     h->BYT, h->BYII, sc);
        break;
      case KIND_STAGE:
        k3_cell<KIND_STAGE><<<nc, 64, CELL_SMEM, h->st>>>(K, h->U, h->T, h->UII, h->Fxh, h->Fyh, sc);
        k3_bface<KIND_STAGE><<<nf, 128, 0, h->st>>>(K, h->Fxh, h->Fyh, h->EzV, h->BX, h->BXT, h->BXII, h->BY,
                                                     h->BYT, h->BYII, sc);
        break;
      case KIND_FIVE:
        k3_cell<KIND_FIVE><<<nc, 64, CELL_SMEM, h->st>>>(K, h->U, h->T, h->UII, h->Fxh, h->Fyh, sc);
        k3_bface<KIND_FIVE><<<nf, 128, 0, h->st>>>(K, h->Fxh, h->Fyh, h->EzV, h->BX, h->BXT, h->BXII, h->BY,
                                                    h->BYT, h->BYII, sc);
        break;
      default:
        k3_cell<KIND_LAST><<<nc, 64, CELL_SMEM, h->st>>>(K, h->U, h->T, h->UII, h->Fxh, h->Fyh, sc);
        k3_bface<KIND_LAST><<<nf, 128, 0, h->st>>>(K, h->Fxh, h->Fyh, h->EzV, h->BX, h->BXT, h->BXII, h->BY,
                                                    h->BYT, h->BYII, sc);
        break;
    }
  });
}

// set_bc of U, then its Lh
int launch_lh(GdfP3Handle* h, int kind, const Scal3* sc) {
  int rc = launch_set_bc(h, h->U, h->BX, h->BY, sc);
  return rc ? rc : launch_lh_body(h, kind, sc);
}

// TVB_Limiter + div_free_Balsara: (T, BXT, BYT), ghosts as they are -> (U, BX, BY)
int launch_limit_body(GdfP3Handle* h, const Scal3* sc, int32_t* flags) {
  const K3& K = h->K;
  int rc = GDF_OK;
  if (!rc)
    rc = run(h, [&] {
      k3_faceb_limit<<<nblk(K.fxplane + K.fyplane, 128), 128, 0, h->st>>>(K, h->BXT, h->BYT, h->BX, h->BY, sc);
    });
  if (!rc)
    rc = run(h, [&] {
      k3_limit<<<nblk((long long)K.nx * K.ny, 64), 64, 0, h->st>>>(K, h->T, h->U, h->BX, h->BY, flags, sc);
    });
  return rc;
}

// set_bc of T, then the limiter
int launch_limit(GdfP3Handle* h, const Scal3* sc, int32_t* flags) {
  int rc = launch_set_bc(h, h->T, h->BXT, h->BYT, sc);
  return rc ? rc : launch_limit_body(h, sc, flags);
}

int launch_dt(GdfP3Handle* h, int step) {
  const K3& K = h->K;
  int rc = run(h, [&] { k3_dt_partial<<<h->dt_blocks, DT_BS, 0, h->st>>>(K, h->U, h->part, h->sc, step); });
  if (!rc) rc = run(h, [&] { k3_dt_final<<<1, DT_BS, 0, h->st>>>(K, h->part, h->dt_blocks, h->sc, step); });
  return rc;
}

// one RK4 step (main.f90:1335-1423). The limiting after stage 5 is not run:
// its result is overwritten by the combination that follows it (uh = uI).
int enqueue_step(GdfP3Handle* h) {
  const Scal3* sc = h->sc;
  int rc = launch_dt(h, 1);
  for (int s = 1; s <= 10 && !rc; ++s) {
    const int kind = s == 1 ? KIND_FIRST : s == 5 ? KIND_FIVE : s == 10 ? KIND_LAST : KIND_STAGE;
    rc = launch_lh(h, kind, sc);
    if (!rc && s != 5) rc = launch_limit(h, sc, nullptr);
  }
  return rc;
}

int ensure_graph(GdfP3Handle* h) {
  if (h->graph) return GDF_OK;
  cudaGraph_t g = nullptr;
  const int64_t before = h->launches;
  CK3(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
  int rc = enqueue_step(h);
  cudaError_t e = cudaStreamEndCapture(h->st, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return fail(GDF_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&h->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    h->graph = nullptr;
    return fail(GDF_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  }
  h->step_launches = h->launches - before;
  h->launches = before;
  return GDF_OK;
}

int sync_scal(GdfP3Handle* h) {
  CK3(cudaMemcpyAsync(h->sc_host, h->sc, sizeof(Scal3), cudaMemcpyDeviceToHost, h->st));
  CK3(cudaStreamSynchronize(h->st));
  return GDF_OK;
}

int push_scal(GdfP3Handle* h) {
  CK3(cudaMemcpyAsync(h->sc, h->sc_host, sizeof(Scal3), cudaMemcpyHostToDevice, h->st));
  CK3(cudaStreamSynchronize(h->st));
  return GDF_OK;
}

// host uh (full 15-slot layout) -> device live slots; the slots the method
// keeps at zero must be zero
int upload_cells(GdfP3Handle* h, const double* uh, double* D) {
  const size_t pl = (size_t)h->K.plane;
  for (int n = 0; n < NE; ++n)
    for (int d = 0; d < NP3; ++d) {
      const double* src = uh + pl * (d + (size_t)NP3 * n);
      const int s = slot3(n, d);
      if (s < 0) {
        for (size_t q = 0; q < pl; ++q)
          if (src[q] != 0.0)
            return fail(GDF_ERR_ARG, "uh slot (d=" + std::to_string(d + 1) + ", n=" + std::to_string(n + 1) +
                                         ") must be zero: the k = 3 method never fills it");
        continue;
      }
      CK3(cudaMemcpyAsync(D + pl * s, src, pl * sizeof(double), cudaMemcpyHostToDevice, h->st));
    }
  CK3(cudaStreamSynchronize(h->st));
  return GDF_OK;
}

int download_cells(GdfP3Handle* h, const double* D, double* uh) {
  const size_t pl = (size_t)h->K.plane;
  for (int n = 0; n < NE; ++n)
    for (int d = 0; d < NP3; ++d) {
      double* dst = uh + pl * (d + (size_t)NP3 * n);
      const int s = slot3(n, d);
      if (s < 0) {
        std::memset(dst, 0, pl * sizeof(double));
        continue;
      }
      CK3(cudaMemcpyAsync(dst, D + pl * s, pl * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    }
  CK3(cudaStreamSynchronize(h->st));
  return GDF_OK;
}

size_t bx_bytes(const K3& K) { return (size_t)K.bxplane * NB3 * sizeof(double); }
size_t by_bytes(const K3& K) { return (size_t)K.byplane * NB3 * sizeof(double); }

int check_status(GdfP3Handle* h) {
  if (h->sc_host->status & 1)
    return fail(GDF_ERR_NUMERIC, "non-positive density, non-finite energy or non-positive dt at t = " +
                                     std::to_string(h->sc_host->t));
  return GDF_OK;
}

}  // namespace

extern "C" {

int gdf_p3_create(const GdfP3Config* cfg, GdfP3Handle** out) {
  if (!out) return fail(GDF_ERR_ARG, "null handle pointer");
  *out = nullptr;
  int rc = check_config(cfg);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(GDF_ERR_CUDA, "no CUDA device available");
  }
  GdfP3Handle* h = new GdfP3Handle();
  h->cfg = *cfg;
  build_k3(*cfg, h->K);
  const K3& K = h->K;
  const size_t ub = (size_t)K.plane * NS3 * sizeof(double);
  const long long ncell = (long long)cfg->nx * cfg->ny;
  h->dt_blocks = (int)nblk(ncell, DT_BS);
  auto alloc = [&](double** p, size_t bytes) -> bool {
    if (cudaMalloc((void**)p, bytes) != cudaSuccess) return false;
    return cudaMemset(*p, 0, bytes) == cudaSuccess;
  };
  bool ok = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && alloc(&h->U, ub) && alloc(&h->T, ub) && alloc(&h->UII, ub);
  ok = ok && alloc(&h->BX, bx_bytes(K)) && alloc(&h->BXT, bx_bytes(K)) && alloc(&h->BXII, bx_bytes(K));
  ok = ok && alloc(&h->BY, by_bytes(K)) && alloc(&h->BYT, by_bytes(K)) && alloc(&h->BYII, by_bytes(K));
  ok = ok && alloc(&h->Fxh, (size_t)K.fxplane * NG * NE * sizeof(double)) &&
       alloc(&h->Fyh, (size_t)K.fyplane * NG * NE * sizeof(double));
  ok = ok && alloc(&h->EzV, (size_t)K.vplane * sizeof(double));
  ok = ok && alloc(&h->part, (size_t)h->dt_blocks * 2 * sizeof(double));
  ok = ok && alloc(&h->diag, (size_t)ncell * 2 * sizeof(double));
  ok = ok && cudaMalloc((void**)&h->flags, (size_t)ncell * sizeof(int32_t)) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&h->sc, sizeof(Scal3)) == cudaSuccess;
  ok = ok && cudaMallocHost((void**)&h->sc_host, sizeof(Scal3)) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    gdf_p3_destroy(h);
    return fail(GDF_ERR_NOMEM, "device allocation failed for a " + std::to_string(cfg->nx) + "x" +
                                   std::to_string(cfg->ny) + " grid");
  }
  std::memset(h->sc_host, 0, sizeof(Scal3));
  h->sc_host->tend = 1e300;
  h->sc_host->active = 1;
  if (push_scal(h)) {
    gdf_p3_destroy(h);
    return GDF_ERR_CUDA;
  }
  *out = h;
  return GDF_OK;
}

int gdf_p3_destroy(GdfP3Handle* h) {
  if (!h) return GDF_OK;
  if (h->graph) cudaGraphExecDestroy(h->graph);
  for (double* p : {h->U, h->T, h->UII, h->BX, h->BXT, h->BXII, h->BY, h->BYT, h->BYII, h->Fxh, h->Fyh, h->EzV,
                    h->part, h->diag})
    if (p) cudaFree(p);
  if (h->flags) cudaFree(h->flags);
  if (h->sc) cudaFree(h->sc);
  if (h->sc_host) cudaFreeHost(h->sc_host);
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
  return GDF_OK;
}

int gdf_p3_upload(GdfP3Handle* h, const double* uh, const double* bx, const double* by) {
  if (!h || !uh || !bx || !by) return fail(GDF_ERR_ARG, "null argument");
  int rc = upload_cells(h, uh, h->U);
  if (rc) return rc;
  CK3(cudaMemcpyAsync(h->BX, bx, bx_bytes(h->K), cudaMemcpyHostToDevice, h->st));
  CK3(cudaMemcpyAsync(h->BY, by, by_bytes(h->K), cudaMemcpyHostToDevice, h->st));
  h->sc_host->t = 0;
  h->sc_host->dt = 0;
  h->sc_host->active = 1;
  h->sc_host->status = 0;
  h->sc_host->steps = 0;
  rc = push_scal(h);
  if (rc) return rc;
  h->uploaded = 1;
  return GDF_OK;
}

int gdf_p3_download(GdfP3Handle* h, double* uh, double* bx, double* by) {
  if (!h || !uh || !bx || !by) return fail(GDF_ERR_ARG, "null argument");
  if (!h->uploaded) return fail(GDF_ERR_STATE, "no state uploaded");
  int rc = download_cells(h, h->U, uh);
  if (rc) return rc;
  CK3(cudaMemcpyAsync(bx, h->BX, bx_bytes(h->K), cudaMemcpyDeviceToHost, h->st));
  CK3(cudaMemcpyAsync(by, h->BY, by_bytes(h->K), cudaMemcpyDeviceToHost, h->st));
  CK3(cudaStreamSynchronize(h->st));
  return GDF_OK;
}

int gdf_p3_set_time(GdfP3Handle* h, double t) {
  if (!h) return fail(GDF_ERR_ARG, "null handle");
  int rc = sync_scal(h);
  if (rc) return rc;
  h->sc_host->t = t;
  return push_scal(h);
}

int gdf_p3_prepare(GdfP3Handle* h) {
  if (!h) return fail(GDF_ERR_ARG, "null handle");
  if (!h->uploaded) return fail(GDF_ERR_STATE, "no state uploaded");
  const K3& K = h->K;
  CK3(cudaMemcpyAsync(h->T, h->U, (size_t)K.plane * NS3 * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
  CK3(cudaMemcpyAsync(h->BXT, h->BX, bx_bytes(K), cudaMemcpyDeviceToDevice, h->st));
  CK3(cudaMemcpyAsync(h->BYT, h->BY, by_bytes(h->K), cudaMemcpyDeviceToDevice, h->st));
  int rc = launch_limit(h, nullptr, nullptr);
  if (rc) return rc;
  CK3(cudaStreamSynchronize(h->st));
  return GDF_OK;
}

int gdf_p3_step(GdfP3Handle* h, double tend, double* t, double* dt) {
  if (!h) return fail(GDF_ERR_ARG, "null handle");
  if (!h->uploaded) return fail(GDF_ERR_STATE, "no state uploaded");
  int rc = sync_scal(h);
  if (rc) return rc;
  h->sc_host->tend = tend;
  h->sc_host->active = 1;
  if ((rc = push_scal(h))) return rc;
  if ((rc = ensure_graph(h))) return rc;
  CK3(cudaGraphLaunch(h->graph, h->st));
  h->launches += h->step_launches;
  if ((rc = sync_scal(h))) return rc;
  if (t) *t = h->sc_host->t;
  if (dt) *dt = h->sc_host->dt;
  return check_status(h);
}

static int advance_impl(GdfP3Handle* h, double tend, int32_t max_steps, double* t, int32_t* steps, double* ms,
                        bool exact_count) {
  if (!h) return fail(GDF_ERR_ARG, "null handle");
  if (!h->uploaded) return fail(GDF_ERR_STATE, "no state uploaded");
  if (max_steps < 0) return fail(GDF_ERR_ARG, "max_steps < 0");
  int rc = sync_scal(h);
  if (rc) return rc;
  h->sc_host->tend = tend;
  h->sc_host->active = 1;
  const long long s0 = h->sc_host->steps;
  if ((rc = push_scal(h))) return rc;
  if ((rc = ensure_graph(h))) return rc;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (ms) {
    CK3(cudaEventCreate(&e0));
    CK3(cudaEventCreate(&e1));
    CK3(cudaEventRecord(e0, h->st));
  }
  int done = 0;
  const int chunk = exact_count ? max_steps : 16;
  while (done < max_steps) {
    const int n = std::min(chunk, max_steps - done);
    for (int k = 0; k < n; ++k) CK3(cudaGraphLaunch(h->graph, h->st));
    h->launches += (int64_t)n * h->step_launches;
    done += n;
    if (!exact_count) {
      if ((rc = sync_scal(h))) return rc;
      if (!h->sc_host->active || !(h->sc_host->t < tend) || (h->sc_host->status & 1)) break;
    }
  }
  if (ms) {
    CK3(cudaEventRecord(e1, h->st));
    CK3(cudaEventSynchronize(e1));
    float f = 0.f;
    cudaEventElapsedTime(&f, e0, e1);
    *ms = f;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  if ((rc = sync_scal(h))) return rc;
  if (t) *t = h->sc_host->t;
  if (steps) *steps = (int32_t)(h->sc_host->steps - s0);
  return check_status(h);
}

int gdf_p3_advance(GdfP3Handle* h, double tend, int32_t max_steps, double* t, int32_t* steps) {
  return advance_impl(h, tend, max_steps, t, steps, nullptr, false);
}

int gdf_p3_advance_timed(GdfP3Handle* h, double tend, int32_t steps, double* t, int32_t* steps_taken, double* ms) {
  if (!ms) return fail(GDF_ERR_ARG, "null ms");
  return advance_impl(h, tend, steps, t, steps_taken, ms, true);
}

int64_t gdf_p3_kernel_launches(GdfP3Handle* h) { return h ? h->launches : 0; }

// ------------------------------------------------- stage-level control ----
int gdf_p3_block_arrays(GdfP3Handle* h, double** U, double** T, double** BX, double** BY, double** BXT,
                        double** BYT) {
  if (!h) return fail(GDF_ERR_ARG, "null handle");
  if (U) *U = h->U;
  if (T) *T = h->T;
  if (BX) *BX = h->BX;
  if (BY) *BY = h->BY;
  if (BXT) *BXT = h->BXT;
  if (BYT) *BYT = h->BYT;
  return GDF_OK;
}

void* gdf_p3_stream(GdfP3Handle* h) { return h ? (void*)h->st : nullptr; }

int gdf_p3_step_speeds(GdfP3Handle* h, double* ax, double* ay) {
  if (!h || !ax || !ay) return fail(GDF_ERR_ARG, "null argument");
  if (!h->uploaded) return fail(GDF_ERR_STATE, "no state uploaded");
  int rc = launch_dt(h, 2);
  if (rc || (rc = sync_scal(h))) return rc;
  *ax = h->sc_host->ax;
  *ay = h->sc_host->ay;
  return GDF_OK;
}

int gdf_p3_step_begin(GdfP3Handle* h, double ax, double ay, double tend, double* t, double* dt) {
  if (!h) return fail(GDF_ERR_ARG, "null handle");
  if (!h->uploaded) return fail(GDF_ERR_STATE, "no state uploaded");
  int rc = sync_scal(h);
  if (rc) return rc;
  h->sc_host->tend = tend;
  h->sc_host->active = 1;
  if ((rc = push_scal(h))) return rc;
  if ((rc = run(h, [&] { k3_dt_set<<<1, 1, 0, h->st>>>(h->K, ax, ay, h->sc); }))) return rc;
  if ((rc = sync_scal(h))) return rc;
  if (t) *t = h->sc_host->t;
  if (dt) *dt = h->sc_host->dt;
  return check_status(h);
}

int gdf_p3_stage_lh(GdfP3Handle* h, int32_t stage) {
  if (!h) return fail(GDF_ERR_ARG, "null handle");
  if (stage < 1 || stage > 10) return fail(GDF_ERR_ARG, "stage must be 1..10");
  const int kind = stage == 1 ? KIND_FIRST : stage == 5 ? KIND_FIVE : stage == 10 ? KIND_LAST : KIND_STAGE;
  return launch_lh_body(h, kind, h->sc);
}

int gdf_p3_stage_load_t(GdfP3Handle* h) {
  if (!h) return fail(GDF_ERR_ARG, "null handle");
  const K3& K = h->K;
  CK3(cudaMemcpyAsync(h->T, h->U, (size_t)K.plane * NS3 * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
  CK3(cudaMemcpyAsync(h->BXT, h->BX, bx_bytes(K), cudaMemcpyDeviceToDevice, h->st));
  CK3(cudaMemcpyAsync(h->BYT, h->BY, by_bytes(K), cudaMemcpyDeviceToDevice, h->st));
  return GDF_OK;
}

int gdf_p3_stage_limit(GdfP3Handle* h) {
  if (!h) return fail(GDF_ERR_ARG, "null handle");
  return launch_limit_body(h, h->sc, nullptr);
}

int gdf_p3_lh(GdfP3Handle* h, const double* uh, const double* bx, const double* by, double* du, double* dbx,
              double* dby) {
  if (!h || !uh || !bx || !by || !du || !dbx || !dby) return fail(GDF_ERR_ARG, "null argument");
  const K3& K = h->K;
  int rc = upload_cells(h, uh, h->U);
  if (rc) return rc;
  CK3(cudaMemcpyAsync(h->BX, bx, bx_bytes(K), cudaMemcpyHostToDevice, h->st));
  CK3(cudaMemcpyAsync(h->BY, by, by_bytes(K), cudaMemcpyHostToDevice, h->st));
  CK3(cudaMemsetAsync(h->T, 0, (size_t)K.plane * NS3 * sizeof(double), h->st));
  CK3(cudaMemsetAsync(h->BXT, 0, bx_bytes(K), h->st));
  CK3(cudaMemsetAsync(h->BYT, 0, by_bytes(K), h->st));
  if ((rc = launch_lh(h, KIND_LH, nullptr))) return rc;
  if ((rc = download_cells(h, h->T, du))) return rc;
  CK3(cudaMemcpyAsync(dbx, h->BXT, bx_bytes(K), cudaMemcpyDeviceToHost, h->st));
  CK3(cudaMemcpyAsync(dby, h->BYT, by_bytes(K), cudaMemcpyDeviceToHost, h->st));
  CK3(cudaStreamSynchronize(h->st));
  h->uploaded = 1;
  return GDF_OK;
}

int gdf_p3_limit(GdfP3Handle* h, double* uh, double* bx, double* by) {
  if (!h || !uh || !bx || !by) return fail(GDF_ERR_ARG, "null argument");
  const K3& K = h->K;
  int rc = upload_cells(h, uh, h->T);
  if (rc) return rc;
  CK3(cudaMemcpyAsync(h->BXT, bx, bx_bytes(K), cudaMemcpyHostToDevice, h->st));
  CK3(cudaMemcpyAsync(h->BYT, by, by_bytes(K), cudaMemcpyHostToDevice, h->st));
  // the cells' ghosts keep the values set_bc gives them
  if ((rc = launch_set_bc(h, h->T, h->BXT, h->BYT, nullptr))) return rc;
  CK3(cudaMemcpyAsync(h->U, h->T, (size_t)K.plane * NS3 * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
  CK3(cudaMemcpyAsync(h->BX, h->BXT, bx_bytes(K), cudaMemcpyDeviceToDevice, h->st));
  CK3(cudaMemcpyAsync(h->BY, h->BYT, by_bytes(K), cudaMemcpyDeviceToDevice, h->st));
  if ((rc = launch_limit(h, nullptr, nullptr))) return rc;
  if ((rc = download_cells(h, h->U, uh))) return rc;
  CK3(cudaMemcpyAsync(bx, h->BX, bx_bytes(K), cudaMemcpyDeviceToHost, h->st));
  CK3(cudaMemcpyAsync(by, h->BY, by_bytes(K), cudaMemcpyDeviceToHost, h->st));
  CK3(cudaStreamSynchronize(h->st));
  h->uploaded = 1;
  return GDF_OK;
}

int gdf_p3_dt(GdfP3Handle* h, const double* uh, double* dt) {
  if (!h || !uh || !dt) return fail(GDF_ERR_ARG, "null argument");
  int rc = upload_cells(h, uh, h->U);
  if (rc) return rc;
  if ((rc = launch_dt(h, 0))) return rc;
  if ((rc = sync_scal(h))) return rc;
  *dt = h->sc_host->dt;
  return GDF_OK;
}

int gdf_p3_diagnostics(GdfP3Handle* h, double* umax, double* totaldiv) {
  if (!h) return fail(GDF_ERR_ARG, "null handle");
  if (!h->uploaded) return fail(GDF_ERR_STATE, "no state uploaded");
  const K3& K = h->K;
  const long long nc = (long long)K.nx * K.ny;
  int rc = run(h, [&] { k3_diag<<<nblk(nc, 128), 128, 0, h->st>>>(K, h->U, h->diag, h->diag + nc); });
  if (rc) return rc;
  std::vector<double> v((size_t)nc * 2);
  CK3(cudaMemcpyAsync(v.data(), h->diag, v.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK3(cudaStreamSynchronize(h->st));
  // the reference's loop order: i outer, j inner
  double um = 0, td = 0;
  for (int i = 0; i < K.nx; ++i)
    for (int j = 0; j < K.ny; ++j) {
      const size_t q = (size_t)i + (size_t)K.nx * j;
      if (v[q] > um) um = v[q];
      td = td + v[(size_t)nc + q];
    }
  if (umax) *umax = um;
  if (totaldiv) *totaldiv = td / ((double)K.nx * (double)K.ny);
  return GDF_OK;
}

}  // extern "C"
