// gdf_device.cuh -- the per-item device code of the GDF P2 step: one face
// quadrature point, vertex, cell or face per call, in the reference's
// arithmetic order. The single-problem kernels (gdf_kernels.cu) and the
// ensemble's persistent stage kernel (gdf_ensemble.cu) both run these.
#pragma once

#include <cuda_runtime.h>

#include "../../include/gdf.h"
#include "gdf_kernels.cuh"
#include "gdf_mlp.cuh"

#include <mutex>

namespace gdf {

// Grid-independent basis tables (one copy per device and module; each
// translation unit that launches kernels fills its own with
// upload_basis_once before its first launch on a device).
static __constant__ Basis c_basis;

// ------------------------------------------------------------ live slots --
__host__ __device__ constexpr int LI(int n, int d) {
  return n < 5 ? n * 6 + d
               : n == 5 ? 30 + (d <= 6 ? d : 7)
                        : n == 6 ? 38 + (d <= 5 ? d : (d == 7 ? 6 : 7)) : 46 + d;
}
static __constant__ unsigned char c_live_n[NLIVE] = {0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 2, 2, 2, 2, 2, 2,
                                              3, 3, 3, 3, 3, 3, 4, 4, 4, 4, 4, 4, 5, 5, 5, 5, 5, 5,
                                              5, 5, 6, 6, 6, 6, 6, 6, 6, 6, 7, 7, 7, 7, 7, 7};
static __constant__ unsigned char c_live_d[NLIVE] = {0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5,
                                              0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5,
                                              6, 8, 0, 1, 2, 3, 4, 5, 7, 9, 0, 1, 2, 3, 4, 5};

// variable and mode of live slot s (the order of c_live_n / c_live_d)
__host__ __device__ constexpr int slot_n(int s) { return s < 30 ? s / 6 : s < 38 ? 5 : s < 46 ? 6 : 7; }
__host__ __device__ constexpr int slot_d(int s) {
  return s < 30 ? s % 6 : s < 38 ? (s - 30 <= 6 ? s - 30 : 8) : s < 46 ? (s - 38 <= 5 ? s - 38 : (s == 44 ? 7 : 9)) : s - 46;
}
// structural zeros of the volume basis derivatives: phixG vanishes for
// modes 1, 3, 6, 10 and phiyG for modes 1, 2, 4, 7 (get_basis.f90)
__host__ __device__ constexpr bool px_zero(int d) { return d == 0 || d == 2 || d == 5 || d == 9; }
__host__ __device__ constexpr bool py_zero(int d) { return d == 0 || d == 1 || d == 3 || d == 6; }

__device__ __forceinline__ long long gtid() { return (long long)blockIdx.x * blockDim.x + threadIdx.x; }

// ------------------------------------------------------------- set_bc ----
// set_bc.f90:5-27. Ghost (i,j) takes the value of (mapx(i), mapy(j)): the
// x pass first and then the y pass over full rows make every corner ghost
// the image of an interior cell under both maps. zeroB also clears the
// ghost Bx/By modes, as div_free_Balsara.f90:11 leaves them.
__host__ __device__ __forceinline__ long long set_bc_items(const Consts& K) {
  return (2LL * (K.nx + 2) + 2LL * K.ny) * NLIVE;
}
__device__ __forceinline__ void set_bc_item(const Consts& K, double* __restrict__ U, int zeroB, long long t) {
  const long long nper = 2LL * (K.nx + 2) + 2LL * K.ny;
  const int k = (int)(t / nper);
  const long long q = t - (long long)k * nper;
  int i, j;
  if (q < K.nx + 2) { i = (int)q; j = 0; }
  else if (q < 2LL * (K.nx + 2)) { i = (int)(q - (K.nx + 2)); j = K.ny + 1; }
  else if (q < 2LL * (K.nx + 2) + K.ny) { i = 0; j = (int)(q - 2LL * (K.nx + 2)) + 1; }
  else { i = K.nx + 1; j = (int)(q - 2LL * (K.nx + 2) - K.ny) + 1; }
  int si = i, sj = j;
  if (i == 0) si = (K.bc_l == GDF_BC_PERIODIC) ? K.nx : 1;
  else if (i == K.nx + 1) si = (K.bc_r == GDF_BC_PERIODIC) ? 1 : K.nx;
  if (j == 0) sj = (K.bc_d == GDF_BC_PERIODIC) ? K.ny : 1;
  else if (j == K.ny + 1) sj = (K.bc_u == GDF_BC_PERIODIC) ? 1 : K.ny;
  const int n = c_live_n[k], d = c_live_d[k];
  const long long off = K.plane * (d + 10 * n);
  double v = U[off + si + (long long)K.nx2 * sj];
  if (zeroB && (n == 5 || n == 6)) v = 0.0;
  U[off + i + (long long)K.nx2 * j] = v;
}

// k_cell asks for its faces' fluxes in L2 before its volume loop
#ifndef GDF_CELL_PREFETCH
#define GDF_CELL_PREFETCH 1
#endif

// Products with the exact 1 and -1 entries of the basis tables written as
// the value itself (x * 1 == x, x * -1 == -x for every double)
#ifndef GDF_FOLD_UNIT
#define GDF_FOLD_UNIT 1
#endif

// ---------------------------------------------------- face Riemann -------
// Lh.f90:72-265 and LhEz.f90:6-31 for one face quadrature point.
// DIR 0: x face (i = 0..Nx, j = 1..Ny) between cells (i,j) and (i+1,j).
// DIR 1: y face (i = 1..Nx, j = 0..Ny) between cells (i,j) and (i,j+1).
template <int DIR>
__host__ __device__ __forceinline__ long long face_items(const Consts& K) {
  return DIR == 0 ? (long long)(K.nx + 1) * NG * K.ny : (long long)K.nx * NG * (K.ny + 1);
}
// One face quadrature point from the modes of its two cells, read through
// mL(n, d) (the cell on the low side) and mR(n, d) (the high side); o is the
// face's offset in its plane. The arithmetic is that of Lh.f90:72-265 and
// LhEz.f90:6-31 whichever memory the modes come from.
// SMB: the face basis is read from sb, a copy in shared memory of the low
// cell's table (phiGR / phiGU) followed by the high cell's (phiGL / phiGD),
// [2][NG][NP], for lanes whose points g differ (the constant cache would
// serialise their addresses).
template <int DIR, bool SMB = false, class ML, class MR>
__device__ __forceinline__ void face_point(const Consts& K, ML mL, MR mR, int g, double* __restrict__ Fh_out,
                                           double* __restrict__ Ez_out, long long o,
                                           const double* __restrict__ sb = nullptr) {
  double uL[NE], uR[NE];
#pragma unroll
  for (int n = 0; n < NE; ++n) {
    double a = 0.0, b = 0.0;
#pragma unroll
    for (int d = 0; d < NP; ++d) {
      if (!live_mode(n, d)) continue;
      const double pl = SMB ? sb[g * NP + d] : DIR == 0 ? c_basis.phiGR[g][d] : c_basis.phiGU[g][d];
      const double pr = SMB ? sb[(NG + g) * NP + d] : DIR == 0 ? c_basis.phiGL[g][d] : c_basis.phiGD[g][d];
      // the face basis is 1 for mode 1, and for mode 2 (x faces) or 3 (y
      // faces) 1 on the low cell's face and -1 on the high cell's
      // (get_basis.f90): those products are exact and written out
      const int du = DIR == 0 ? 1 : 2;
      if (GDF_FOLD_UNIT && d == 0) {
        a = a + mL(n, d);
        b = b + mR(n, d);
      } else if (GDF_FOLD_UNIT && d == du) {
        a = a + mL(n, d);
        b = b + (-mR(n, d));
      } else {
        a = a + mL(n, d) * pl;
        b = b + mR(n, d) * pr;
      }
    }
    uL[n] = a;
    uR[n] = b;
  }
  Side L, R;
  make_side<true>(K.P, uL, L);
  make_side<true>(K.P, uR, R);
  double Fh[NE], fL[NE], fR[NE];
  face_flux_sides<true>(K.P, L, R, DIR, Fh, fL, fR);
  const long long fp = DIR == 0 ? K.fxplane : K.fyplane;
#pragma unroll
  for (int n = 0; n < NE; ++n) Fh_out[(n * NG + g) * fp + o] = Fh[n];
  double ez;
  if (DIR == 0) {
    if (K.ez_fhat) {
      ez = -Fh[6];
    } else {
      const double S = fmax2(fabs(L.u), fabs(R.u));
      ez = -0.5 * (fL[6] + fR[6] - S * (uR[6] - uL[6]));
    }
  } else {
    if (K.ez_fhat) {
      ez = Fh[5];
    } else {
      const double S = fmax2(fabs(L.v), fabs(R.v));
      ez = 0.5 * (fL[5] + fR[5] - S * (uR[5] - uL[5]));
    }
  }
  Ez_out[g * fp + o] = ez;
}

// GFAST: items run point-fastest (item = g + NG * face), so the five points
// of a face sit on adjacent lanes and their loads of the two cells' modes
// are served by the same cache lines; the face basis then comes from sb
// (see face_point). Otherwise faces run fastest (item = face + nf * (g + NG
// * row)) and every lane of a warp has the same g.
template <int DIR, bool GFAST = false>
__device__ __forceinline__ void face_item(const Consts& K, const double* __restrict__ U, double* __restrict__ Fh_out,
                                          double* __restrict__ Ez_out, long long item,
                                          const double* __restrict__ sb = nullptr) {
  const int nf = DIR == 0 ? K.nx + 1 : K.nx;
  int i0, g, j0;
  if (GFAST) {
    g = (int)(item % NG);
    const long long f = item / NG;
    i0 = (int)(f % nf);
    j0 = (int)(f / nf);
  } else {
    i0 = (int)(item % nf);
    const long long r = item / nf;
    g = (int)(r % NG);
    j0 = (int)(r / NG);
  }
  long long cL, cR;
  if (DIR == 0) {
    cL = i0 + (long long)K.nx2 * (j0 + 1);
    cR = cL + 1;
  } else {
    cL = (i0 + 1) + (long long)K.nx2 * j0;
    cR = cL + K.nx2;
  }
  const long long pl = K.plane;
  face_point<DIR, GFAST>(
      K, [&](int n, int d) { return U[pl * (d + 10 * n) + cL]; }, [&](int n, int d) { return U[pl * (d + 10 * n) + cR]; },
      g, Fh_out, Ez_out, i0 + (long long)nf * j0, sb);
}

// Faces of one block, staged: FACE_TILE faces of one face row at all NG
// points (FACE_TILE * NG threads of a 128-thread block). The modes of the
// cells they touch are copied once into shared memory with coalesced loads
// (x faces: the FACE_TILE + 1 cells of one cell row; y faces: FACE_TILE
// cells of the two cell rows), and every face point reads its two cells
// from there instead of issuing 104 scattered global loads of its own.
constexpr int FACE_TILE = 25;
constexpr int FACE_TILE_W = FACE_TILE + 1;   // cells per staged row
template <int DIR>
__device__ __forceinline__ void face_tile(const Consts& K, const double* __restrict__ U, double* __restrict__ Fh_out,
                                          double* __restrict__ Ez_out, int f0, int j0,
                                          double (*ms)[2 * FACE_TILE_W]) {
  const int nf = DIR == 0 ? K.nx + 1 : K.nx;
  const int rows = DIR == 0 ? 1 : 2;
  const int ncx = DIR == 0 ? min(FACE_TILE_W, nf + 1 - f0) : min(FACE_TILE, nf - f0);
  const long long pl = K.plane;
  const int per_slot = rows * ncx;
  for (int q = threadIdx.x; q < NLIVE * per_slot; q += blockDim.x) {
    const int s = q / per_slot, rk = q - s * per_slot;
    const int r = rk / ncx, k = rk - r * ncx;
    const long long cell = DIR == 0 ? f0 + k + (long long)K.nx2 * (j0 + 1) : (f0 + 1 + k) + (long long)K.nx2 * (j0 + r);
    ms[s][r * FACE_TILE_W + k] = U[cell + pl * (c_live_d[s] + 10 * c_live_n[s])];
  }
  __syncthreads();
  const int t = threadIdx.x;
  if (t >= FACE_TILE * NG) return;
  const int f = t % FACE_TILE, g = t / FACE_TILE;
  const int i0 = f0 + f;
  if (i0 >= nf) return;
  const int kR = DIR == 0 ? f + 1 : FACE_TILE_W + f;
  face_point<DIR>(
      K, [&](int n, int d) { return ms[LI(n, d)][f]; }, [&](int n, int d) { return ms[LI(n, d)][kR]; }, g, Fh_out,
      Ez_out, i0 + (long long)nf * j0);
}

// ------------------------------------------------------- vertex Ez -------
// LhEz.f90:34-69: corner traces of the four cells around vertex (i,j),
// i = 0..Nx, j = 0..Ny, and the 2-D Riemann solver.
__device__ __forceinline__ void vertex_item(const Consts& K, const double* __restrict__ U, double* __restrict__ EzV,
                                            long long item) {
  const int i = (int)(item % (K.nx + 1));
  const int j = (int)(item / (K.nx + 1));
  const long long cLD = i + (long long)K.nx2 * j;  // cell (i,j): its RU corner
  const long long cRD = cLD + 1;                   // (i+1,j): LU corner
  const long long cLU = cLD + K.nx2;               // (i,j+1): RD corner
  const long long cRU = cLU + 1;                   // (i+1,j+1): LD corner
  double URU[NE], ULU[NE], URD[NE], ULD[NE];
#pragma unroll
  for (int n = 0; n < NE; ++n) {
    double a = 0, b = 0, c = 0, e = 0;
#pragma unroll
    for (int d = 0; d < NP; ++d) {
      if (!live_mode(n, d)) continue;
      const long long off = K.plane * (d + 10 * n);
      if (GDF_FOLD_UNIT && (d == 0 || d == 1 || d == 2 || d == 4)) {
        // corner values of modes 1, 2, 3 and 5 are +-1 (get_basis.f90):
        // phiLD = (1,-1,-1,.,1), phiRD = (1,1,-1,.,-1), phiLU = (1,-1,1,.,-1),
        // phiRU = (1,1,1,.,1); the products are exact and written out
        const double xa = U[off + cRU], xb = U[off + cLU], xc = U[off + cRD], xe = U[off + cLD];
        a = a + ((d == 1 || d == 2) ? -xa : xa);
        b = b + ((d == 2 || d == 4) ? -xb : xb);
        c = c + ((d == 1 || d == 4) ? -xc : xc);
        e = e + xe;
      } else {
        a = a + U[off + cRU] * c_basis.phiLD[d];
        b = b + U[off + cLU] * c_basis.phiRD[d];
        c = c + U[off + cRD] * c_basis.phiLU[d];
        e = e + U[off + cLD] * c_basis.phiRU[d];
      }
    }
    URU[n] = a; ULU[n] = b; URD[n] = c; ULD[n] = e;
  }
  EzV[item] = vertex_ez(K.P, URU, ULU, URD, ULD);
}

// ------------------------------------------------ residual + combine -----
// Lh.f90:11-68 (volume), :268-304 (surface, mass) and the RK3.f90 stage
// combine for one cell of the whole (Nx+2)x(Ny+2) array (ghost cells have
// du = 0, as Lh leaves them). stage 0 writes du instead (gdf_lh).
constexpr int CELL_BS = 64;

// The residual kernels read their staged modes in pairs, one 128-bit
// shared-memory load per two modes: blast 2048^2 step 45.6 against 46.5 ms,
// same values (GDF_CELL_PAIRS=0: one 64-bit load per mode).
#ifndef GDF_CELL_PAIRS
#define GDF_CELL_PAIRS 1
#endif

// ms: the block's NLIVE * CELL_BS staging array (blockDim.x == CELL_BS).
// PAIRS: ms holds the live slots in pairs (2L, 2L+1) per thread, 16-byte
// aligned, and the volume loop reads a pair with one 128-bit load (ms must
// then be 16-byte aligned). SHFL: the x-face fluxes are loaded once per face:
// each lane reads its cell's right face and takes its left face, the right
// face of cell i-1, from the lane below by a warp shuffle (lane 0 reads its
// own); every lane of the warp must then call with consecutive items, valid
// or not (valid = false: a lane past the array's end, no work). Both leave
// every value and the order of every sum as they are.
template <bool SHFL = false, bool PAIRS = false>
__device__ __forceinline__ void cell_item(const Consts& K, const double* __restrict__ U, double* __restrict__ U0,
                                          double* __restrict__ UI, const double* __restrict__ Fxh,
                                          const double* __restrict__ Fyh, double* __restrict__ duout,
                                          const Scal* __restrict__ sc, int stage, long long item, double* ms,
                                          bool valid = true) {
  const int tid = threadIdx.x;
  const int i = (int)(item % K.nx2);
  const int j = (int)(item / K.nx2);
  const bool interior = valid && i >= 1 && i <= K.nx && j >= 1 && j <= K.ny;
  auto msi = [&](int L) { return PAIRS ? ((L >> 1) * CELL_BS + tid) * 2 + (L & 1) : L * CELL_BS + tid; };
  double du[NLIVE];
#pragma unroll
  for (int k = 0; k < NLIVE; ++k) du[k] = 0.0;
  // Lh.f90:268-304 for variable n from the fluxes of the cell's four faces
  auto surface = [&](int n, const double* fr, const double* fl, const double* fu, const double* fd) {
#pragma unroll
    for (int d = 0; d < NP; ++d) {
      if (!live_mode(n, d)) continue;
      double acc = du[LI(n, d)];
      // at the middle point (lambda = 0) the face basis of modes 3, 5, 8,
      // 10 (x faces) and 2, 5, 9, 7 (y faces) vanishes on both sides
#pragma unroll
      for (int g = 0; g < NG; ++g) {
        if (g == 2 && (d == 2 || d == 4 || d == 7 || d == 9)) continue;
        // modes 1 and 2 of the x-face basis are 1 on the right face and
        // +-1 on the left (get_basis.f90): x * 1 and x * -1 are exact, so
        // those products are written out
        const double t = (GDF_FOLD_UNIT && d == 0) ? fr[g] - fl[g]
                         : (GDF_FOLD_UNIT && d == 1) ? fr[g] - (-fl[g])
                                                     : fr[g] * c_basis.phiGR[g][d] - fl[g] * c_basis.phiGL[g][d];
        acc = acc - K.cxs * c_basis.w[g] * t;
      }
#pragma unroll
      for (int g = 0; g < NG; ++g) {
        if (g == 2 && (d == 1 || d == 4 || d == 8 || d == 6)) continue;
        // modes 1 and 3 of the y-face basis: 1 on the upper face, +-1 on
        // the lower
        const double t = (GDF_FOLD_UNIT && d == 0) ? fu[g] - fd[g]
                         : (GDF_FOLD_UNIT && d == 2) ? fu[g] - (-fd[g])
                                                     : fu[g] * c_basis.phiGU[g][d] - fd[g] * c_basis.phiGD[g][d];
        acc = acc - K.cys * c_basis.w[g] * t;
      }
      // mm(1) = 1 (get_basis.f90): x / 1 == x
      du[LI(n, d)] = (GDF_FOLD_UNIT && d == 0) ? acc
                     : (n == 3 || n == 7)     ? dv(acc, c_basis.mm[d])
                                              : acc / c_basis.mm[d];
    }
  };
  if (interior) {
#pragma unroll
    for (int n = 0; n < NE; ++n)
#pragma unroll
      for (int d = 0; d < NP; ++d)
        if (live_mode(n, d)) ms[msi(LI(n, d))] = U[item + K.plane * (d + 10 * n)];
    if (GDF_CELL_PREFETCH) {
      // the surface term reads the fluxes of the cell's four faces after the
      // volume loop: ask for them in L2 now, so the loads that follow the
      // volume work do not wait on DRAM
      const long long px = (i - 1) + 1 + (long long)(K.nx + 1) * (j - 1);
      const long long py = (i - 1) + (long long)K.nx * j;
#pragma unroll 1
      for (int q = 0; q < NE * NG; ++q) {
        asm volatile("prefetch.global.L2 [%0];" ::"l"(Fxh + q * K.fxplane + px - 1));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(Fyh + q * K.fyplane + py));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(Fyh + q * K.fyplane + py - K.nx));
      }
    }
    // volume term
#pragma unroll 1
    for (int a = 0; a < NG; ++a) {
#pragma unroll 1
      for (int b = 0; b < NG; ++b) {
        double v[NE];
#pragma unroll
        for (int n = 0; n < NE; ++n) {
          double acc = 0.0;
          double mv[8];
          if (PAIRS) {
            const int nl = (n == 5 || n == 6) ? 8 : 6;
#pragma unroll
            for (int k = 0; k < 8; k += 2)
              if (k < nl) {
                const double2 q = reinterpret_cast<const double2*>(ms)[((LI(n, 0) + k) >> 1) * CELL_BS + tid];
                mv[k] = q.x;
                mv[k + 1] = q.y;
              }
          }
#pragma unroll
          for (int d = 0; d < NP; ++d) {
            if (!live_mode(n, d)) continue;
            const double m = PAIRS ? mv[LI(n, d) - LI(n, 0)] : ms[LI(n, d) * CELL_BS + tid];
            // mode 1 of the volume basis is 1 at every point: m * 1 == m
            if (GDF_FOLD_UNIT && d == 0) acc = acc + m;
            else acc = acc + m * c_basis.phiG[a][b][d];
          }
          v[n] = acc;
        }
        const double rho = v[0];
        const double u = v[1] / rho, vv = v[2] / rho, w = dv(v[3], rho);   // rho w = 0 in 2-D runs
        const double E = v[4], B1 = v[5], B2 = v[6], B3 = v[7];
        const double BB = sq(B1) + sq(B2) + sq(B3);
        const double p = K.P.gamma1 * (E - 0.5 * rho * (sq(u) + sq(vv) + sq(w)) - 0.5 * BB);
        const double S = p + 0.5 * BB;
        const double T = E + S;
        const double Kc = u * B1 + vv * B2 + w * B3;
        double Fx[NE], Fy[NE];
        Fx[0] = v[1];
        Fx[1] = rho * sq(u) + S - sq(B1);
        Fx[2] = rho * u * vv - B1 * B2;
        Fx[3] = rho * u * w - B1 * B3;
        Fx[4] = T * u - Kc * B1;
        Fx[5] = 0.0;
        Fx[6] = u * B2 - vv * B1;
        Fx[7] = u * B3 - w * B1;
        Fy[0] = v[2];
        Fy[1] = rho * u * vv - B1 * B2;
        Fy[2] = rho * sq(vv) + S - sq(B2);
        Fy[3] = rho * vv * w - B2 * B3;
        Fy[4] = T * vv - Kc * B2;
        Fy[5] = vv * B1 - u * B2;
        Fy[6] = 0.0;
        Fy[7] = vv * B3 - w * B2;
        const double coef = 0.25 * c_basis.w[a] * c_basis.w[b];
        // du(d,n) += coef*(Fx*phixG + Fy*phiyG); a product with an exact zero
        // (phixG of modes 1,3,6,10, phiyG of modes 1,2,4,7, Fx(6), Fy(7))
        // contributes +-0 and is left out
#pragma unroll
        for (int d = 1; d < NP; ++d)
#pragma unroll
          for (int n = 0; n < NE; ++n) {
            if (!live_mode(n, d)) continue;
            const bool hx = n != 5 && !px_zero(d);
            const bool hy = n != 6 && !py_zero(d);
            if (hx && hy)
              du[LI(n, d)] = du[LI(n, d)] + coef * (Fx[n] * K.phix[a][b][d] + Fy[n] * K.phiy[a][b][d]);
            else if (hx)
              du[LI(n, d)] = du[LI(n, d)] + coef * (Fx[n] * K.phix[a][b][d]);
            else if (hy)
              du[LI(n, d)] = du[LI(n, d)] + coef * (Fy[n] * K.phiy[a][b][d]);
          }
      }
    }
    if (!SHFL) {
      // surface terms in the reference order (x faces, then y faces), mass
      const long long ox = (i - 1) + 1 + (long long)(K.nx + 1) * (j - 1);  // Fxhat(i,j)
      const long long oy = (i - 1) + (long long)K.nx * j;                  // Fyhat(i,j)
#pragma unroll
      for (int n = 0; n < NE; ++n) {
        double fr[NG], fl[NG], fu[NG], fd[NG];
#pragma unroll
        for (int g = 0; g < NG; ++g) {
          fr[g] = Fxh[(n * NG + g) * K.fxplane + ox];
          fl[g] = Fxh[(n * NG + g) * K.fxplane + ox - 1];
          fu[g] = Fyh[(n * NG + g) * K.fyplane + oy];
          fd[g] = Fyh[(n * NG + g) * K.fyplane + oy - K.nx];
        }
        surface(n, fr, fl, fu, fd);
      }
    }
  }
  if (SHFL) {
    // the right x face of every cell of rows 1..ny with i <= nx (ghost
    // column 0 included: its right face is the left face of cell 1)
    const bool has_r = valid && j >= 1 && j <= K.ny && i <= K.nx;
    const long long ox = i + (long long)(K.nx + 1) * (j - 1);  // Fxhat(i,j)
    const long long oy = (i - 1) + (long long)K.nx * j;        // Fyhat(i,j)
    const bool own_l = (threadIdx.x & 31) == 0;
#pragma unroll
    for (int n = 0; n < NE; ++n) {
      double fr[NG], fl[NG], fu[NG], fd[NG];
#pragma unroll
      for (int g = 0; g < NG; ++g) fr[g] = has_r ? Fxh[(n * NG + g) * K.fxplane + ox] : 0.0;
#pragma unroll
      for (int g = 0; g < NG; ++g) fl[g] = __shfl_up_sync(0xffffffffu, fr[g], 1);
      if (interior) {
#pragma unroll
        for (int g = 0; g < NG; ++g) {
          if (own_l) fl[g] = Fxh[(n * NG + g) * K.fxplane + ox - 1];
          fu[g] = Fyh[(n * NG + g) * K.fyplane + oy];
          fd[g] = Fyh[(n * NG + g) * K.fyplane + oy - K.nx];
        }
        surface(n, fr, fl, fu, fd);
      }
    }
  }
  if (!valid) return;
  if (stage == 0) {
    if (interior) {
#pragma unroll
      for (int n = 0; n < NE; ++n)
#pragma unroll
        for (int d = 0; d < NP; ++d)
          if (live_mode(n, d)) duout[item + K.plane * (d + 10 * n)] = du[LI(n, d)];
    }
    return;
  }
  const double dt = sc->dt;
#pragma unroll
  for (int n = 0; n < NE; ++n)
#pragma unroll
    for (int d = 0; d < NP; ++d) {
      if (!live_mode(n, d)) continue;
      const long long c = item + K.plane * (d + 10 * n);
      const double dd = du[LI(n, d)];
      if (stage == 1) {
        const double u0 = U[c];
        U0[c] = u0;
        UI[c] = u0 + dt * dd;
      } else if (stage == 2) {
        const double v = UI[c] + dt * dd;
        UI[c] = (3.0 / 4.0) * U0[c] + (1.0 / 4.0) * v;
      } else {
        const double v = UI[c] + dt * dd;
        UI[c] = (1.0 / 3.0) * U0[c] + (2.0 / 3.0) * v;
      }
    }
}

// --------------------------------------------------- face-B update -------
// LhEz.f90:71-96 (dEz1 on x faces, dEz2 on y faces) and the face-B stage
// combine of RK3.f90. stage 0 writes dEz only (gdf_lhez).
__device__ __forceinline__ void bface_item(const Consts& K, const double* __restrict__ EzRL,
                                           const double* __restrict__ EzUD, const double* __restrict__ EzV,
                                           double* __restrict__ BX, double* __restrict__ BX0,
                                           double* __restrict__ BXI, double* __restrict__ BY,
                                           double* __restrict__ BY0, double* __restrict__ BYI,
                                           double* __restrict__ dez1, double* __restrict__ dez2,
                                           const Scal* __restrict__ sc, int stage, long long item) {
  const long long nbx = K.fxplane;
  double dez[3];
  long long o, fp;
  double *B, *B0, *BI, *dout;
  if (item < nbx) {
    const int i = (int)(item % (K.nx + 1));
    const int j = (int)(item / (K.nx + 1)) + 1;
    o = item;
    fp = K.fxplane;
    const double v1 = EzV[i + (long long)(K.nx + 1) * j];
    const double v0 = EzV[i + (long long)(K.nx + 1) * (j - 1)];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      double acc = 0.0;
#pragma unroll
      for (int g = 0; g < NG; ++g) acc = acc + 0.5 * c_basis.w[g] * EzRL[g * fp + o] * K.EzyG[g][d];
      dez[d] = (acc - v1 * c_basis.EzU[d] / K.hy + v0 * c_basis.EzD[d] / K.hy) / c_basis.mmE[d];
    }
    B = BX; B0 = BX0; BI = BXI; dout = dez1;
  } else {
    const long long k = item - nbx;
    const int i = (int)(k % K.nx) + 1;
    const int j = (int)(k / K.nx);
    o = k;
    fp = K.fyplane;
    const double v1 = EzV[i + (long long)(K.nx + 1) * j];
    const double v0 = EzV[(i - 1) + (long long)(K.nx + 1) * j];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      double acc = 0.0;
#pragma unroll
      for (int g = 0; g < NG; ++g) acc = acc - 0.5 * c_basis.w[g] * EzUD[g * fp + o] * K.EzxG[g][d];
      dez[d] = (acc + v1 * c_basis.EzR[d] / K.hx - v0 * c_basis.EzL[d] / K.hx) / c_basis.mmE[d];
    }
    B = BY; B0 = BY0; BI = BYI; dout = dez2;
  }
  if (stage == 0) {
#pragma unroll
    for (int d = 0; d < 3; ++d) dout[o + fp * d] = dez[d];
    return;
  }
  const double dt = sc->dt;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const long long c = o + fp * d;
    if (stage == 1) {
      const double b = B[c];
      B0[c] = b;
      const double bi = b + dt * dez[d];
      BI[c] = bi;
      B[c] = bi;
    } else if (stage == 2) {
      const double v = BI[c] + dt * dez[d];
      const double bii = (3.0 / 4.0) * B0[c] + (1.0 / 4.0) * v;
      BI[c] = bii;
      B[c] = bii;
    } else {
      const double v = BI[c] + dt * dez[d];
      B[c] = (1.0 / 3.0) * B0[c] + (2.0 / 3.0) * v;
    }
  }
}

// ------------------------------------------- learned-indicator features ---
// Per cell (ghosts included) the first six P2 modes of rho (copied), of the
// pressure and of |B|^2 (L2 projections with a 3x3 Gauss rule, in FP32):
// 18 floats per cell, QM[(q*6 + d) * plane + cell], q = rho, p, |B|^2.
// These feed the troubled-cell network; the FP64 solver state is untouched.
constexpr int QMODES = 18;

__device__ __forceinline__ float basis10(int d, float x, float y) {
  switch (d) {
    case 0: return 1.f;
    case 1: return x;
    case 2: return y;
    case 3: return x * x - (1.f / 3.f);
    case 4: return x * y;
    case 5: return y * y - (1.f / 3.f);
    case 6: return x * x * x - 0.6f * x;
    case 7: return (x * x - (1.f / 3.f)) * y;
    case 8: return x * (y * y - (1.f / 3.f));
    default: return y * y * y - 0.6f * y;
  }
}

__device__ __forceinline__ void qmodes_item(const Consts& K, const double* __restrict__ S, float* __restrict__ QM,
                                            long long c) {
  const float gx[3] = {-0.7745966692414834f, 0.f, 0.7745966692414834f};
  const float gw[3] = {5.f / 9.f, 8.f / 9.f, 5.f / 9.f};
  const float mmf[6] = {1.f, 1.f / 3.f, 1.f / 3.f, 4.f / 45.f, 1.f / 9.f, 4.f / 45.f};
  float m[NE][NP];
#pragma unroll
  for (int n = 0; n < NE; ++n)
#pragma unroll
    for (int d = 0; d < NP; ++d) m[n][d] = live_mode(n, d) ? (float)S[c + K.plane * (d + 10 * n)] : 0.f;
  float pm[6], bm[6];
#pragma unroll
  for (int d = 0; d < 6; ++d) { pm[d] = 0.f; bm[d] = 0.f; }
  const float g1 = (float)K.P.gamma1;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      float v[NE];
#pragma unroll
      for (int n = 0; n < NE; ++n) {
        float x = 0.f;
#pragma unroll
        for (int d = 0; d < NP; ++d)
          if (live_mode(n, d)) x += m[n][d] * basis10(d, gx[a], gx[b]);
        v[n] = x;
      }
      const float rho = v[0];
      const float b2 = v[5] * v[5] + v[6] * v[6] + v[7] * v[7];
      const float kin = (v[1] * v[1] + v[2] * v[2] + v[3] * v[3]) / rho;
      const float pr = g1 * (v[4] - 0.5f * kin - 0.5f * b2);
      const float wq = gw[a] * gw[b] * 0.25f;
#pragma unroll
      for (int d = 0; d < 6; ++d) {
        const float ph = basis10(d, gx[a], gx[b]);
        pm[d] += wq * ph * pr;
        bm[d] += wq * ph * b2;
      }
    }
#pragma unroll
  for (int d = 0; d < 6; ++d) {
    QM[(long long)d * K.plane + c] = m[0][d];
    QM[(long long)(6 + d) * K.plane + c] = pm[d] / mmf[d];
    QM[(long long)(12 + d) * K.plane + c] = bm[d] / mmf[d];
  }
}

// The 90 inputs of interior cell (i, j): for the cell and its neighbours
// (i+1,j), (i-1,j), (i,j+1), (i,j-1), the 6 modes of rho, p, |B|^2, each
// quantity scaled by the largest |mean| over the five cells, with the
// cell's own mean subtracted from the means; clamped to [-8, 8].
constexpr int NFEAT = 90;
__device__ __forceinline__ void gather_features(const Consts& K, const float* __restrict__ QM, long long c,
                                                float* out /* 90 */) {
  const long long nb[5] = {c, c + 1, c - 1, c + K.nx2, c - K.nx2};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    float sc = 0.f;
#pragma unroll
    for (int k = 0; k < 5; ++k) sc = fmaxf(sc, fabsf(QM[(long long)(q * 6) * K.plane + nb[k]]));
    sc = sc + 1e-30f;
    const float inv = 1.f / sc;
    const float mean_c = QM[(long long)(q * 6) * K.plane + c];
#pragma unroll
    for (int k = 0; k < 5; ++k)
#pragma unroll
      for (int d = 0; d < 6; ++d) {
        float v = QM[(long long)(q * 6 + d) * K.plane + nb[k]];
        if (d == 0) v -= mean_c;
        out[(k * 3 + q) * 6 + d] = fminf(8.f, fmaxf(-8.f, v * inv));
      }
  }
}


// ------------------------------------------------------------ limiter ----
// TVB_Limiter_P2.f90:16-121 (characteristic TVB, Jacobi over cells), with
// KXRCF_Detector.f90 as gate, pp_Limiter.f90, and div_free_Balsara.f90:13-79
// fused, for one interior cell. S is the pre-limit state (ghosts as the
// reference leaves them), D receives the limited state.
constexpr int LIM_BS = 64;
// the second limiter pass (gated cells only) with rolled 8x8 products and
// one out-of-line eigenmatrix (same arithmetic, smaller instruction
// stream); off by default: measured the same as the unrolled form (rotor
// 512^2 steps 104-203, k_limit_tvb 0.606 against 0.612 ms per launch)
#ifndef GDF_TVB_ROLLED
#define GDF_TVB_ROLLED false
#endif
// dynamic shared memory of a learned-mode limiter block: X, W1t, W2t, H1
// tiles (BF16) and the LIM_BS logits
constexpr size_t LIMIT_SMEM_LEARNED = (size_t)(LIM_BS + MLP_H) * MLP_LDX * 2 + (size_t)(MLP_H + LIM_BS) * MLP_LDH * 2 +
                                      LIM_BS * sizeof(float);

template <bool ROLLED = false>
__device__ __forceinline__ void matvec8(const double* A, const double* x, double* y) {
  if (ROLLED) {
    // the same sums with the row loop kept as a loop: the second limiter
    // pass (k_limit_tvb) waits on instruction fetch when its twelve 8x8
    // products are unrolled
#pragma unroll 1
    for (int r = 0; r < 8; ++r) {
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < 8; ++k) acc = acc + A[r + 8 * k] * x[k];
      y[r] = acc;
    }
    return;
  }
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) acc = acc + A[r + 8 * k] * x[k];
    y[r] = acc;
  }
}

// eigenmatrix as one out-of-line copy, for the rolled limiter
static __device__ __noinline__ void eigenmatrix_call(const Phys& P, int dir, double rho, double u1, double u2,
                                                     double u3, double E, double B1, double B2, double B3,
                                                     double* R, double* L) {
  eigenmatrix(P, dir, rho, u1, u2, u3, E, B1, B2, B3, R, L);
}

__device__ __forceinline__ void trace8(const Consts& K, const double* __restrict__ S, long long c,
                                       const double* phi, double* out) {
#pragma unroll
  for (int n = 0; n < NE; ++n) {
    double a = 0.0;
#pragma unroll
    for (int d = 0; d < NP; ++d)
      if (live_mode(n, d)) a = a + S[c + K.plane * (d + 10 * n)] * phi[d];
    out[n] = a;
  }
}

// KXRCF_Detector.f90:187-236 for cell c (interior), given its modes m.
static __device__ bool kxrcf_flag(const Consts& K, const double* __restrict__ S, long long c, const double (*m)[NP],
                           bool prev) {
  double I[NE];
#pragma unroll
  for (int n = 0; n < NE; ++n) I[n] = 0.0;
  double Lij = 1e-12;
  double A[NE], B[NE];
  const long long pl = K.plane;
  if (S[c + 1 + pl * 10] < 0) {  // uh(i+1,j,1,2) < 0: right side inflow
#pragma unroll 1
    for (int g = 0; g < NG; ++g) {
      trace8(K, S, c, c_basis.phiGR[g], A);
      trace8(K, S, c + 1, c_basis.phiGL[g], B);
#pragma unroll
      for (int n = 0; n < NE; ++n) I[n] = I[n] + K.hy1 * c_basis.w[g] * (A[n] - B[n]);
      Lij = Lij + K.hy;
    }
  }
  if (S[c - 1 + pl * 10] > 0) {
#pragma unroll 1
    for (int g = 0; g < NG; ++g) {
      trace8(K, S, c, c_basis.phiGL[g], A);
      trace8(K, S, c - 1, c_basis.phiGR[g], B);
#pragma unroll
      for (int n = 0; n < NE; ++n) I[n] = I[n] + K.hy1 * c_basis.w[g] * (A[n] - B[n]);
      Lij = Lij + K.hy;
    }
  }
  if (S[c + K.nx2 + pl * 20] < 0) {
#pragma unroll 1
    for (int g = 0; g < NG; ++g) {
      trace8(K, S, c, c_basis.phiGU[g], A);
      trace8(K, S, c + K.nx2, c_basis.phiGD[g], B);
#pragma unroll
      for (int n = 0; n < NE; ++n) I[n] = I[n] + K.hx1 * c_basis.w[g] * (A[n] - B[n]);
      Lij = Lij + K.hx;
    }
  }
  if (S[c - K.nx2 + pl * 20] > 0) {
#pragma unroll 1
    for (int g = 0; g < NG; ++g) {
      trace8(K, S, c, c_basis.phiGD[g], A);
      trace8(K, S, c - K.nx2, c_basis.phiGU[g], B);
#pragma unroll
      for (int n = 0; n < NE; ++n) I[n] = I[n] + K.hx1 * c_basis.w[g] * (A[n] - B[n]);
      Lij = Lij + K.hx;
    }
  }
  // with every integral zero each ratio is exactly 0 (the denominator is
  // positive), so the flag is decided without the point maxima
  bool all_zero = true;
#pragma unroll
  for (int n = 0; n < NE; ++n) all_zero = all_zero && (I[n] == 0.0);
  if (all_zero) return prev || (0.0 >= K.ck);
  double uinf[NE];
#pragma unroll
  for (int n = 0; n < NE; ++n) uinf[n] = 0.0;
#pragma unroll 1
  for (int a = 0; a < NG; ++a)
#pragma unroll 1
    for (int b = 0; b < NG; ++b)
#pragma unroll
      for (int n = 0; n < NE; ++n) {
        double v = 0.0;
#pragma unroll
        for (int d = 0; d < NP; ++d)
          if (live_mode(n, d)) v = v + m[n][d] * c_basis.phiG[a][b][d];
        if (fabs(v) + 1e-12 > uinf[n]) uinf[n] = fabs(v) + 1e-12;
      }
  bool flag = prev;
#pragma unroll
  for (int n = 0; n < NE; ++n) {
    const double r = dv(fabs(I[n]), K.pow_hxhy * Lij * uinf[n]);
    if (r >= K.ck) flag = true;
  }
  return flag;
}

// calculate_tq of pp_Limiter.f90:101-126
static __device__ double pp_tq(const Consts& K, const double* ubar, const double* uq) {
  double ta = 0.0, tb = 1.0;
  double ut[NE];
  // bisection on [0,1] to width 1e-14 ends after at most 47 halvings
#pragma unroll 1
  for (int it = 0; it < 64 && tb - ta > 1e-14; ++it) {
    const double tq = 0.5 * (ta + tb);
#pragma unroll
    for (int n = 0; n < NE; ++n) ut[n] = tq * uq[n] + (1 - tq) * ubar[n];
    if (pressure(K.P.gamma, ut) < 1e-12) tb = tq; else ta = tq;
  }
  return ta;
}

// pp_Limiter.f90:10-81 for one cell's modes (in place)
// Bound on |u_q - u_bar| over the 50 GLL-mixed points for variable n:
// sum_d |m_d| max_q |phi_d(q)|, inflated to cover the rounding of the point
// sums (relative error < 2.3e-15 of |u_bar| + the bound).
__device__ __forceinline__ double pp_spread(const Consts& K, const double (*m)[NP], int n) {
  double b = 0.0;
#pragma unroll
  for (int d = 1; d < NP; ++d)
    if (live_mode(n, d)) b = b + fabs(m[n][d]) * c_basis.ppM[d];
  return b * (1.0 + 1e-12) + 1e-12 * fabs(m[n][0]);
}

// pp_Limiter.f90:10-81 for one cell's modes (in place). The density part
// acts only if some point has |rho_bar - rho_q| > rho_bar - 1e-13, and the
// pressure part only if some point has a negative pressure; when the
// bounds of pp_spread rule that out (with margins far above rounding) the
// point evaluations are skipped and the cell is left exactly as the full
// evaluation would leave it.
static __device__ void pp_cell(const Consts& K, double (*m)[NP]) {
  const double epsilon = 1e-13;
  double eta = 1.0;
  const double rb = m[0][0];
  const bool rho_safe = pp_spread(K, m, 0) < (rb - epsilon) * (1.0 - 1e-12);
  if (!rho_safe) {
#pragma unroll 1
  for (int a = 0; a < NG; ++a)
#pragma unroll 1
    for (int b = 0; b < NG; ++b)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        double rq = 0.0;
#pragma unroll
        for (int d = 0; d < NP; ++d)
          if (live_mode(0, d)) rq = rq + m[0][d] * c_basis.phiGLL[s][a][b][d];
        const double eta1 = fabs((rb - epsilon) / (rb - rq));
        if (eta1 < 1) eta = eta1;
      }
  if (eta < 1) {
    const double f = 0.5 * eta;
#pragma unroll
    for (int d = 1; d < NP; ++d) m[0][d] = f * m[0][d];
  }
  }
  {
    // lower bound of the pressure at every point from bounds on the point
    // values; a positive bound (beyond rounding) means no point has pq < 0
    double dv[NE];
#pragma unroll
    for (int n = 0; n < NE; ++n) dv[n] = pp_spread(K, m, n);
    const double rho_lo = m[0][0] - dv[0];
    if (rho_lo > 0.0) {
      const double e_lo = m[4][0] - dv[4];
      const double k_hi = 0.5 * (sq(fabs(m[1][0]) + dv[1]) + sq(fabs(m[2][0]) + dv[2]) + sq(fabs(m[3][0]) + dv[3])) /
                          rho_lo * (1.0 + 1e-12);
      const double b_hi = 0.5 * (sq(fabs(m[5][0]) + dv[5]) + sq(fabs(m[6][0]) + dv[6]) + sq(fabs(m[7][0]) + dv[7])) *
                          (1.0 + 1e-12);
      const double p_lo = e_lo - k_hi - b_hi;
      if (p_lo > 1e-10 * (fabs(e_lo) + k_hi + b_hi)) return;   // eta stays 1: nothing changes
    }
  }
  double ubar[NE];
#pragma unroll
  for (int n = 0; n < NE; ++n) ubar[n] = m[n][0];
  eta = 1.0;
  double eta1 = 1.0;
#pragma unroll 1
  for (int a = 0; a < NG; ++a)
#pragma unroll 1
    for (int b = 0; b < NG; ++b)
#pragma unroll 1
      for (int s = 0; s < 2; ++s) {
        double uq[NE];
#pragma unroll
        for (int n = 0; n < NE; ++n) {
          double acc = 0.0;
#pragma unroll
          for (int d = 0; d < NP; ++d)
            if (live_mode(n, d)) acc = acc + m[n][d] * c_basis.phiGLL[s][a][b][d];
          uq[n] = acc;
        }
        const double pq = pressure(K.P.gamma, uq);
        if (pq < 0) {
          const double tq = pp_tq(K, ubar, uq);
          double n1 = 0.0, n2 = 0.0;
#pragma unroll
          for (int n = 0; n < NE; ++n) {
            const double sqv = tq * uq[n] + (1 - tq) * ubar[n];
            n1 = n1 + sq(sqv - ubar[n]);
            n2 = n2 + sq(uq[n] - ubar[n]);
          }
          eta1 = sqrt(n1) / sqrt(n2);
        }
        if (eta1 < eta) eta = eta1;
      }
  if (eta < 1) eta = 0.5 * eta;
#pragma unroll
  for (int n = 0; n < NE; ++n)
#pragma unroll
    for (int d = 1; d < NP; ++d) m[n][d] = eta * m[n][d];
}

// One interior cell (item < nx*ny). LIM_INFER: called by every thread of a
// LIM_BS-thread block on LIM_BS consecutive items (those past nx*ny idle),
// with lsm the block's LIMIT_SMEM_LEARNED bytes of dynamic shared memory.
// LM (the detector mode): LIM_PLAIN, the reference's detectors; LIM_INFER,
// the learned gate with inference (the first stage of a step: the block runs
// the network on its cells and stores each probability in pnet);
// LIM_PNET, the learned gate on the step's stored probabilities (stages 2
// and 3: the network sees the step's stage-1 pre-limit state).
constexpr int LIM_PLAIN = 0, LIM_INFER = 1, LIM_PNET = 2;
// Limiter of one interior cell in three pieces, composed by limit_item:
//   lim_gate    loads the pre-limit modes and decides the gate (detector,
//               sticky KXRCF flag, learned probability); LIM_INFER runs the
//               network for the block first (block-cooperative)
//   lim_tvb     characteristic TVB limiting of a gated cell
//   lim_finish  positivity limiter, div-free reconstruction, store, flags
template <int LM>
__device__ __forceinline__ bool lim_gate(const Consts& K, const double* __restrict__ S, int32_t* __restrict__ trouble,
                                         const MlpDev* __restrict__ net, const float* __restrict__ QM,
                                         float* __restrict__ pnet, float t_lo, float t_hi, long long item,
                                         unsigned char* lsm, bool valid, long long c, double (*m)[NP],
                                         int32_t& word) {
  const long long pl = K.plane;
  float p_net = 0.f;
  if (LM == LIM_INFER) {
    // the learned indicator for the block's 64 cells on the tensor cores
    __nv_bfloat16* Xs = reinterpret_cast<__nv_bfloat16*>(lsm);
    __nv_bfloat16* W1t = Xs + LIM_BS * MLP_LDX;
    __nv_bfloat16* W2t = W1t + MLP_H * MLP_LDX;
    __nv_bfloat16* H1 = W2t + MLP_H * MLP_LDH;
    float* zz = reinterpret_cast<float*>(H1 + LIM_BS * MLP_LDH);
    const int tid = threadIdx.x;
    // weights: 16-byte rows pieces (W1t rows 12 x 16 B, W2t rows 8 x 16 B)
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
    float f[MLP_INP];
    if (valid) {
      gather_features(K, QM, c, f);
    } else {
#pragma unroll
      for (int k = 0; k < NFEAT; ++k) f[k] = 0.f;
    }
#pragma unroll
    for (int k = NFEAT; k < MLP_INP; ++k) f[k] = 0.f;
#pragma unroll
    for (int q = 0; q < MLP_INP / 8; ++q) {
      uint4 v;
      __nv_bfloat162 a = __floats2bfloat162_rn(f[8 * q], f[8 * q + 1]);
      __nv_bfloat162 b = __floats2bfloat162_rn(f[8 * q + 2], f[8 * q + 3]);
      __nv_bfloat162 cc = __floats2bfloat162_rn(f[8 * q + 4], f[8 * q + 5]);
      __nv_bfloat162 d = __floats2bfloat162_rn(f[8 * q + 6], f[8 * q + 7]);
      v.x = *reinterpret_cast<uint32_t*>(&a);
      v.y = *reinterpret_cast<uint32_t*>(&b);
      v.z = *reinterpret_cast<uint32_t*>(&cc);
      v.w = *reinterpret_cast<uint32_t*>(&d);
      *reinterpret_cast<uint4*>(Xs + tid * MLP_LDX + 8 * q) = v;
    }
    __syncthreads();
    mlp_infer_tiles(Xs, W1t, W2t, net->b1, net->b2, net->w3, net->b3, H1, zz, LIM_BS);
    p_net = 1.f / (1.f + expf(-zz[tid]));
    if (valid) pnet[item] = p_net;
  } else if (LM == LIM_PNET) {
    if (valid) p_net = pnet[item];
  }
  if (!valid) return false;
#pragma unroll
  for (int n = 0; n < NE; ++n)
#pragma unroll
    for (int d = 0; d < NP; ++d) m[n][d] = live_mode(n, d) ? S[c + pl * (d + 10 * n)] : 0.0;
  word = 0;
  bool gate = true;
  if (K.detector == GDF_DETECT_KXRCF) {
    const bool prev = K.sticky ? (trouble[item] != 0) : false;
    // a set sticky flag stays set whatever the detector finds
    gate = prev ? true : kxrcf_flag(K, S, c, m, prev);
    trouble[item] = gate ? 1 : 0;
    if (gate) word |= (1 << 24);
  } else if (LM != LIM_PLAIN) {
    // confident network answers decide; KXRCF decides in the uncertain band
    if (p_net >= t_hi) gate = true;
    else if (p_net >= t_lo) gate = kxrcf_flag(K, S, c, m, false);
    else gate = false;
    if (gate) word |= (1 << 24);
  }
  return gate;
}

// TVB_Limiter_P1.f90:19-90: characteristic minmod of the two slopes only;
// a changed variable keeps its limited slopes and loses every higher mode
__device__ __forceinline__ void lim_tvb_p1(const Consts& K, const double* __restrict__ S, long long c,
                                           double (*m)[NP], int32_t& word) {
  const long long pl = K.plane;
  const double rhoij = m[0][0];
  const double u1 = m[1][0] / rhoij, u2 = m[2][0] / rhoij, u3 = dv(m[3][0], rhoij);
  const double Eij = m[4][0], B1 = m[5][0], B2 = m[6][0], B3 = m[7][0];
  double R[64], L[64];
  double DR[NE], DL[NE], D1[NE], t1[NE], t2[NE], tu[NE], mod[NE], Xm[NE], Ym[NE];
  unsigned change = 0;
  eigenmatrix(K.P, 0, rhoij, u1, u2, u3, Eij, B1, B2, B3, R, L);
#pragma unroll
  for (int n = 0; n < NE; ++n) {
    DR[n] = S[c + 1 + pl * (10 * n)] - m[n][0];
    DL[n] = m[n][0] - S[c - 1 + pl * (10 * n)];
    D1[n] = m[n][1];
  }
  matvec8(L, DR, t1);
  matvec8(L, DL, t2);
  matvec8(L, D1, tu);
#pragma unroll
  for (int k = 0; k < NE; ++k) mod[k] = minmod1(tu[k], t1[k], t2[k], K.Mh2x);
  matvec8(R, mod, Xm);
#pragma unroll
  for (int d = 0; d < NE; ++d)
    if (fabs(Xm[d] - D1[d]) > 1e-6) change |= 1u << d;
  eigenmatrix(K.P, 1, rhoij, u1, u2, u3, Eij, B1, B2, B3, R, L);
#pragma unroll
  for (int n = 0; n < NE; ++n) {
    DR[n] = S[c + K.nx2 + pl * (10 * n)] - m[n][0];
    DL[n] = m[n][0] - S[c - K.nx2 + pl * (10 * n)];
    D1[n] = m[n][2];
  }
  matvec8(L, DR, t1);
  matvec8(L, DL, t2);
  matvec8(L, D1, tu);
#pragma unroll
  for (int k = 0; k < NE; ++k) mod[k] = minmod1(tu[k], t1[k], t2[k], K.Mh2y);
  matvec8(R, mod, Ym);
#pragma unroll
  for (int d = 0; d < NE; ++d)
    if (fabs(Ym[d] - D1[d]) > 1e-6) change |= 1u << d;
#pragma unroll
  for (int n = 0; n < NE; ++n) {
    if (change & (1u << n)) {
#pragma unroll
      for (int d = 3; d < NP; ++d) m[n][d] = 0.0;
      m[n][1] = Xm[n];
      m[n][2] = Ym[n];
    }
  }
  word |= (int32_t)change;
}

// One direction of TVB_Limiter_P2.f90's characteristic part
// (:24-55 x, :57-90 y): the face slopes Dp (mean to + face) and Dm (- face
// to mean) limited against the mean differences DR, DL in the
// characteristic variables of the cell mean (minmod with the bound Mh2),
// back in conserved variables as Yp, Ym. The left eigenvectors are built
// and used in the four products with L before the right ones are built, so
// one 8x8 matrix is live at a time; the products and sums are those of
// eigenmatrix's R and L. With the identity fallback of eigenmatrix.f90:
// 397-404 (either matrix summing above 1e4 in absolute value) both
// matrices are the identity, and the products are taken with it.
__device__ __forceinline__ void char_limit_dir(const Consts& K, int dir, double rho, double u1, double u2,
                                               double u3, double E, double B1, double B2, double B3,
                                               const double* DR, const double* DL, const double* Dp,
                                               const double* Dm, double Mh2, double* Yp, double* Ym) {
  EigFrame f;
  eigen_frame(K.P, dir, rho, u1, u2, u3, E, B1, B2, B3, f);
  double t1[NE], t2[NE], tp[NE], tm[NE];
  double sl = 0.0;
  {
    double L[64];
    eigen_left(dir, f, rho, u1, u2, u3, B1, B2, B3, L);
    if (K.P.eig_identity) {
#pragma unroll
      for (int q = 0; q < 64; ++q) sl = sl + fabs(L[q]);
    }
    matvec8(L, DR, t1);
    matvec8(L, DL, t2);
    matvec8(L, Dp, tp);
    matvec8(L, Dm, tm);
  }
  double R[64];
  eigen_right(dir, f, rho, u1, u2, u3, B1, B2, B3, R);
  if (K.P.eig_identity) {
    double sr = 0.0;
#pragma unroll
    for (int q = 0; q < 64; ++q) sr = sr + fabs(R[q]);
    if (sr > 1e4 || sl > 1e4) {
#pragma unroll
      for (int q = 0; q < 64; ++q) R[q] = (q % 9 == 0) ? 1.0 : 0.0;
      matvec8(R, DR, t1);
      matvec8(R, DL, t2);
      matvec8(R, Dp, tp);
      matvec8(R, Dm, tm);
    }
  }
  double mod[NE];
#pragma unroll
  for (int k = 0; k < NE; ++k) mod[k] = minmod1(tp[k], t1[k], t2[k], Mh2);
  matvec8(R, mod, Yp);
#pragma unroll
  for (int k = 0; k < NE; ++k) mod[k] = minmod1(tm[k], t1[k], t2[k], Mh2);
  matvec8(R, mod, Ym);
}

// STREAM: lim_tvb through char_limit_dir (one eigenvector matrix live at a
// time) instead of both matrices at once; same values. GDF_TVB_STREAM=1
// (the default) gives it to the second limiter pass: with the paired
// residual loads, the developed rotor 512^2 (steps 104-303) runs 4.86
// against 4.94 ms per step (k_limit_tvb 0.48 against 0.51 ms per launch)
// and the blast 2048^2 step, which never launches that kernel, is unchanged
// (45.64 against 45.65 ms), two A/B pairs with equal hashes. An earlier
// build without the paired loads had measured that blast step 46.3 against
// 45.5 ms with it.
#ifndef GDF_TVB_STREAM
#define GDF_TVB_STREAM 1
#endif
// the same for the characteristic limiter run inline by the one-pass
// limiter (the learned gate, and the reference's all-cells limiter):
// Orszag-Tang 512^2 (every cell limited) 3.64 against 3.67 ms per step, but
// the learned blast 2048^2 45.9 against 45.6 ms and the learned blast 512^2
// 5.70 against 5.68 (two A/B pairs, equal hashes), so it stays off
#ifndef GDF_TVB_STREAM_INLINE
#define GDF_TVB_STREAM_INLINE 0
#endif

template <bool ROLLED = false, bool STREAM = false>
__device__ __forceinline__ void lim_tvb(const Consts& K, const double* __restrict__ S, long long c,
                                        double (*m)[NP], int32_t& word) {
  if (K.tvb_p1) {
    lim_tvb_p1(K, S, c, m, word);
    return;
  }
  const long long pl = K.plane;
    const double c23 = 2.0 / 3.0;
    const double rhoij = m[0][0];
    const double u1 = m[1][0] / rhoij, u2 = m[2][0] / rhoij, u3 = dv(m[3][0], rhoij);
    const double Eij = m[4][0], B1 = m[5][0], B2 = m[6][0], B3 = m[7][0];
    double R[64], L[64];
    double DR[NE], DL[NE], Dp[NE], Dm[NE], t1[NE], t2[NE], tu[NE], mod[NE];
    double Rp[NE], Rm[NE], Up[NE], Um[NE];
    unsigned change = 0;
    if (!ROLLED && STREAM) {
#pragma unroll
      for (int n = 0; n < NE; ++n) {
        DR[n] = S[c + 1 + pl * (10 * n)] - m[n][0];
        DL[n] = m[n][0] - S[c - 1 + pl * (10 * n)];
        Dp[n] = m[n][1] + c23 * m[n][3];
        Dm[n] = m[n][1] - c23 * m[n][3];
      }
      char_limit_dir(K, 0, rhoij, u1, u2, u3, Eij, B1, B2, B3, DR, DL, Dp, Dm, K.Mh2x, Rp, Rm);
#pragma unroll
      for (int d = 0; d < NE; ++d)
        if (fabs(Rp[d] - Dp[d]) > 1e-6 || fabs(Rm[d] - Dm[d]) > 1e-6) change |= 1u << d;
#pragma unroll
      for (int n = 0; n < NE; ++n) {
        DR[n] = S[c + K.nx2 + pl * (10 * n)] - m[n][0];
        DL[n] = m[n][0] - S[c - K.nx2 + pl * (10 * n)];
        Dp[n] = m[n][2] + c23 * m[n][5];
        Dm[n] = m[n][2] - c23 * m[n][5];
      }
      if (K.eig_y_zero_w)
        char_limit_dir(K, 1, rhoij, u1, u2, 0.0, Eij, B1, B2, 0.0, DR, DL, Dp, Dm, K.Mh2y, Up, Um);
      else
        char_limit_dir(K, 1, rhoij, u1, u2, u3, Eij, B1, B2, B3, DR, DL, Dp, Dm, K.Mh2y, Up, Um);
#pragma unroll
      for (int d = 0; d < NE; ++d)
        if (fabs(Up[d] - Dp[d]) > 1e-6 || fabs(Um[d] - Dm[d]) > 1e-6) change |= 1u << d;
    } else {
    // x direction
    if (ROLLED) eigenmatrix_call(K.P, 0, rhoij, u1, u2, u3, Eij, B1, B2, B3, R, L);
    else eigenmatrix(K.P, 0, rhoij, u1, u2, u3, Eij, B1, B2, B3, R, L);
#pragma unroll
    for (int n = 0; n < NE; ++n) {
      DR[n] = S[c + 1 + pl * (10 * n)] - m[n][0];
      DL[n] = m[n][0] - S[c - 1 + pl * (10 * n)];
      Dp[n] = m[n][1] + c23 * m[n][3];
      Dm[n] = m[n][1] - c23 * m[n][3];
    }
    matvec8<ROLLED>(L, DR, t1);
    matvec8<ROLLED>(L, DL, t2);
    matvec8<ROLLED>(L, Dp, tu);
#pragma unroll
    for (int k = 0; k < NE; ++k) mod[k] = minmod1(tu[k], t1[k], t2[k], K.Mh2x);
    matvec8<ROLLED>(R, mod, Rp);
#pragma unroll
    for (int d = 0; d < NE; ++d)
      if (fabs(Rp[d] - Dp[d]) > 1e-6) change |= 1u << d;
    matvec8<ROLLED>(L, Dm, tu);
#pragma unroll
    for (int k = 0; k < NE; ++k) mod[k] = minmod1(tu[k], t1[k], t2[k], K.Mh2x);
    matvec8<ROLLED>(R, mod, Rm);
#pragma unroll
    for (int d = 0; d < NE; ++d)
      if (fabs(Rm[d] - Dm[d]) > 1e-6) change |= 1u << d;
    // y direction
    if (ROLLED)
      eigenmatrix_call(K.P, 1, rhoij, u1, u2, K.eig_y_zero_w ? 0.0 : u3, Eij, B1, B2, K.eig_y_zero_w ? 0.0 : B3, R, L);
    else if (K.eig_y_zero_w)
      eigenmatrix(K.P, 1, rhoij, u1, u2, 0.0, Eij, B1, B2, 0.0, R, L);
    else
      eigenmatrix(K.P, 1, rhoij, u1, u2, u3, Eij, B1, B2, B3, R, L);
#pragma unroll
    for (int n = 0; n < NE; ++n) {
      DR[n] = S[c + K.nx2 + pl * (10 * n)] - m[n][0];
      DL[n] = m[n][0] - S[c - K.nx2 + pl * (10 * n)];
      Dp[n] = m[n][2] + c23 * m[n][5];
      Dm[n] = m[n][2] - c23 * m[n][5];
    }
    matvec8<ROLLED>(L, DR, t1);
    matvec8<ROLLED>(L, DL, t2);
    matvec8<ROLLED>(L, Dp, tu);
#pragma unroll
    for (int k = 0; k < NE; ++k) mod[k] = minmod1(tu[k], t1[k], t2[k], K.Mh2y);
    matvec8<ROLLED>(R, mod, Up);
#pragma unroll
    for (int d = 0; d < NE; ++d)
      if (fabs(Up[d] - Dp[d]) > 1e-6) change |= 1u << d;
    matvec8<ROLLED>(L, Dm, tu);
#pragma unroll
    for (int k = 0; k < NE; ++k) mod[k] = minmod1(tu[k], t1[k], t2[k], K.Mh2y);
    matvec8<ROLLED>(R, mod, Um);
#pragma unroll
    for (int d = 0; d < NE; ++d)
      if (fabs(Um[d] - Dm[d]) > 1e-6) change |= 1u << d;
    }
#pragma unroll
    for (int n = 0; n < NE; ++n) {
      if (change & (1u << n)) {
#pragma unroll
        for (int d = 6; d < NP; ++d) m[n][d] = 0.0;
        m[n][4] = 0.0;
        m[n][1] = 0.5 * (Rp[n] + Rm[n]);
        m[n][2] = 0.5 * (Up[n] + Um[n]);
        m[n][3] = K.tvb_slope * (Rp[n] - Rm[n]);
        m[n][5] = K.tvb_slope * (Up[n] - Um[n]);
      }
    }
    word |= (int32_t)change;
  }

__device__ __forceinline__ void lim_finish(const Consts& K, double* __restrict__ D, const double* __restrict__ BX,
                                           const double* __restrict__ BY, int32_t* __restrict__ flags, int stage,
                                           int divfree, Scal* __restrict__ sc, long long item, int i, int j,
                                           long long c, double (*m)[NP], int32_t word) {
  const long long pl = K.plane;
  if (K.pp) pp_cell(K, m);
  if (divfree) {
    // div_free_Balsara.f90:30-75 from the four face polynomials
    const long long fxp = K.fxplane, fyp = K.fyplane;
    const long long ox = i + (long long)(K.nx + 1) * (j - 1);
    const long long oy = (i - 1) + (long long)K.nx * j;
    const double a0R = BX[ox], a1R = BX[ox + fxp], a2R = BX[ox + 2 * fxp];
    const double a0L = BX[ox - 1], a1L = BX[ox - 1 + fxp], a2L = BX[ox - 1 + 2 * fxp];
    const double b0U = BY[oy], b1U = BY[oy + fyp], b2U = BY[oy + 2 * fyp];
    const double b0D = BY[oy - K.nx], b1D = BY[oy - K.nx + fyp], b2D = BY[oy - K.nx + 2 * fyp];
    const double rxy = K.rxy, ryx = K.ryx;
    const double c16 = 1.0 / 6.0, c115 = 1.0 / 15.0, c14 = 1.0 / 4.0, c12 = 1.0 / 2.0;
#pragma unroll
    for (int d = 0; d < NP; ++d) { m[5][d] = 0.0; m[6][d] = 0.0; }
    m[5][0] = c12 * (a0R + a0L) + c16 * rxy * (b1U - b1D);
    m[5][1] = c12 * (a0R - a0L) + c115 * rxy * (b2U - b2D);
    m[5][2] = c12 * (a1R + a1L);
    m[5][3] = -c14 * rxy * (b1U - b1D);
    m[5][4] = c12 * (a1R - a1L);
    m[5][5] = c12 * (a2R + a2L);
    m[5][6] = -c16 * rxy * (b2U - b2D);
    m[5][8] = c12 * (a2R - a2L);
    m[6][0] = c12 * (b0U + b0D) + c16 * ryx * (a1R - a1L);
    m[6][2] = c12 * (b0U - b0D) + c115 * ryx * (a2R - a2L);
    m[6][1] = c12 * (b1U + b1D);
    m[6][5] = -c14 * ryx * (a1R - a1L);
    m[6][4] = c12 * (b1U - b1D);
    m[6][3] = c12 * (b2U + b2D);
    m[6][9] = -c16 * ryx * (a2R - a2L);
    m[6][7] = c12 * (b2U - b2D);
  }
#pragma unroll
  for (int n = 0; n < NE; ++n)
#pragma unroll
    for (int d = 0; d < NP; ++d)
      if (live_mode(n, d)) D[c + pl * (d + 10 * n)] = m[n][d];
  if (flags) {
    int32_t w = (word & 0xff) << (8 * (stage - 1));
    if (word & (1 << 24)) w |= (1 << (23 + stage));
    if (stage <= 1) flags[item] = w; else flags[item] |= w;
  }
  if (!(m[0][0] > 0.0) || !isfinite(m[4][0])) atomicOr(&sc->status, 1);
}

// Appends the gated cells among the calling warp's active lanes to list
// (one atomic per warp); true for a gated cell.
__device__ __forceinline__ bool lim_defer(bool gate, long long item, int32_t* __restrict__ list,
                                          int32_t* __restrict__ count) {
  const unsigned act = __activemask();
  const unsigned bal = __ballot_sync(act, gate);
  if (!gate) return false;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(bal) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(count, __popc(bal));
  base = __shfl_sync(bal, base, leader);
  list[base + __popc(bal & ((1u << lane) - 1u))] = (int32_t)item;
  return true;
}

// One interior cell of the limiter. COMPACT: a gated cell is only appended
// to list (limit_tvb_item finishes it in a second pass over full warps, so
// the characteristic limiter never runs beside idle lanes); an ungated one
// is finished here.
template <int LM, bool COMPACT = false>
__device__ __forceinline__ void limit_item(const Consts& K, const double* __restrict__ S, double* __restrict__ D,
                                           const double* __restrict__ BX, const double* __restrict__ BY,
                                           int32_t* __restrict__ flags, int32_t* __restrict__ trouble, int stage,
                                           int divfree, Scal* __restrict__ sc, const MlpDev* __restrict__ net,
                                           const float* __restrict__ QM, float* __restrict__ pnet,
                                           float t_lo, float t_hi, long long item, unsigned char* lsm,
                                           int32_t* __restrict__ list = nullptr,
                                           int32_t* __restrict__ count = nullptr) {
  const bool valid = item < (long long)K.nx * K.ny;
  const int i = valid ? (int)(item % K.nx) + 1 : 1;
  const int j = valid ? (int)(item / K.nx) + 1 : 1;
  const long long c = i + (long long)K.nx2 * j;
  double m[NE][NP];
  int32_t word = 0;
  const bool gate = lim_gate<LM>(K, S, trouble, net, QM, pnet, t_lo, t_hi, item, lsm, valid, c, m, word);
  if (!valid) return;
  if (COMPACT) {
    if (lim_defer(gate, item, list, count)) return;
  } else if (gate) {
    lim_tvb<false, GDF_TVB_STREAM_INLINE != 0>(K, S, c, m, word);
  }
  lim_finish(K, D, BX, BY, flags, stage, divfree, sc, item, i, j, c, m, word);
}

// The second pass for a cell limit_item<LM, true> deferred: its pre-limit
// modes again, the detector bit lim_gate set for it (KXRCF and the learned
// gate set it; GDF_DETECT_ALL does not), the characteristic limiter and the
// finish.
__device__ __forceinline__ void limit_tvb_item(const Consts& K, const double* __restrict__ S, double* __restrict__ D,
                                               const double* __restrict__ BX, const double* __restrict__ BY,
                                               int32_t* __restrict__ flags, int stage, int divfree,
                                               Scal* __restrict__ sc, long long item) {
  const long long pl = K.plane;
  const int i = (int)(item % K.nx) + 1;
  const int j = (int)(item / K.nx) + 1;
  const long long c = i + (long long)K.nx2 * j;
  double m[NE][NP];
#pragma unroll
  for (int n = 0; n < NE; ++n)
#pragma unroll
    for (int d = 0; d < NP; ++d) m[n][d] = live_mode(n, d) ? S[c + pl * (d + 10 * n)] : 0.0;
  int32_t word = K.detector != GDF_DETECT_ALL ? (1 << 24) : 0;
  lim_tvb<GDF_TVB_ROLLED, GDF_TVB_STREAM != 0>(K, S, c, m, word);
  lim_finish(K, D, BX, BY, flags, stage, divfree, sc, item, i, j, c, m, word);
}

// Face-B TVB limiter of TVB_Limiter_P2.f90:128-187 (applied when enabled):
// S holds the limited cell state with ghosts set, pre div-free.
__device__ __forceinline__ double minmodB(double a, double b, double c, double Mh2) {
  if (fabs(a) <= Mh2) return a;
  const double s = (sgn1(a) + sgn1(b) + sgn1(c)) / 3.0;
  if (fabs(s) == 1) return s * fmin2(fmin2(fabs(a), fabs(b)), fabs(c));
  return 0.0;
}

__device__ __forceinline__ void faceb_item(const Consts& K, const double* __restrict__ S, double* __restrict__ BX,
                                           double* __restrict__ BY, long long item) {
  const long long pl = K.plane;
  const double c23 = 2.0 / 3.0, c25 = 2.0 / 5.0;
  (void)c25;
  if (item < K.fxplane) {
    const int i = (int)(item % (K.nx + 1));
    const int j = (int)(item / (K.nx + 1)) + 1;
    const long long cL = i + (long long)K.nx2 * j, cR = cL + 1;
    const long long s6 = pl * 50;  // Bx slots start at d + 10*5
    // aRM(i,j,d) (d = 2,3) of cell i and aLM(i+1,j,d) of cell i+1
    const double aRM2 = S[cL + s6 + pl * 2] + S[cL + s6 + pl * 4];
    const double aRM3 = S[cL + s6 + pl * 5] + S[cL + s6 + pl * 8];
    const double aLM2 = S[cR + s6 + pl * 2] - S[cR + s6 + pl * 4];
    const double aLM3 = S[cR + s6 + pl * 5] - S[cR + s6 + pl * 8];
    BX[item + K.fxplane] = minmodB(BX[item + K.fxplane], aRM2, aLM2, K.Mh2x_b);
    BX[item + 2 * K.fxplane] = minmodB(BX[item + 2 * K.fxplane], aRM3, aLM3, K.Mh2x_b);
    (void)c23;
  } else if (item < K.fxplane + K.fyplane) {
    const long long k = item - K.fxplane;
    const int i = (int)(k % K.nx) + 1;
    const int j = (int)(k / K.nx);
    const long long cD = i + (long long)K.nx2 * j, cU = cD + K.nx2;
    const long long s7 = pl * 60;
    const double bUM2 = S[cD + s7 + pl * 1] + S[cD + s7 + pl * 4];
    const double bUM3 = S[cD + s7 + pl * 3] + S[cD + s7 + pl * 7];
    const double bDM2 = S[cU + s7 + pl * 1] - S[cU + s7 + pl * 4];
    const double bDM3 = S[cU + s7 + pl * 3] - S[cU + s7 + pl * 7];
    BY[k + K.fyplane] = minmodB(BY[k + K.fyplane], bUM2, bDM2, K.Mh2y_b);
    BY[k + 2 * K.fyplane] = minmodB(BY[k + 2 * K.fyplane], bUM3, bDM3, K.Mh2y_b);
  }
}

// div_free_Balsara.f90:13-79 on its own (used after the face-B limiter)
__device__ __forceinline__ void divfree_item(const Consts& K, double* __restrict__ D, const double* __restrict__ BX,
                                             const double* __restrict__ BY, long long item) {
  const int i = (int)(item % K.nx) + 1;
  const int j = (int)(item / K.nx) + 1;
  const long long c = i + (long long)K.nx2 * j;
  const long long pl = K.plane, fxp = K.fxplane, fyp = K.fyplane;
  const long long ox = i + (long long)(K.nx + 1) * (j - 1);
  const long long oy = (i - 1) + (long long)K.nx * j;
  const double a0R = BX[ox], a1R = BX[ox + fxp], a2R = BX[ox + 2 * fxp];
  const double a0L = BX[ox - 1], a1L = BX[ox - 1 + fxp], a2L = BX[ox - 1 + 2 * fxp];
  const double b0U = BY[oy], b1U = BY[oy + fyp], b2U = BY[oy + 2 * fyp];
  const double b0D = BY[oy - K.nx], b1D = BY[oy - K.nx + fyp], b2D = BY[oy - K.nx + 2 * fyp];
  const double rxy = K.rxy, ryx = K.ryx;
  const double c16 = 1.0 / 6.0, c115 = 1.0 / 15.0, c14 = 1.0 / 4.0, c12 = 1.0 / 2.0;
  double* X = D + c + pl * 50;
  double* Y = D + c + pl * 60;
  X[0] = c12 * (a0R + a0L) + c16 * rxy * (b1U - b1D);
  X[pl * 1] = c12 * (a0R - a0L) + c115 * rxy * (b2U - b2D);
  X[pl * 2] = c12 * (a1R + a1L);
  X[pl * 3] = -c14 * rxy * (b1U - b1D);
  X[pl * 4] = c12 * (a1R - a1L);
  X[pl * 5] = c12 * (a2R + a2L);
  X[pl * 6] = -c16 * rxy * (b2U - b2D);
  X[pl * 8] = c12 * (a2R - a2L);
  Y[0] = c12 * (b0U + b0D) + c16 * ryx * (a1R - a1L);
  Y[pl * 2] = c12 * (b0U - b0D) + c115 * ryx * (a2R - a2L);
  Y[pl * 1] = c12 * (b1U + b1D);
  Y[pl * 5] = -c14 * ryx * (a1R - a1L);
  Y[pl * 4] = c12 * (b1U - b1D);
  Y[pl * 3] = c12 * (b2U + b2D);
  Y[pl * 9] = -c16 * ryx * (a2R - a2L);
  Y[pl * 7] = c12 * (b2U - b2D);
}

// --------------------------------------------------------- dt -----------
// calculate_dt.f90:11-25: per-block maxima of |u_n +- c_f| over the cell
// averages, then one block folds them and advances t (RK3.f90:60-71).
constexpr int DT_BS = 256;

__device__ __forceinline__ double max_ign_nan(double a, double b) {
  if (b != b) return a;
  if (a != a) return b;
  return b > a ? b : a;
}

// calculate_dt.f90:15-22 for interior cell `item`: the largest |fast
// speeds| of its average in x (ax) and y (ay); flags a non-positive density
// or non-finite energy in sc->status.
__device__ __forceinline__ void dt_cell_speeds(const Consts& K, const double* __restrict__ U, long long item,
                                               double& ax, double& ay, Scal* __restrict__ sc) {
  const int i = (int)(item % K.nx) + 1;
  const int j = (int)(item / K.nx) + 1;
  const long long c = i + (long long)K.nx2 * j;
  double Uv[NE];
#pragma unroll
  for (int n = 0; n < NE; ++n) Uv[n] = U[c + K.plane * (10 * n)];
  double a1, a2;
  fast_speeds(K.P, Uv, 0, a1, a2);
  if (fabs(a1) > ax || fabs(a2) > ax) ax = fmax2(fabs(a1), fabs(a2));
  fast_speeds(K.P, Uv, 1, a1, a2);
  if (fabs(a1) > ay || fabs(a2) > ay) ay = fmax2(fabs(a1), fabs(a2));
  if (!(Uv[0] > 0.0) || !isfinite(Uv[4])) atomicOr(&sc->status, 1);
}

// calculate_dt.f90:23-25 and RK3.f90:60-71 from the grid maxima: mode 0
// sets dt only (gdf_dt); mode 1 takes a time step (t, dt, active, steps).
__device__ __forceinline__ void dt_advance(const Consts& K, double ax, double ay, Scal* __restrict__ sc, int mode) {
  double dt = K.cfl / (ax / K.hx + ay / K.hy);
  if (mode == 0) {
    sc->dt = dt;
    return;
  }
  double t = sc->t;
  if (!(t < sc->tend)) {
    sc->active = 0;
    return;
  }
  if (t + dt >= sc->tend) {
    dt = sc->tend - t;
    t = sc->tend;
  } else {
    t = t + dt;
  }
  if (K.dt_floor_stop && dt < 1e-7) t = sc->tend;
  if (!(dt > 0.0) || !isfinite(dt)) sc->status |= 1;
  sc->dt = dt;
  sc->t = t;
  sc->active = 1;
  sc->steps += 1;
}

// Fills this module's c_basis on the current device (the tables do not
// depend on the configuration). always: on every call (handle creation:
// survives a reset of the device between handles); otherwise once per
// device and process. Returns a cudaError_t.
static inline cudaError_t upload_basis_once(const Consts& K, bool always = false) {
  static std::mutex mu;
  static bool done[256] = {false};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 256) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(mu);
  if (done[dev] && !always) return cudaSuccess;
  Basis B;
  basis_of(K, B);
  e = cudaMemcpyToSymbol(c_basis, &B, sizeof(Basis));
  if (e == cudaSuccess) done[dev] = true;
  return e;
}

}  // namespace gdf

