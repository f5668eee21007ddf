// gdf_cy.cu -- the cylindrical variant of the GDF MHD method
// (MHD_GDF_cy3D_0421/) on sm_100a, behind the C ABI of include/gdf_cy.h:
// modal P2 in (r, z) with the cubic slots of r*B written by the Balsara
// reconstruction, 2*Lphi planes in phi coupled by Fourier sums, geometric
// and manufactured source terms, SSP-RK3.
//
// One item per thread, in the reference's operation order (the product
// build has no FMA contraction). Items that couple the phi planes (the
// volume term's d(Fz)/dphi, the faces' d(E)/dphi, the reconstruction's
// d(Bphi)/dphi, the divergence diagnostic) put the planes of one cell or
// face point on adjacent lanes and exchange their values with warp
// shuffles, summing over the planes in the reference's order. Per stage:
//   k_cy_set_bc        set_bc.f90 (ghost cells, all live slots)
//   k_cy_face<0>, <1>  traces, cylindrical fluxes, eigenvalueMm, HLL/LF,
//                      the LF edge fields and their d/dphi (Lh.f90:149-368,
//                      LhEz.f90:5-127)
//   k_cy_vertex        corner values and LF_Flux_2D (LhEz.f90:129-161)
//   k_cy_cell<KIND>    volume term with the geometric source and the
//                      Fourier derivative, surface terms, mass matrix
//                      (Lh.f90:14-407, LhEz.f90:36-55), fused with the
//                      stage's RK3 combination (RK3.f90:72-133)
//   k_cy_bface<KIND>   dBr, dBz (LhEz.f90:163-200) with the combination
//   k_cy_bproj         B = rB / r projected on the P2 modes
//                      (TVB_Limiter_P2.f90:14-40)
//   k_cy_tvb           characteristic TVB (TVB_Limiter_P2.f90:42-140)
//   k_cy_faceb         face-B minmod (TVB_Limiter_P2.f90:144-210)
//   k_cy_divfree       div_free_Balsara.f90
// and per step k_cy_dt_partial + k_cy_dt_final (calculate_dt.f90 and the
// clamp of RK3.f90:42-58). A step is captured once as a CUDA graph.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gdf_cy.h"
#include "gdf_physics.cuh"

namespace gdf {
int set_last_error(int code, const char* msg);
}

namespace gdfc {

using gdf::fmax2;
using gdf::fmin2;
using gdf::Phys;
using gdf::sq;

constexpr int NG = 5, NE = 8, NQC = 6, NPC = 10;
constexpr int LMAX = 8, PMAX = 16;   // Lphi <= 8, 2*Lphi planes
constexpr int NFQ = 10;              // per face point: 7 fluxes, E, E', dE/dphi

// ------------------------------------------------------------ live slots ---
// 54 slots per cell plane: modes 1-6 of every variable, and the cubic modes
// 7-9 of r*B_r (a30, a21, a12) and 8-10 of r*B_z (b21, b12, b03) that
// div_free_Balsara writes. Every other slot stays zero and is not stored.
constexpr int NSC = 54;
__host__ __device__ constexpr int slotc(int n, int d) {
  return d < NQC ? NQC * n + d
                 : (n == 5 && d >= 6 && d <= 8) ? 48 + (d - 6) : (n == 6 && d >= 7 && d <= 9) ? 51 + (d - 7) : -1;
}

constexpr int KIND_LH = 0;  // du only (gdf_cy_lh)
constexpr int KIND_S1 = 1;  // uI = uh + dt du; uh0 = uh; uh = uI
constexpr int KIND_S2 = 2;  // uII = 3/4 uh0 + 1/4 (uI + dt du); uh = uII
constexpr int KIND_S3 = 3;  // uh = 1/3 uh0 + 2/3 (uII + dt du)

struct BasisC {
  double lam[NG], w[NG];
  double phiG[NG][NG][NPC], phixG[NG][NG][NPC], phiyG[NG][NG][NPC];
  double phiGLL[2][NG][NG][NPC];
  double phiGR[NG][NQC], phiGL[NG][NQC], phiGU[NG][NQC], phiGD[NG][NQC];
  double phiRU[NPC], phiLU[NPC], phiRD[NPC], phiLD[NPC];
  double mm[NPC];
  double EzG[NG][3], EzxG[NG][3], EzyG[NG][3], mmE[3], EzR[3], EzL[3], EzU[3], EzD[3];
};

struct KC {
  int nx, ny, nx2, ny2, nph, lphi;
  long long ncp, nxf, nyf, nvx;   // cell planes; x faces, y faces, vertices (each x nph)
  double ra, rb, za, hr, hz, hr1, hz1, cxs, czs, Mh2r, Mh2z, change_tol, cfl, jet_r;
  int bc_r, bc_l, bc_u, bc_d, flux, src;
  Phys P;
  double sink[LMAX][PMAX], cosk[LMAX][PMAX], phi[PMAX];
  BasisC B;
};

struct ScalC {
  double t, dt, tend, trk[3];
  int active;   // 0 once t has reached tend: the step's kernels return at once
  int status;   // bit 0: non-positive density, non-finite energy or dt seen
  long long steps;
};

__device__ __forceinline__ long long gtid() { return (long long)blockIdx.x * blockDim.x + threadIdx.x; }

__device__ __forceinline__ double ld(const double* p) { return __ldg(p); }

// Source.f90:1-62 (CUDA's sin and cos: within a few ulp of the host's)
__device__ double S1f(double r, double z, double t) { return (1 + 0.5 * sin((r + z) - 2 * t)) / r; }
__device__ double S2f(double r, double z, double phi, double t) {
  const double cp2 = sq(cos(phi));
  return (0.25 * sin(r - t) * cos(r - t) * cp2 + 0.25 * sin(r - t) * cos(z - t) * cp2) + (1 + 0.5 * sin((r + z) - 2 * t)) / r;
}
__device__ double S3f(double r, double z, double phi, double t) {
  const double cp2 = sq(cos(phi)), sp2 = sq(sin(phi));
  return ((0.25 * cos(r - t) * sin(z - t) * cp2 + 0.25 * sin(z - t) * cos(z - t)) + (1 + 0.5 * sin((r + z) - 2 * t)) / r) +
         0.25 * sin(r - t) * sin(z - t) * sp2 / r;
}
__device__ double S4f(double r, double z, double phi, double t) {
  return -(0.25 * sin(r - t) * cos(z - t) * sin(phi) * cos(phi)) - 0.25 * sq(sin(r - t)) * sin(phi) * cos(phi) / r;
}
__device__ double S5f(double r, double z, double phi, double t, double g) {
  const double cp2 = sq(cos(phi)), sp2 = sq(sin(phi));
  const double t1 = 0.25 * sin(r - t) * cos(r - t) * cp2;
  const double t2 = 0.25 * cos(r - t) * sin(z - t) * cp2;
  const double t3 = 0.25 * sin(z - t) * cos(z - t);
  const double t4 = 0.25 * sin(r - t) * cos(z - t) * cp2;
  const double t5 = 0.25 * (sin(r - t) - sin(z - t)) * sin(z - t) * sp2 / r;
  const double t6 = (g / (g - 1) + 1 + 0.5 * sin((r + z) - 2 * t) + 0.25 * sq(sin(z - t)) + 0.25 * sq(sin(r - t)) * cp2) / r;
  return t1 + t2 + t3 + t4 + t5 + t6;
}
__device__ double S6f(double r, double z, double phi, double t) { return -(0.5 * sin(z - t) * cos(phi) / r); }
__device__ double S7f(double r, double phi, double t) { return 0.5 * sin(r - t) * cos(phi) / r; }

// The Fourier derivative in phi at one point (Lh.f90:100-122): v holds this
// lane's plane value, the 2*LP planes of the point sit on adjacent lanes.
// Returns acc + sum_d (Fzzsin(d) sink(kk,d) + Fzzcos(d) cosk(kk,d)) term by
// term (minus: acc - ... - ...). Every lane of the warp must call it. LP is
// Lphi, a template parameter so the sums unroll to straight-line code.
template <int LP>
__device__ __forceinline__ double fourier(const KC& K, double v, int kk, double acc, bool minus) {
  constexpr int NPH = 2 * LP;
  const int base = (threadIdx.x & 31) & ~(NPH - 1);
  double fs[LP], fc[LP];
#pragma unroll
  for (int d = 0; d < LP; ++d) { fs[d] = 0.0; fc[d] = 0.0; }
#pragma unroll
  for (int q = 0; q < NPH; ++q) {
    const double f = __shfl_sync(0xffffffffu, v, base + q);
#pragma unroll
    for (int d = 0; d < LP; ++d) {
      fs[d] = fs[d] + K.sink[d][q] * f;
      fc[d] = fc[d] + K.cosk[d][q] * f;
    }
  }
#pragma unroll
  for (int d = 0; d < LP; ++d) {
    const double sd = fs[d] / LP, cd = fc[d] / LP;
    const double fzs = -((double)(d + 1) * cd), fzc = (double)(d + 1) * sd;
    if (minus)
      acc = acc - fzs * K.sink[d][kk] - fzc * K.cosk[d][kk];
    else
      acc = acc + fzs * K.sink[d][kk] + fzc * K.cosk[d][kk];
  }
  return acc;
}

// conserved (r*B1, r*B2 in slots 5, 6) -> primitives at radius rad
struct PrimC {
  double rho, u, v, w, E, B1, B2, B3, rB1, rB2, rB3, S, T, K;
};
__device__ __forceinline__ void prim_c(const Phys& P, const double* U, double rad, bool dquirk, PrimC& q) {
  q.rho = U[0];
  q.u = U[1] / q.rho;
  q.v = U[2] / q.rho;
  q.w = U[3] / q.rho;
  q.E = U[4];
  q.rB1 = U[5];
  q.rB2 = U[6];
  q.B1 = q.rB1 / rad;
  q.B2 = q.rB2 / rad;
  q.B3 = U[7];
  q.rB3 = q.B3 * rad;
  const double BB = sq(q.B1) + sq(q.B2) + sq(q.B3);
  const double p = dquirk ? P.gamma1 * (q.E - 0.5 * q.rho * (sq(q.u) + sq(q.v) - sq(q.w)) - 0.5 * BB)
                          : P.gamma1 * (q.E - 0.5 * q.rho * (sq(q.u) + sq(q.v) + sq(q.w)) - 0.5 * BB);
  q.S = p + 0.5 * BB;
  q.T = q.E + q.S;
  q.K = q.u * q.B1 + q.v * q.B2 + q.w * q.B3;
}
__device__ __forceinline__ void flux_r(const PrimC& q, const double* U, double* F) {
  F[0] = U[1];
  F[1] = q.rho * sq(q.u) + q.S - sq(q.B1);
  F[2] = q.rho * q.u * q.v - q.B1 * q.B2;
  F[3] = q.rho * q.u * q.w - q.B1 * q.B3;
  F[4] = q.T * q.u - q.K * q.B1;
  F[5] = 0.0;
  F[6] = q.u * q.rB2 - q.v * q.rB1;
  F[7] = q.u * q.B3 - q.w * q.B1;
}
__device__ __forceinline__ void flux_z(const PrimC& q, const double* U, double* F) {
  F[0] = U[2];
  F[1] = q.rho * q.u * q.v - q.B1 * q.B2;
  F[2] = q.rho * sq(q.v) + q.S - sq(q.B2);
  F[3] = q.rho * q.v * q.w - q.B2 * q.B3;
  F[4] = q.T * q.v - q.K * q.B2;
  F[5] = q.v * q.rB1 - q.u * q.rB2;
  F[6] = 0.0;
  F[7] = q.v * q.B3 - q.w * q.B2;
}
__device__ __forceinline__ void flux_phi(const PrimC& q, const double* U, double* F) {
  F[0] = U[3];
  F[1] = q.rho * q.u * q.w - q.B1 * q.B3;
  F[2] = q.rho * q.v * q.w - q.B2 * q.B3;
  F[3] = q.rho * sq(q.w) + q.S - sq(q.B3);
  F[4] = q.T * q.w - q.K * q.B3;
  F[5] = q.w * q.rB1 - q.u * q.rB3;
  F[6] = q.w * q.rB2 - q.v * q.rB3;
  F[7] = 0.0;
}

__device__ __forceinline__ long long cp_of(const KC& K, int i, int j, int kk) {
  return (long long)i + (long long)K.nx2 * (j + (long long)K.ny2 * kk);
}

// --------------------------------------------------------------- set_bc ----
// One x ghost (i = 0 or nx+1) at row j from the interior (set_bc.f90:5-63);
// evenex/oddex rewrite modes 1-6 and leave the cubic slots, which are zero
// there throughout (the reconstruction clears them, nothing else writes).
__device__ __forceinline__ double xghost(const KC& K, const double* __restrict__ U, int right, int j, int kk, int s) {
  const int n = s < 48 ? s / NQC : (s < 51 ? 5 : 6);
  const int d = s < 48 ? s % NQC : -1;
  const int bc = right ? K.bc_r : K.bc_l;
  const int per = right ? 1 : K.nx;       // periodic source column
  const int adj = right ? K.nx : 1;       // mirror source column
  if (bc == 1) return ld(U + cp_of(K, per, j, kk) + K.ncp * s);
  if (bc == 4) {
    const double v = ld(U + cp_of(K, per, j, kk) + K.ncp * s);
    if (n == 5 || n == 6) return right ? v * K.rb / K.ra : v * K.ra / K.rb;
    return v;
  }
  if (bc == 5) {
    if (n == 7) return d == 0 ? (right ? 1.0 / K.rb : 1.0 / K.ra) : 0.0;
    return ld(U + cp_of(K, per, j, kk) + K.ncp * s);
  }
  // 2: evenex of every variable; 3 (left): evenex except oddex of rho u
  // and of r*B_r, the latter from the mirrored row
  if (d < 0) return 0.0;
  bool odd = false;
  int jj = j;
  if (bc == 3) {
    odd = (n == 1 || n == 5);
    if (n == 5) jj = K.ny + 1 - j;
  }
  const double v = ld(U + cp_of(K, adj, jj, kk) + K.ncp * slotc(n, d));
  const bool flip = (d == 1 || d == 4);
  return (flip != odd) ? -v : v;
}

__global__ void __launch_bounds__(128) k_cy_set_bc(const __grid_constant__ KC K, double* __restrict__ U,
                                                   const ScalC* __restrict__ sc) {
  if (sc && !sc->active) return;
  const long long q = gtid();
  const long long nxg = 2LL * K.ny * K.nph, nyg = 2LL * K.nx2 * K.nph;
  if (q < nxg) {
    const int kk = (int)(q % K.nph);
    const long long r = q / K.nph;
    const int right = r < K.ny ? 1 : 0;
    const int j = (int)(r % K.ny) + 1;
    const int gi = right ? K.nx + 1 : 0;
    double* dst = U + cp_of(K, gi, j, kk);
    for (int s = 0; s < NSC; ++s) dst[K.ncp * s] = xghost(K, U, right, j, kk, s);
    return;
  }
  if (q >= nxg + nyg) return;
  const long long q2 = q - nxg;
  const int kk = (int)(q2 % K.nph);
  const long long r = q2 / K.nph;
  const int top = r < K.nx2 ? 1 : 0;
  const int i = (int)(r % K.nx2);
  const int bc = top ? K.bc_u : K.bc_d;
  const int src = top ? (bc == 1 ? 1 : K.ny) : (bc == 1 ? K.ny : 1);
  const int gj = top ? K.ny + 1 : 0;
  double* dst = U + cp_of(K, i, gj, kk);
  const bool inlet = !top && bc == 4 && i >= 1 && i <= K.nx && K.ra + i * K.hr <= K.jet_r;
  for (int s = 0; s < NSC; ++s) {
    double v;
    if (i >= 1 && i <= K.nx)
      v = ld(U + cp_of(K, i, src, kk) + K.ncp * s);
    else
      v = xghost(K, U, i == K.nx + 1, src, kk, s);
    if (inlet && !(s < 48 && s % NQC == 0)) v = 0.0;
    dst[K.ncp * s] = v;
  }
}

// ------------------------------------------------------------- faces -------
// One face point of one plane: traces of both cells from modes 1-6
// (Lh.f90:155-166, 230-241), fluxes at the face radius, eigenvalueMm of the
// B traces, the 1-D flux of flux_type (Lh.f90:300-367), the LF edge fields
// (LhEz.f90:5-34), and their d/dphi over the planes (LhEz.f90:63-127).
// Output per point (index kk + nph*(g + 5*face)): F[0..6], E, E', dE/dphi.
template <int DIR, int LP>
__global__ void __launch_bounds__(128) k_cy_face(const __grid_constant__ KC K, const double* __restrict__ U,
                                                 double* __restrict__ FH, const ScalC* __restrict__ sc) {
  if (sc && !sc->active) return;
  const long long q = gtid();
  const long long nf = DIR == 0 ? K.nxf : K.nyf;   // faces x nph
  const long long npts = nf * NG;
  const bool valid = q < npts;
  const int kk = (int)(q % K.nph);
  const long long r = q / K.nph;
  const int g = (int)(r % NG);
  const long long f = r / NG;
  int i = 0, j = 0;
  if (DIR == 0) { i = (int)(f % (K.nx + 1)); j = (int)(f / (K.nx + 1)) + 1; }
  else { i = (int)(f % K.nx) + 1; j = (int)(f / K.nx); }
  double Ez = 0.0;
  if (valid) {
    const long long cA = cp_of(K, i, j, kk);
    const long long cB = DIR == 0 ? cp_of(K, i + 1, j, kk) : cp_of(K, i, j + 1, kk);
    const double* tA = DIR == 0 ? K.B.phiGR[g] : K.B.phiGU[g];
    const double* tB = DIR == 0 ? K.B.phiGL[g] : K.B.phiGD[g];
    double UA[NE], UB[NE];
#pragma unroll
    for (int n = 0; n < NE; ++n) {
      double a = 0.0, b = 0.0;
#pragma unroll
      for (int d = 0; d < NQC; ++d) {
        a = a + ld(U + cA + K.ncp * (NQC * n + d)) * tA[d];
        b = b + ld(U + cB + K.ncp * (NQC * n + d)) * tB[d];
      }
      UA[n] = a;
      UB[n] = b;
    }
    const double re = DIR == 0 ? K.ra + i * K.hr : K.ra + (i - 0.5) * K.hr + K.hr1 * K.B.lam[g];
    PrimC pa, pb;
    prim_c(K.P, UA, re, false, pa);
    prim_c(K.P, UB, re, DIR == 1, pb);   // Lh.f90:284: the D side's pressure takes -w^2
    double FA[NE], FB[NE];
    if (DIR == 0) { flux_r(pa, UA, FA); flux_r(pb, UB, FB); }
    else { flux_z(pa, UA, FA); flux_z(pb, UB, FB); }
    double VA[NE], VB[NE];
#pragma unroll
    for (int n = 0; n < NE; ++n) { VA[n] = UA[n]; VB[n] = UB[n]; }
    VA[5] = pa.B1; VA[6] = pa.B2;
    VB[5] = pb.B1; VB[6] = pb.B2;
    double aMax, aMin, bMax, bMin;
    gdf::fast_speeds(K.P, VA, DIR, aMax, aMin);
    gdf::fast_speeds(K.P, VB, DIR, bMax, bMin);
    const double SR = fmax2(aMax, bMax), SL = fmin2(aMin, bMin);
    // FR1 = F of the far cell's trace, FL1 = F of the near one
    double Fh[7];
    if (K.flux == 1) {
      const double s = fmax2(fabs(SR), fabs(SL));
#pragma unroll
      for (int n = 0; n < 7; ++n) Fh[n] = 0.5 * (FB[n] + FA[n] - s * (UB[n] - UA[n]));
    } else if (K.flux == 2) {
      if (SR < 0) {
#pragma unroll
        for (int n = 0; n < 7; ++n) Fh[n] = FB[n];
      } else if (SL > 0) {
#pragma unroll
        for (int n = 0; n < 7; ++n) Fh[n] = FA[n];
      } else {
#pragma unroll
        for (int n = 0; n < 7; ++n) Fh[n] = (SR * FA[n] - SL * FB[n] + SL * SR * (UB[n] - UA[n])) / (SR - SL);
      }
    } else {
#pragma unroll
      for (int n = 0; n < 7; ++n) Fh[n] = 0.5 * (FB[n] + FA[n]);
    }
    const int m = DIR == 0 ? 1 : 2;
    const double S = fmax2(fabs(UA[m] / UA[0]), fabs(UB[m] / UB[0]));
    double E1;
    if (DIR == 0) {
      E1 = -(0.5 * (FA[6] + FB[6] - S * (UB[6] - UA[6])));
      Ez = 0.5 * (FA[7] + FB[7] - S * (UB[7] - UA[7]));
    } else {
      E1 = 0.5 * (FA[5] + FB[5] - S * (UB[5] - UA[5]));
      Ez = -(0.5 * (FA[7] + FB[7] - S * (UB[7] - UA[7])));
    }
#pragma unroll
    for (int n = 0; n < 7; ++n) FH[npts * n + q] = Fh[n];
    FH[npts * 7 + q] = E1;
    FH[npts * 8 + q] = Ez;
  }
  const double dE = fourier<LP>(K, Ez, kk, 0.0, DIR == 1);
  if (valid) FH[npts * 9 + q] = dE;
}

// ------------------------------------------------------------ vertices -----
// Corner values from modes 1-10 and LF_Flux_2D.f90 (LhEz.f90:129-161)
__global__ void __launch_bounds__(128) k_cy_vertex(const __grid_constant__ KC K, const double* __restrict__ U,
                                                   double* __restrict__ EzV, const ScalC* __restrict__ sc) {
  if (sc && !sc->active) return;
  const long long q = gtid();
  if (q >= K.nvx) return;
  const int kk = (int)(q % K.nph);
  const long long v = q / K.nph;
  const int i = (int)(v % (K.nx + 1)), j = (int)(v / (K.nx + 1));
  // corner c of cell (ci, cj): vars rho, rho u, rho v, r B_r, r B_z
  auto corner = [&](int ci, int cj, const double* tab, double* out) {
    const long long c = cp_of(K, ci, cj, kk);
    const int vars[5] = {0, 1, 2, 5, 6};
#pragma unroll
    for (int a = 0; a < 5; ++a) {
      const int n = vars[a];
      double s = 0.0;
#pragma unroll
      for (int d = 0; d < NPC; ++d) {
        const int sl = slotc(n, d);
        if (sl >= 0) s = s + ld(U + c + K.ncp * sl) * tab[d];
      }
      out[a] = s;
    }
  };
  double RU[5], LU[5], RD[5], LD[5];
  corner(i + 1, j + 1, K.B.phiLD, RU);   // URU1 = ULD(i+1, j+1)
  corner(i, j + 1, K.B.phiRD, LU);       // ULU1 = URD(i, j+1)
  corner(i + 1, j, K.B.phiLU, RD);       // URD1 = ULU(i+1, j)
  corner(i, j, K.B.phiRU, LD);           // ULD1 = URU(i, j)
  const double ax = fmax2(fmax2(fmax2(fabs(RU[1] / RU[0]), fabs(LU[1] / LU[0])), fabs(RD[1] / RD[0])), fabs(LD[1] / LD[0]));
  const double ay = fmax2(fmax2(fmax2(fabs(RU[2] / RU[0]), fabs(LU[2] / LU[0])), fabs(RD[2] / RD[0])), fabs(LD[2] / LD[0]));
  auto ez = [](const double* V) { return (V[2] / V[0]) * V[3] - (V[1] / V[0]) * V[4]; };
  const double eRU = ez(RU), eLU = ez(LU), eRD = ez(RD), eLD = ez(LD);
  EzV[q] = 0.25 * (eRU + eLU + eRD + eLD) - 0.25 * ay * (0.5 * (RU[3] + LU[3]) - 0.5 * (RD[3] + LD[3])) +
           0.25 * ax * (0.5 * (RU[4] + RD[4]) - 0.5 * (LU[4] + LD[4]));
}

// ---------------------------------------------------------------- cells ----
__device__ __forceinline__ double combine(int KIND, double u, double du, double dt, double* X, double* U0, long long o) {
  if (KIND == KIND_S1) {
    const double x = u + dt * du;
    U0[o] = u;
    X[o] = x;
    return x;
  }
  if (KIND == KIND_S2) {
    const double v = X[o] + dt * du;
    const double x = (3.0 / 4.0) * U0[o] + (1.0 / 4.0) * v;
    X[o] = x;
    return x;
  }
  const double v = X[o] + dt * du;
  return (1.0 / 3.0) * U0[o] + (2.0 / 3.0) * v;
}

// k_cy_cell stages the 54 slots of its cell plane in shared memory once and
// reads them there at each of the 25 Gauss points (GDF_CY_STAGE=0: every
// point reads them from global memory through L1)
#ifndef GDF_CY_STAGE
#define GDF_CY_STAGE 1
#endif
constexpr int CY_CELL_BS = GDF_CY_STAGE ? 64 : 128;

template <int KIND, int LP>
__global__ void __launch_bounds__(CY_CELL_BS) k_cy_cell(const __grid_constant__ KC K, double* __restrict__ U,
                                                        double* __restrict__ X, double* __restrict__ U0,
                                                        double* __restrict__ T, const double* __restrict__ FXH,
                                                        const double* __restrict__ FYH, const ScalC* __restrict__ sc) {
  __shared__ double cms[GDF_CY_STAGE ? NSC * CY_CELL_BS : 1];
  if (KIND != KIND_LH && !sc->active) return;
  const long long q = gtid();
  const long long nitem = (long long)K.nx * K.ny * K.nph;
  const bool valid = q < nitem;
  const int kk = (int)(q % K.nph);
  const long long c = q / K.nph;
  const int i = valid ? (int)(c % K.nx) + 1 : 1, j = valid ? (int)(c / K.nx) + 1 : 1;
  const long long cp = cp_of(K, i, j, kk);
  const double trk = sc ? (KIND == KIND_LH ? sc->trk[0] : sc->trk[KIND - 1]) : 0.0;
  const double rc = K.ra + (i - 0.5) * K.hr;
  const double zc = K.za + (j - 0.5) * K.hz;
  double du[NE][NQC];
#pragma unroll
  for (int n = 0; n < NE; ++n)
#pragma unroll
    for (int d = 0; d < NQC; ++d) du[n][d] = 0.0;
  if (GDF_CY_STAGE) {
    // each thread stages its own plane's slots (its own column: no barrier);
    // a thread past the end sees rho = 1 and zeros, as below
#pragma unroll 6
    for (int sl = 0; sl < NSC; ++sl)
      cms[sl * CY_CELL_BS + threadIdx.x] = valid ? ld(U + cp + K.ncp * sl) : (sl == 0 ? 1.0 : 0.0);
  }
  // volume (Lh.f90:14-146)
#pragma unroll 1
  for (int a = 0; a < NG; ++a) {
    const double rad = rc + K.hr1 * K.B.lam[a];
#pragma unroll 1
    for (int b = 0; b < NG; ++b) {
      const double* G = K.B.phiG[a][b];
      double Uv[NE];
#pragma unroll
      for (int n = 0; n < NE; ++n) {
        double s = 0.0;
#pragma unroll
        for (int d = 0; d < NPC; ++d) {
          const int sl = slotc(n, d);
          if (sl >= 0)
            s = s + (GDF_CY_STAGE ? cms[sl * CY_CELL_BS + threadIdx.x]
                                  : (valid ? ld(U + cp + K.ncp * sl) : (n == 0 && d == 0 ? 1.0 : 0.0))) * G[d];
        }
        Uv[n] = s;
      }
      PrimC pq;
      prim_c(K.P, Uv, rad, false, pq);
      double Fx[NE], Fy[NE], Fz[NE];
      flux_r(pq, Uv, Fx);
      flux_z(pq, Uv, Fy);
      flux_phi(pq, Uv, Fz);
      const double wab = 0.25 * K.B.w[a] * K.B.w[b];
      double C[NE] = {0, 0, 0, 0, 0, 0, 0, 0};
      if (K.src) {
        const double zz = zc + K.hz1 * K.B.lam[b], ph = K.phi[kk];
        C[0] = S1f(rad, zz, trk);
        C[1] = S2f(rad, zz, ph, trk);
        C[2] = S3f(rad, zz, ph, trk);
        C[3] = S4f(rad, zz, ph, trk);
        C[4] = S5f(rad, zz, ph, trk, K.P.gamma);
        C[5] = rad * S6f(rad, zz, ph, trk);
        C[6] = rad * S7f(rad, ph, trk);
      }
#pragma unroll
      for (int n = 0; n < NE; ++n) {
        // RHS of Lh.f90:73-77: geometric source, then the phi derivative
        double R;
        if (n == 0) R = 0.0 - Fx[0];
        else if (n == 1) R = Fz[3] - Fx[1];
        else if (n == 2) R = 0.0 - Fx[2];
        else if (n == 3) R = -Fx[3] - Fx[3];
        else if (n == 4) R = 0.0 - Fx[4];
        else R = 0.0;
        if (n < 7) R = fourier<LP>(K, Fz[n], kk, R, true);
        R = R / rad + C[n];
        const double* PX = K.B.phixG[a][b];
        const double* PY = K.B.phiyG[a][b];
#pragma unroll
        for (int d = 0; d < NQC; ++d) {
          if (d > 0) du[n][d] = du[n][d] + wab * (Fx[n] * PX[d] + Fy[n] * PY[d]);
          if (n < 7) du[n][d] = du[n][d] + wab * R * G[d];
        }
      }
    }
  }
  if (!valid) return;
  // surface terms (Lh.f90:370-407; var 8 from the edge fields, LhEz.f90:37-55)
  const long long npx = K.nxf * NG, npy = K.nyf * NG;
  const long long fR = (long long)i + (K.nx + 1) * (long long)(j - 1), fL = fR - 1;
  const long long fU = (long long)(i - 1) + (long long)K.nx * j, fD = fU - K.nx;
#pragma unroll
  for (int n = 0; n < NE; ++n) {
    const int qx = n < 7 ? n : 8, qy = n < 7 ? n : 8;
#pragma unroll
    for (int d = 0; d < NQC; ++d) {
      double acc = du[n][d];
#pragma unroll
      for (int g = 0; g < NG; ++g) {
        const double r1 = ld(FXH + npx * qx + kk + K.nph * (g + NG * fR));
        const double l1 = ld(FXH + npx * qx + kk + K.nph * (g + NG * fL));
        acc = acc - K.cxs * K.B.w[g] * (r1 * K.B.phiGR[g][d] - l1 * K.B.phiGL[g][d]);
      }
#pragma unroll
      for (int g = 0; g < NG; ++g) {
        const double u1 = ld(FYH + npy * qy + kk + K.nph * (g + NG * fU));
        const double d1 = ld(FYH + npy * qy + kk + K.nph * (g + NG * fD));
        if (n < 7)
          acc = acc - K.czs * K.B.w[g] * (u1 * K.B.phiGU[g][d] - d1 * K.B.phiGD[g][d]);
        else
          acc = acc + K.czs * K.B.w[g] * (u1 * K.B.phiGU[g][d] - d1 * K.B.phiGD[g][d]);
      }
      du[n][d] = acc / K.B.mm[d];
    }
  }
  if (KIND == KIND_LH) {
#pragma unroll
    for (int n = 0; n < NE; ++n)
#pragma unroll
      for (int d = 0; d < NQC; ++d) T[cp + K.ncp * (NQC * n + d)] = du[n][d];
    for (int s = 48; s < NSC; ++s) T[cp + K.ncp * s] = 0.0;
    return;
  }
  const double dt = sc->dt;
#pragma unroll
  for (int n = 0; n < NE; ++n)
#pragma unroll
    for (int d = 0; d < NQC; ++d) {
      const long long o = cp + K.ncp * (NQC * n + d);
      U[o] = combine(KIND, U[o], du[n][d], dt, X, U0, o);
    }
  for (int s = 48; s < NSC; ++s) {
    const long long o = cp + K.ncp * s;
    U[o] = combine(KIND, U[o], 0.0, dt, X, U0, o);
  }
}

// ---------------------------------------------------------------- face B ---
// dBr on r-faces, dBz on z-faces (LhEz.f90:163-200) and the combination.
template <int KIND>
__global__ void __launch_bounds__(128) k_cy_bface(const __grid_constant__ KC K, const double* __restrict__ FXH,
                                                  const double* __restrict__ FYH, const double* __restrict__ EzV,
                                                  double* __restrict__ BR, double* __restrict__ BRX,
                                                  double* __restrict__ BR0, double* __restrict__ BZ,
                                                  double* __restrict__ BZX, double* __restrict__ BZ0,
                                                  const ScalC* __restrict__ sc) {
  if (KIND != KIND_LH && !sc->active) return;
  const long long q = gtid();
  const double trk = sc ? (KIND == KIND_LH ? sc->trk[0] : sc->trk[KIND - 1]) : 0.0;
  if (q < K.nxf) {
    // thread order = Br(0:nx, 1:ny, 0:nph-1) memory order
    const int i = (int)(q % (K.nx + 1));
    const long long r = q / (K.nx + 1);
    const int j = (int)(r % K.ny) + 1, kk = (int)(r / K.ny);
    const long long f = (long long)i + (K.nx + 1) * (long long)(j - 1);
    const long long npx = K.nxf * NG;
    const double re = K.ra + i * K.hr;
    const double vU = ld(EzV + kk + K.nph * ((long long)i + (K.nx + 1) * (long long)j));
    const double vD = ld(EzV + kk + K.nph * ((long long)i + (K.nx + 1) * (long long)(j - 1)));
    double S6v[NG];
    if (K.src) {
      const double zc = K.za + (j - 0.5) * K.hz;
#pragma unroll
      for (int g = 0; g < NG; ++g) S6v[g] = S6f(re, zc + K.hz1 * K.B.lam[g], K.phi[kk], trk);
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      double acc = 0.0;
#pragma unroll
      for (int g = 0; g < NG; ++g) {
        const long long p = kk + K.nph * (g + NG * f);
        acc = acc + 0.5 * K.B.w[g] * ld(FXH + npx * 7 + p) * K.B.EzyG[g][d];
        acc = acc + 0.5 * K.B.w[g] * ld(FXH + npx * 9 + p) * K.B.EzG[g][d];
        if (K.src) acc = acc + 0.5 * K.B.w[g] * re * S6v[g] * K.B.EzG[g][d];
      }
      const double dB = (acc - vU * K.B.EzU[d] / K.hz + vD * K.B.EzD[d] / K.hz) / K.B.mmE[d];
      const long long o = q + K.nxf * d;
      if (KIND == KIND_LH) BRX[o] = dB;
      else BR[o] = combine(KIND, BR[o], dB, sc->dt, BRX, BR0, o);
    }
    return;
  }
  const long long q2 = q - K.nxf;
  if (q2 >= K.nyf) return;
  const int i = (int)(q2 % K.nx) + 1;
  const long long r = q2 / K.nx;
  const int j = (int)(r % (K.ny + 1)), kk = (int)(r / (K.ny + 1));
  const long long f = (long long)(i - 1) + (long long)K.nx * j;
  const long long npy = K.nyf * NG;
  const double vR = ld(EzV + kk + K.nph * ((long long)i + (K.nx + 1) * (long long)j));
  const double vL = ld(EzV + kk + K.nph * ((long long)(i - 1) + (K.nx + 1) * (long long)j));
  double S7v[NG], rpv[NG];
  if (K.src) {
    const double rc = K.ra + (i - 0.5) * K.hr;
#pragma unroll
    for (int g = 0; g < NG; ++g) {
      rpv[g] = rc + K.hr1 * K.B.lam[g];
      S7v[g] = S7f(rpv[g], K.phi[kk], trk);
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double acc = 0.0;
#pragma unroll
    for (int g = 0; g < NG; ++g) {
      const long long p = kk + K.nph * (g + NG * f);
      acc = acc - 0.5 * K.B.w[g] * ld(FYH + npy * 7 + p) * K.B.EzxG[g][d];
      acc = acc + 0.5 * K.B.w[g] * ld(FYH + npy * 9 + p) * K.B.EzG[g][d];
      if (K.src) acc = acc + 0.5 * K.B.w[g] * rpv[g] * S7v[g] * K.B.EzG[g][d];
    }
    const double dB = (acc + vR * K.B.EzR[d] / K.hr - vL * K.B.EzL[d] / K.hr) / K.B.mmE[d];
    const long long o = q2 + K.nyf * d;
    if (KIND == KIND_LH) BZX[o] = dB;
    else BZ[o] = combine(KIND, BZ[o], dB, sc->dt, BZX, BZ0, o);
  }
}

// ------------------------------------------------------------- limiter -----
// B = rB / r on the P2 modes of every cell plane, ghosts included
// (TVB_Limiter_P2.f90:14-40) -> BP[6*(n-5) + d]
__global__ void __launch_bounds__(128) k_cy_bproj(const __grid_constant__ KC K, const double* __restrict__ U,
                                                  double* __restrict__ BP, const ScalC* __restrict__ sc) {
  if (sc && !sc->active) return;
  const long long q = gtid();
  if (q >= K.ncp) return;
  const int i = (int)(q % K.nx2);
  double acc[2][NQC];
#pragma unroll
  for (int v = 0; v < 2; ++v)
#pragma unroll
    for (int d = 0; d < NQC; ++d) acc[v][d] = 0.0;
  const double r0 = K.ra + (i - 0.5) * K.hr;
#pragma unroll 1
  for (int a = 0; a < NG; ++a) {
    const double rad = r0 + K.hr1 * K.B.lam[a];
#pragma unroll 1
    for (int b = 0; b < NG; ++b) {
      const double* G = K.B.phiG[a][b];
      const double wab = 0.25 * K.B.w[a] * K.B.w[b];
#pragma unroll
      for (int v = 0; v < 2; ++v) {
        const int n = 5 + v;
        double s = 0.0;
#pragma unroll
        for (int d = 0; d < NPC; ++d) {
          const int sl = slotc(n, d);
          if (sl >= 0) s = s + ld(U + q + K.ncp * sl) * G[d];
        }
#pragma unroll
        for (int d = 0; d < NQC; ++d) acc[v][d] = acc[v][d] + wab * s / rad * G[d] / K.B.mm[d];
      }
    }
  }
#pragma unroll
  for (int v = 0; v < 2; ++v)
#pragma unroll
    for (int d = 0; d < NQC; ++d) BP[q + K.ncp * (NQC * v + d)] = acc[v][d];
}

__device__ __forceinline__ void mv8(const double* A, const double* x, double* y) {
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) acc = acc + A[r + 8 * k] * x[k];
    y[r] = acc;
  }
}

// characteristic limiting in one direction (TVB_Limiter_P2.f90:57-125):
// L of the differences, minmod, R; the left vectors are built and used
// before the right ones (the same values, one matrix live at a time)
__device__ __forceinline__ void char_dir(const Phys& P, int dir, const double* m, const double* DR, const double* DL,
                                         const double* Dp, const double* Dm, double Mh2, double* Yp, double* Ym) {
  const double rho = m[0], u1 = m[1] / rho, u2 = m[2] / rho, u3 = m[3] / rho;
  gdf::EigFrame f;
  gdf::eigen_frame(P, dir, rho, u1, u2, u3, m[4], m[5], m[6], m[7], f);
  double t1[NE], t2[NE], tp[NE], tm[NE];
  {
    double L[64];
    gdf::eigen_left(dir, f, rho, u1, u2, u3, m[5], m[6], m[7], L);
    mv8(L, DR, t1);
    mv8(L, DL, t2);
    mv8(L, Dp, tp);
    mv8(L, Dm, tm);
  }
  double R[64];
  gdf::eigen_right(dir, f, rho, u1, u2, u3, m[5], m[6], m[7], R);
  double mod[NE];
#pragma unroll
  for (int k = 0; k < NE; ++k) mod[k] = gdf::minmod1(tp[k], t1[k], t2[k], Mh2);
  mv8(R, mod, Yp);
#pragma unroll
  for (int k = 0; k < NE; ++k) mod[k] = gdf::minmod1(tm[k], t1[k], t2[k], Mh2);
  mv8(R, mod, Ym);
}

// the P2 mode d of variable n with r*B replaced by B (the projection)
__device__ __forceinline__ double modeB(const KC& K, const double* U, const double* BP, long long c, int n, int d) {
  return (n == 5 || n == 6) ? ld(BP + c + K.ncp * (NQC * (n - 5) + d)) : ld(U + c + K.ncp * (NQC * n + d));
}

__global__ void __launch_bounds__(64) k_cy_tvb(const __grid_constant__ KC K, double* __restrict__ U,
                                               const double* __restrict__ BP, int32_t* __restrict__ flags,
                                               const ScalC* __restrict__ sc) {
  if (sc && !sc->active) return;
  const long long q = gtid();
  if (q >= (long long)K.nx * K.ny * K.nph) return;
  const int i = (int)(q % K.nx) + 1;
  const long long r = q / K.nx;
  const int j = (int)(r % K.ny) + 1, kk = (int)(r / K.ny);
  const long long c = cp_of(K, i, j, kk);
  const long long cE = cp_of(K, i + 1, j, kk), cW = cp_of(K, i - 1, j, kk);
  const long long cN = cp_of(K, i, j + 1, kk), cS = cp_of(K, i, j - 1, kk);
  double m[NE];
#pragma unroll
  for (int n = 0; n < NE; ++n) m[n] = modeB(K, U, BP, c, n, 0);
  const double c23 = 2.0 / 3.0;
  int change = 0;
  double Xp[NE], Xm[NE], Yp[NE], Ym[NE];
  {
    double DR[NE], DL[NE], Dp[NE], Dm[NE];
#pragma unroll
    for (int n = 0; n < NE; ++n) {
      DR[n] = modeB(K, U, BP, cE, n, 0) - m[n];
      DL[n] = m[n] - modeB(K, U, BP, cW, n, 0);
      const double m2 = modeB(K, U, BP, c, n, 1), m4 = modeB(K, U, BP, c, n, 3);
      Dp[n] = m2 + c23 * m4;
      Dm[n] = m2 - c23 * m4;
    }
    char_dir(K.P, 0, m, DR, DL, Dp, Dm, K.Mh2r, Xp, Xm);
#pragma unroll
    for (int n = 0; n < NE; ++n)
      if (fabs(Xp[n] - Dp[n]) > K.change_tol || fabs(Xm[n] - Dm[n]) > K.change_tol) change |= 1 << n;
  }
  {
    double DR[NE], DL[NE], Dp[NE], Dm[NE];
#pragma unroll
    for (int n = 0; n < NE; ++n) {
      DR[n] = modeB(K, U, BP, cN, n, 0) - m[n];
      DL[n] = m[n] - modeB(K, U, BP, cS, n, 0);
      const double m3 = modeB(K, U, BP, c, n, 2), m6 = modeB(K, U, BP, c, n, 5);
      Dp[n] = m3 + c23 * m6;
      Dm[n] = m3 - c23 * m6;
    }
    char_dir(K.P, 1, m, DR, DL, Dp, Dm, K.Mh2z, Yp, Ym);
#pragma unroll
    for (int n = 0; n < NE; ++n)
      if (fabs(Yp[n] - Dp[n]) > K.change_tol || fabs(Ym[n] - Dm[n]) > K.change_tol) change |= 1 << n;
  }
#pragma unroll
  for (int n = 0; n < NE; ++n)
    if (change & (1 << n)) {
      U[c + K.ncp * (NQC * n + 1)] = 0.5 * (Xp[n] + Xm[n]);
      U[c + K.ncp * (NQC * n + 2)] = 0.5 * (Yp[n] + Ym[n]);
      U[c + K.ncp * (NQC * n + 3)] = (3.0 / 4.0) * (Xp[n] - Xm[n]);
      U[c + K.ncp * (NQC * n + 4)] = 0.0;
      U[c + K.ncp * (NQC * n + 5)] = (3.0 / 4.0) * (Yp[n] - Ym[n]);
      if (n == 5)
        for (int s = 48; s < 51; ++s) U[c + K.ncp * s] = 0.0;
      if (n == 6)
        for (int s = 51; s < 54; ++s) U[c + K.ncp * s] = 0.0;
    }
  if (flags) flags[q] = change;
}

// face-B minmod of modes 2-3 against the neighbouring cells' r*B slopes
// (TVB_Limiter_P2.f90:147-210)
__global__ void __launch_bounds__(128) k_cy_faceb(const __grid_constant__ KC K, const double* __restrict__ U,
                                                  double* __restrict__ BR, double* __restrict__ BZ,
                                                  const ScalC* __restrict__ sc) {
  if (sc && !sc->active) return;
  const long long q = gtid();
  if (q < K.nxf) {
    const int i = (int)(q % (K.nx + 1));
    const long long r = q / (K.nx + 1);
    const int j = (int)(r % K.ny) + 1, kk = (int)(r / K.ny);
    const long long cA = cp_of(K, i, j, kk), cB = cp_of(K, i + 1, j, kk);
    const double re = K.ra + i * K.hr;
    auto s = [&](long long c, int sl) { return ld(U + c + K.ncp * sl); };
    const double aR2 = s(cA, slotc(5, 2)) + s(cA, slotc(5, 4)), aR3 = s(cA, slotc(5, 5)) + s(cA, slotc(5, 8));
    const double aL2 = s(cB, slotc(5, 2)) - s(cB, slotc(5, 4)), aL3 = s(cB, slotc(5, 5)) - s(cB, slotc(5, 8));
    BR[q + K.nxf] = gdf::minmod1(BR[q + K.nxf], aR2 * re, aL2 * re, K.Mh2z);
    BR[q + 2 * K.nxf] = gdf::minmod1(BR[q + 2 * K.nxf], aR3 * re, aL3 * re, K.Mh2z);
    return;
  }
  const long long q2 = q - K.nxf;
  if (q2 >= K.nyf) return;
  const int i = (int)(q2 % K.nx) + 1;
  const long long r = q2 / K.nx;
  const int j = (int)(r % (K.ny + 1)), kk = (int)(r / (K.ny + 1));
  const long long cA = cp_of(K, i, j, kk), cB = cp_of(K, i, j + 1, kk);
  const double rc = K.ra + (i - 0.5) * K.hr;
  auto s = [&](long long c, int sl) { return ld(U + c + K.ncp * sl); };
  const double bU2 = s(cA, slotc(6, 1)) + s(cA, slotc(6, 4)), bU3 = s(cA, slotc(6, 3)) + s(cA, slotc(6, 7));
  const double bD2 = s(cB, slotc(6, 1)) - s(cB, slotc(6, 4)), bD3 = s(cB, slotc(6, 3)) - s(cB, slotc(6, 7));
  BZ[q2 + K.nyf] = gdf::minmod1(BZ[q2 + K.nyf], bU2 * rc, bD2 * rc, K.Mh2r);
  BZ[q2 + 2 * K.nyf] = gdf::minmod1(BZ[q2 + 2 * K.nyf], bU3 * rc, bD3 * rc, K.Mh2r);
}

// div_free_Balsara.f90:13-147: r*B of every interior cell plane from its
// four faces and the projection of d(Bphi)/dphi
template <int LP>
__global__ void __launch_bounds__(128) k_cy_divfree(const __grid_constant__ KC K, double* __restrict__ U,
                                                    const double* __restrict__ BR, const double* __restrict__ BZ,
                                                    const ScalC* __restrict__ sc) {
  if (sc && !sc->active) return;
  const long long q = gtid();
  const long long nitem = (long long)K.nx * K.ny * K.nph;
  const bool valid = q < nitem;
  const int kk = (int)(q % K.nph);
  const long long c = q / K.nph;
  const int i = valid ? (int)(c % K.nx) + 1 : 1, j = valid ? (int)(c / K.nx) + 1 : 1;
  const long long cp = cp_of(K, i, j, kk);
  double m8[NQC];
#pragma unroll
  for (int d = 0; d < NQC; ++d) m8[d] = valid ? ld(U + cp + K.ncp * (NQC * 7 + d)) : 0.0;
  double bpp[NQC];
#pragma unroll
  for (int d = 0; d < NQC; ++d) bpp[d] = 0.0;
#pragma unroll 1
  for (int a = 0; a < NG; ++a)
#pragma unroll 1
    for (int b = 0; b < NG; ++b) {
      const double* G = K.B.phiG[a][b];
      double s = 0.0;
#pragma unroll
      for (int d = 0; d < NQC; ++d) s = s + m8[d] * G[d];
      const double dv = fourier<LP>(K, s, kk, 0.0, false);
      const double wab = 0.25 * K.B.w[a] * K.B.w[b];
#pragma unroll
      for (int d = 0; d < NQC; ++d) bpp[d] = bpp[d] + wab * dv * G[d] / K.B.mm[d];
    }
  if (!valid) return;
  auto br = [&](int ii, int d) { return ld(BR + ii + (K.nx + 1) * ((long long)(j - 1) + (long long)K.ny * (kk + (long long)K.nph * d))); };
  auto bz = [&](int jj, int d) { return ld(BZ + (i - 1) + (long long)K.nx * (jj + (long long)(K.ny + 1) * (kk + (long long)K.nph * d))); };
  const double a0R = br(i, 0), a1R = br(i, 1), a2R = br(i, 2);
  const double a0L = br(i - 1, 0), a1L = br(i - 1, 1), a2L = br(i - 1, 2);
  const double b0U = bz(j, 0), b1U = bz(j, 1), b2U = bz(j, 2);
  const double b0D = bz(j - 1, 0), b1D = bz(j - 1, 1), b2D = bz(j - 1, 2);
  const double c10 = -bpp[1], c01 = -bpp[2], c20 = -bpp[3], c11 = -bpp[4], c02 = -bpp[5];
  const double hr = K.hr, hz = K.hz;
  const double a11 = 0.5 * (a1R - a1L), a02 = 0.5 * (a2R + a2L), a12 = 0.5 * (a2R - a2L);
  const double b11 = 0.5 * (b1U - b1D), b20 = 0.5 * (b2U + b2D), b21 = 0.5 * (b2U - b2D);
  const double a20 = (hr / 4) * (c10 - 2.0 / hz * b11);
  const double a21 = (hr / 8) * c11;
  const double b12 = (hz / 8) * c11;
  const double a30 = (hr / 6) * (c20 - 2.0 / hz * b21);
  const double b02 = (hz / 4) * (c01 - 2.0 / hr * a11);
  const double b03 = (hz / 6) * (c02 - 2.0 / hr * a12);
  const double a01 = 0.5 * (a1R + a1L) - (2.0 / 3.0) * a21;
  const double b10 = 0.5 * (b1U + b1D) - (2.0 / 3.0) * b12;
  const double b01 = 0.5 * (b0U - b0D) - (2.0 / 5.0) * b03;
  const double b00 = 0.5 * (b0U + b0D) - (2.0 / 3.0) * b02;
  const double a10 = 0.5 * (a0R - a0L) - (2.0 / 5.0) * a30;
  const double a00 = 0.5 * (a0R + a0L) - (2.0 / 3.0) * a20;
  double* u = U + cp;
  const long long P = K.ncp;
  u[P * slotc(5, 0)] = a00; u[P * slotc(5, 1)] = a10; u[P * slotc(5, 2)] = a01;
  u[P * slotc(5, 3)] = a20; u[P * slotc(5, 4)] = a11; u[P * slotc(5, 5)] = a02;
  u[P * slotc(5, 6)] = a30; u[P * slotc(5, 7)] = a21; u[P * slotc(5, 8)] = a12;
  u[P * slotc(6, 0)] = b00; u[P * slotc(6, 1)] = b10; u[P * slotc(6, 2)] = b01;
  u[P * slotc(6, 3)] = b20; u[P * slotc(6, 4)] = b11; u[P * slotc(6, 5)] = b02;
  u[P * slotc(6, 7)] = b21; u[P * slotc(6, 8)] = b12; u[P * slotc(6, 9)] = b03;
}

// ------------------------------------------------------------------ dt -----
constexpr int DT_BS = 256;

__device__ __forceinline__ double max_skip_nan(double a, double b) { return b > a ? b : a; }

// calculate_dt.f90:14-29: the largest |u_n +- c_f| of the cell averages,
// with B = rB / Rc(i)
__global__ void __launch_bounds__(DT_BS) k_cy_dt_partial(const __grid_constant__ KC K, const double* __restrict__ U,
                                                         double* __restrict__ part, ScalC* __restrict__ sc, int step) {
  if (step == 1 && !sc->active) return;
  __shared__ double sx[DT_BS], sy[DT_BS];
  const long long q = gtid();
  double ax = 0.0, ay = 0.0;
  if (q < (long long)K.nx * K.ny * K.nph) {
    const int i = (int)(q % K.nx) + 1;
    const long long r = q / K.nx;
    const int j = (int)(r % K.ny) + 1, kk = (int)(r / K.ny);
    const long long c = cp_of(K, i, j, kk);
    double V[NE];
#pragma unroll
    for (int n = 0; n < NE; ++n) V[n] = ld(U + c + K.ncp * (NQC * n));
    const double rc = K.ra + (i - 0.5) * K.hr;
    V[5] = V[5] / rc;
    V[6] = V[6] / rc;
    double a1, a2;
    gdf::fast_speeds(K.P, V, 0, a1, a2);
    ax = max_skip_nan(max_skip_nan(ax, fabs(a1)), fabs(a2));
    gdf::fast_speeds(K.P, V, 1, a1, a2);
    ay = max_skip_nan(max_skip_nan(ay, fabs(a1)), fabs(a2));
    if (!(V[0] > 0.0) || !isfinite(V[4])) atomicOr(&sc->status, 1);
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

// step 0: dt only (gdf_cy_dt); 1: a time step (RK3.f90:42-58: clamp to tend,
// the dt < 1e-7 stop, and the stage times tRK)
__global__ void __launch_bounds__(DT_BS) k_cy_dt_final(const __grid_constant__ KC K, const double* __restrict__ part,
                                                       int nblocks, ScalC* __restrict__ sc, int step) {
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
  double dt = K.cfl / (sx[0] / K.hr + sy[0] / K.hz);
  if (!step) {
    sc->dt = dt;
    return;
  }
  const double t0 = sc->t;
  double t;
  if (t0 + dt >= sc->tend) {
    dt = sc->tend - t0;
    t = sc->tend;
  } else {
    t = t0 + dt;
  }
  if (dt < 1e-7) t = sc->tend;
  if (!(dt > 0.0) || !isfinite(dt)) sc->status |= 1;
  sc->dt = dt;
  sc->t = t;
  sc->trk[0] = t0;
  sc->trk[1] = t0 + dt;
  sc->trk[2] = sc->trk[1] - 0.5 * dt;
  sc->active = 1;
  sc->steps += 1;
}

// diagnostics per cell plane: |rho mean|, the smallest Gauss-Lobatto
// pressure (calculate_pmin.f90, with the r*B slots as the reference passes
// them) and, on the plane-0 lane, the cell's sum over (i1, j1, kk) of
// w w |div B|^2 (calculate_totaldiv.f90:14-68)
template <int LP>
__global__ void __launch_bounds__(128) k_cy_diag(const __grid_constant__ KC K, const double* __restrict__ U,
                                                 double* __restrict__ out) {
  const long long q = gtid();
  const long long nitem = (long long)K.nx * K.ny * K.nph;
  const bool valid = q < nitem;
  const int kk = (int)(q % K.nph);
  const long long c = q / K.nph;
  const int i = valid ? (int)(c % K.nx) + 1 : 1, j = valid ? (int)(c / K.nx) + 1 : 1;
  const long long cp = cp_of(K, i, j, kk);
  auto sv = [&](int n, int d) {
    const int sl = slotc(n, d);
    return (valid && sl >= 0) ? ld(U + cp + K.ncp * sl) : 0.0;
  };
  double td = 0.0, pm = 1000000;
  const double rc = K.ra + (i - 0.5) * K.hr;
  for (int a = 0; a < NG; ++a)
    for (int b = 0; b < NG; ++b) {
      double dv = 0.0, g8 = 0.0;
      for (int d = 0; d < NPC; ++d) {
        dv = dv + sv(5, d) * K.B.phixG[a][b][d] + sv(6, d) * K.B.phiyG[a][b][d];
        g8 = g8 + sv(7, d) * K.B.phiG[a][b][d];
      }
      const double ph = fourier<LP>(K, g8, kk, 0.0, false);
      const double v = (dv + ph) / (rc + K.hr1 * K.B.lam[a]);
      const double term = K.B.w[a] * K.B.w[b] * sq(v);
      const int base = (threadIdx.x & 31) & ~(2 * LP - 1);
#pragma unroll
      for (int p = 0; p < 2 * LP; ++p) {
        const double tp = __shfl_sync(0xffffffffu, term, base + p);
        td = td + tp;
      }
      for (int s = 0; s < 2; ++s) {
        double V[NE];
        for (int n = 0; n < NE; ++n) {
          double acc = 0.0;
          for (int d = 0; d < NPC; ++d) acc = acc + sv(n, d) * K.B.phiGLL[s][a][b][d];
          V[n] = acc;
        }
        const double p1 = gdf::pressure(K.P.gamma, V);
        if (p1 < pm) pm = p1;
      }
    }
  if (!valid) return;
  out[q] = fabs(sv(0, 0));
  out[nitem + q] = pm;
  out[2 * nitem + q] = kk == 0 ? td : 0.0;
}

}  // namespace gdfc

// =================================================================== host ==
using namespace gdfc;

struct GdfCyHandle {
  GdfCyConfig cfg{};
  KC K{};
  cudaStream_t st = nullptr;
  double *U = nullptr, *X = nullptr, *U0 = nullptr, *T = nullptr, *BP = nullptr;
  double *BR = nullptr, *BRX = nullptr, *BR0 = nullptr, *BZ = nullptr, *BZX = nullptr, *BZ0 = nullptr;
  double *FXH = nullptr, *FYH = nullptr, *EzV = nullptr, *part = nullptr, *diag = nullptr;
  ScalC* sc = nullptr;
  ScalC* sc_host = nullptr;
  int dt_blocks = 0;
  int uploaded = 0;
  int64_t launches = 0;
  int64_t step_launches = 0;
  cudaGraphExec_t graph = nullptr;
};

namespace {

int fail(int code, const std::string& msg) { return gdf::set_last_error(code, msg.c_str()); }

#define CKC(x)                                                                  \
  do {                                                                          \
    cudaError_t e_ = (x);                                                       \
    if (e_ != cudaSuccess) return fail(GDF_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
  } while (0)

unsigned nblk(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

int check_config(const GdfCyConfig* c) {
  if (!c) return fail(GDF_ERR_ARG, "null configuration");
  if (c->nr < 2 || c->nz < 2) return fail(GDF_ERR_ARG, "the grid needs at least 2 x 2 cells");
  if (c->lphi != 1 && c->lphi != 2 && c->lphi != 4 && c->lphi != 8) return fail(GDF_ERR_ARG, "lphi must be 1, 2, 4 or 8");
  if ((long long)(c->nr + 2) * (c->nz + 2) * 2 * c->lphi > (1LL << 31) / NSC)
    return fail(GDF_ERR_ARG, "grid too large for one device");
  if (c->bc_r != 1 && c->bc_r != 2 && c->bc_r != 4 && c->bc_r != 5) return fail(GDF_ERR_ARG, "bc_r must be 1, 2, 4 or 5");
  if (c->bc_l < 1 || c->bc_l > 5) return fail(GDF_ERR_ARG, "bc_l must be 1..5");
  if (c->bc_u != 1 && c->bc_u != 2) return fail(GDF_ERR_ARG, "bc_u must be 1 or 2");
  if (c->bc_d != 1 && c->bc_d != 2 && c->bc_d != 4) return fail(GDF_ERR_ARG, "bc_d must be 1, 2 or 4");
  if (c->flux_type < 0 || c->flux_type > 2)
    return fail(GDF_ERR_ARG, "flux_type must be 0, 1 or 2 (the reference comments HLLC and HLLD out)");
  if (!(c->rb > c->ra) || !(c->zb > c->za)) return fail(GDF_ERR_ARG, "empty domain");
  if ((c->bc_r == 4 || c->bc_l == 4 || c->bc_r == 5 || c->bc_l == 5) && !(c->ra != 0.0))
    return fail(GDF_ERR_ARG, "boundary codes 4 and 5 divide by ra");
  if (!(c->gamma > 1.0) || !(c->cfl > 0.0) || !(c->tvb_m >= 0.0) || !(c->change_tol >= 0.0))
    return fail(GDF_ERR_ARG, "gamma > 1, cfl > 0, tvb_m >= 0, change_tol >= 0");
  return GDF_OK;
}

// get_basis.f90:1-196 with hx = hr, hy = hz
void build_basis(double hr1, double hz1, BasisC& B) {
  const double lam[NG] = {-0.9061798459386639927976269, -0.5384693101056830910363144, 0,
                          0.5384693101056830910363144, 0.9061798459386639927976269};
  const double w[NG] = {0.2369268850561890875142640, 0.4786286704993664680412915, 0.5688888888888888888888889,
                        0.4786286704993664680412915, 0.2369268850561890875142640};
  const double lamL[NG] = {-1, -0.6546536707079771437983, 0, 0.654653670707977143798, 1};
  const double c23 = 2.0 / 3.0, c25 = 2.0 / 5.0, c13 = 1.0 / 3.0, c35 = 3.0 / 5.0;
  for (int a = 0; a < NG; ++a) { B.lam[a] = lam[a]; B.w[a] = w[a]; }
  auto p2 = [&](double l) { return l * l - c13; };
  auto p3 = [&](double l) { return l * l * l - 3.0 * l / 5.0; };
  auto fill_G = [&](double li, double lj, double* G) {
    G[0] = 1; G[1] = li; G[2] = lj; G[3] = p2(li); G[4] = li * lj; G[5] = p2(lj);
    G[6] = p3(li); G[7] = p2(li) * (lj); G[8] = (li) * p2(lj); G[9] = p3(lj);
  };
  for (int a = 0; a < NG; ++a)
    for (int b = 0; b < NG; ++b) {
      const double li = lam[a], lj = lam[b];
      fill_G(li, lj, B.phiG[a][b]);
      fill_G(lamL[a], lj, B.phiGLL[0][a][b]);
      fill_G(li, lamL[b], B.phiGLL[1][a][b]);
      double* X = B.phixG[a][b];
      double* Y = B.phiyG[a][b];
      X[0] = 0; Y[0] = 0;
      X[1] = 1.0 / hr1; Y[1] = 0;
      X[2] = 0; Y[2] = 1.0 / hz1;
      X[3] = 2.0 * li / hr1; Y[3] = 0;
      X[4] = lj / hr1; Y[4] = li / hz1;
      X[5] = 0; Y[5] = 2.0 * lj / hz1;
      X[6] = (3 * (li * li) - c35) / hr1; Y[6] = 0;
      X[7] = 2.0 * li * lj / hr1; Y[7] = p2(li) / hz1;
      X[8] = p2(lj) / hr1; Y[8] = 2.0 * li * lj / hz1;
      X[9] = 0; Y[9] = (3 * (lj * lj) - c35) / hz1;
    }
  for (int g = 0; g < NG; ++g) {
    const double l = lam[g];
    const double R[NQC] = {1, 1, l, c23, l, p2(l)}, L[NQC] = {1, -1, l, c23, -l, p2(l)};
    const double Uu[NQC] = {1, l, 1, p2(l), l, c23}, D[NQC] = {1, l, -1, p2(l), -l, c23};
    for (int d = 0; d < NQC; ++d) { B.phiGR[g][d] = R[d]; B.phiGL[g][d] = L[d]; B.phiGU[g][d] = Uu[d]; B.phiGD[g][d] = D[d]; }
    B.EzG[g][0] = 1; B.EzG[g][1] = l; B.EzG[g][2] = p2(l);
    B.EzxG[g][0] = 0; B.EzxG[g][1] = 1 / hr1; B.EzxG[g][2] = 2 * l / hr1;
    B.EzyG[g][0] = 0; B.EzyG[g][1] = 1 / hz1; B.EzyG[g][2] = 2 * l / hz1;
  }
  const double ru[NPC] = {1, 1, 1, c23, 1, c23, c25, c23, c23, c25};
  const double lu[NPC] = {1, -1, 1, c23, -1, c23, -c25, c23, -c23, c25};
  const double rd[NPC] = {1, 1, -1, c23, -1, c23, c25, -c23, c23, -c25};
  const double ldv[NPC] = {1, -1, -1, c23, 1, c23, -c25, -c23, -c23, -c25};
  const double mm[NPC] = {1, 1.0 / 3.0, 1.0 / 3.0, 4.0 / 45.0, 1.0 / 9.0, 4.0 / 45.0, 4.0 / 175.0, 4.0 / 135.0,
                          4.0 / 135.0, 4.0 / 175.0};
  for (int d = 0; d < NPC; ++d) {
    B.phiRU[d] = ru[d]; B.phiLU[d] = lu[d]; B.phiRD[d] = rd[d]; B.phiLD[d] = ldv[d]; B.mm[d] = mm[d];
  }
  B.EzR[0] = 1; B.EzR[1] = 1; B.EzR[2] = c23;
  B.EzL[0] = 1; B.EzL[1] = -1; B.EzL[2] = c23;
  for (int d = 0; d < 3; ++d) { B.EzU[d] = B.EzR[d]; B.EzD[d] = B.EzL[d]; }
  B.mmE[0] = 1; B.mmE[1] = 1.0 / 3.0; B.mmE[2] = 4.0 / 45.0;
}

void build_kc(const GdfCyConfig& c, KC& K) {
  std::memset(&K, 0, sizeof(K));
  K.nx = c.nr;
  K.ny = c.nz;
  K.nx2 = c.nr + 2;
  K.ny2 = c.nz + 2;
  K.lphi = c.lphi;
  K.nph = 2 * c.lphi;
  K.ncp = (long long)K.nx2 * K.ny2 * K.nph;
  K.nxf = (long long)(c.nr + 1) * c.nz * K.nph;
  K.nyf = (long long)c.nr * (c.nz + 1) * K.nph;
  K.nvx = (long long)(c.nr + 1) * (c.nz + 1) * K.nph;
  // init_data.f90:18-34
  K.ra = c.ra;
  K.rb = c.rb;
  K.za = c.za;
  K.hr = (c.rb - c.ra) / c.nr;
  K.hz = (c.zb - c.za) / c.nz;
  K.hr1 = 0.5 * K.hr;
  K.hz1 = 0.5 * K.hz;
  K.cxs = 0.5 / K.hr;
  K.czs = 0.5 / K.hz;
  K.Mh2r = c.tvb_m * (K.hr * K.hr);
  K.Mh2z = c.tvb_m * (K.hz * K.hz);
  K.change_tol = c.change_tol;
  K.cfl = c.cfl;
  K.jet_r = c.jet_r;
  K.bc_r = c.bc_r;
  K.bc_l = c.bc_l;
  K.bc_u = c.bc_u;
  K.bc_d = c.bc_d;
  K.flux = c.flux_type;
  K.src = c.rhsc_open == 1;
  K.P.gamma = c.gamma;
  K.P.gamma1 = c.gamma - 1;
  K.P.gflux = 5.0 / 3.0;   // eigenmatrix.f90:19 parameter
  K.P.flux = c.flux_type;
  K.P.kml_w = 1;
  K.P.eig_p_typo = 0;
  K.P.eig_identity = 0;    // eigenmatrix.f90:396-402 commented out
  // get_basis.f90:191-196 (host sin/cos, as the reference's)
  const double pi = 4 * std::atan(1.0), hphi = 2 * pi / K.nph;
  for (int kk = 0; kk < K.nph; ++kk) K.phi[kk] = kk * hphi;
  for (int d = 1; d <= K.lphi; ++d)
    for (int kk = 0; kk < K.nph; ++kk) {
      K.sink[d - 1][kk] = std::sin(d * K.phi[kk]);
      K.cosk[d - 1][kk] = std::cos(d * K.phi[kk]);
    }
  build_basis(K.hr1, K.hz1, K.B);
}

template <class F>
int run(GdfCyHandle* h, F&& launch) {
  launch();
  h->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(GDF_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  return GDF_OK;
}

int launch_set_bc(GdfCyHandle* h, const ScalC* sc) {
  const KC& K = h->K;
  const long long n = (2LL * K.ny + 2LL * K.nx2) * K.nph;
  return run(h, [&] { k_cy_set_bc<<<nblk(n, 128), 128, 0, h->st>>>(K, h->U, sc); });
}

// set_bc, then Lh + LhEz of U fused with the stage's combination (kind)
template <int LP>
int launch_lh_lp(GdfCyHandle* h, int kind, const ScalC* sc) {
  const KC& K = h->K;
  int rc = launch_set_bc(h, sc);
  if (!rc) rc = run(h, [&] { k_cy_face<0, LP><<<nblk(K.nxf * NG, 128), 128, 0, h->st>>>(K, h->U, h->FXH, sc); });
  if (!rc) rc = run(h, [&] { k_cy_face<1, LP><<<nblk(K.nyf * NG, 128), 128, 0, h->st>>>(K, h->U, h->FYH, sc); });
  if (!rc) rc = run(h, [&] { k_cy_vertex<<<nblk(K.nvx, 128), 128, 0, h->st>>>(K, h->U, h->EzV, sc); });
  if (rc) return rc;
  const unsigned nc = nblk((long long)K.nx * K.ny * K.nph, CY_CELL_BS), nf = nblk(K.nxf + K.nyf, 128);
  h->launches++;  // the pair below is two launches
  return run(h, [&] {
    switch (kind) {
      case KIND_LH:
        k_cy_cell<KIND_LH, LP><<<nc, CY_CELL_BS, 0, h->st>>>(K, h->U, h->X, h->U0, h->T, h->FXH, h->FYH, sc);
        k_cy_bface<KIND_LH><<<nf, 128, 0, h->st>>>(K, h->FXH, h->FYH, h->EzV, h->BR, h->BRX, h->BR0, h->BZ, h->BZX,
                                                    h->BZ0, sc);
        break;
      case KIND_S1:
        k_cy_cell<KIND_S1, LP><<<nc, CY_CELL_BS, 0, h->st>>>(K, h->U, h->X, h->U0, h->T, h->FXH, h->FYH, sc);
        k_cy_bface<KIND_S1><<<nf, 128, 0, h->st>>>(K, h->FXH, h->FYH, h->EzV, h->BR, h->BRX, h->BR0, h->BZ, h->BZX,
                                                    h->BZ0, sc);
        break;
      case KIND_S2:
        k_cy_cell<KIND_S2, LP><<<nc, CY_CELL_BS, 0, h->st>>>(K, h->U, h->X, h->U0, h->T, h->FXH, h->FYH, sc);
        k_cy_bface<KIND_S2><<<nf, 128, 0, h->st>>>(K, h->FXH, h->FYH, h->EzV, h->BR, h->BRX, h->BR0, h->BZ, h->BZX,
                                                    h->BZ0, sc);
        break;
      default:
        k_cy_cell<KIND_S3, LP><<<nc, CY_CELL_BS, 0, h->st>>>(K, h->U, h->X, h->U0, h->T, h->FXH, h->FYH, sc);
        k_cy_bface<KIND_S3><<<nf, 128, 0, h->st>>>(K, h->FXH, h->FYH, h->EzV, h->BR, h->BRX, h->BR0, h->BZ, h->BZX,
                                                    h->BZ0, sc);
        break;
    }
  });
}

int launch_lh(GdfCyHandle* h, int kind, const ScalC* sc) {
  switch (h->K.lphi) {
    case 1: return launch_lh_lp<1>(h, kind, sc);
    case 2: return launch_lh_lp<2>(h, kind, sc);
    case 4: return launch_lh_lp<4>(h, kind, sc);
    default: return launch_lh_lp<8>(h, kind, sc);
  }
}

// TVB_Limiter_P2 + div_free_Balsara of (U, BR, BZ) in place
int launch_limit(GdfCyHandle* h, const ScalC* sc, int32_t* flags) {
  const KC& K = h->K;
  const long long ncell = (long long)K.nx * K.ny * K.nph;
  int rc = launch_set_bc(h, sc);
  if (!rc) rc = run(h, [&] { k_cy_bproj<<<nblk(K.ncp, 128), 128, 0, h->st>>>(K, h->U, h->BP, sc); });
  if (!rc) rc = run(h, [&] { k_cy_tvb<<<nblk(ncell, 64), 64, 0, h->st>>>(K, h->U, h->BP, flags, sc); });
  if (!rc) rc = launch_set_bc(h, sc);
  if (!rc) rc = run(h, [&] { k_cy_faceb<<<nblk(K.nxf + K.nyf, 128), 128, 0, h->st>>>(K, h->U, h->BR, h->BZ, sc); });
  if (!rc)
    rc = run(h, [&] {
      const unsigned nb = nblk(ncell, 128);
      switch (K.lphi) {
        case 1: k_cy_divfree<1><<<nb, 128, 0, h->st>>>(K, h->U, h->BR, h->BZ, sc); break;
        case 2: k_cy_divfree<2><<<nb, 128, 0, h->st>>>(K, h->U, h->BR, h->BZ, sc); break;
        case 4: k_cy_divfree<4><<<nb, 128, 0, h->st>>>(K, h->U, h->BR, h->BZ, sc); break;
        default: k_cy_divfree<8><<<nb, 128, 0, h->st>>>(K, h->U, h->BR, h->BZ, sc); break;
      }
    });
  return rc;
}

int launch_dt(GdfCyHandle* h, int step) {
  const KC& K = h->K;
  int rc = run(h, [&] { k_cy_dt_partial<<<h->dt_blocks, DT_BS, 0, h->st>>>(K, h->U, h->part, h->sc, step); });
  if (!rc) rc = run(h, [&] { k_cy_dt_final<<<1, DT_BS, 0, h->st>>>(K, h->part, h->dt_blocks, h->sc, step); });
  return rc;
}

// one RK3 step (RK3.f90:42-133)
int enqueue_step(GdfCyHandle* h) {
  int rc = launch_dt(h, 1);
  for (int s = 1; s <= 3 && !rc; ++s) {
    rc = launch_lh(h, s == 1 ? KIND_S1 : s == 2 ? KIND_S2 : KIND_S3, h->sc);
    if (!rc) rc = launch_limit(h, h->sc, nullptr);
  }
  return rc;
}

int ensure_graph(GdfCyHandle* h) {
  if (h->graph) return GDF_OK;
  cudaGraph_t g = nullptr;
  const int64_t before = h->launches;
  CKC(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
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

int sync_scal(GdfCyHandle* h) {
  CKC(cudaMemcpyAsync(h->sc_host, h->sc, sizeof(ScalC), cudaMemcpyDeviceToHost, h->st));
  CKC(cudaStreamSynchronize(h->st));
  return GDF_OK;
}

int push_scal(GdfCyHandle* h) {
  CKC(cudaMemcpyAsync(h->sc, h->sc_host, sizeof(ScalC), cudaMemcpyHostToDevice, h->st));
  CKC(cudaStreamSynchronize(h->st));
  return GDF_OK;
}

size_t cell_plane_bytes(const KC& K) { return (size_t)K.ncp * sizeof(double); }
size_t br_bytes(const KC& K) { return (size_t)K.nxf * 3 * sizeof(double); }
size_t bz_bytes(const KC& K) { return (size_t)K.nyf * 3 * sizeof(double); }

// host uh (10 modes x 8 variables of full planes) -> the 54 live slots; the
// slots the method keeps at zero must be zero
int upload_cells(GdfCyHandle* h, const double* uh, double* D) {
  const size_t pl = (size_t)h->K.ncp;
  for (int n = 0; n < NE; ++n)
    for (int d = 0; d < NPC; ++d) {
      const double* src = uh + pl * (d + (size_t)NPC * n);
      const int s = slotc(n, d);
      if (s < 0) {
        for (size_t q = 0; q < pl; ++q)
          if (src[q] != 0.0)
            return fail(GDF_ERR_ARG, "uh slot (d=" + std::to_string(d + 1) + ", n=" + std::to_string(n + 1) +
                                         ") must be zero: the cylindrical method never fills it");
        continue;
      }
      CKC(cudaMemcpyAsync(D + pl * s, src, pl * sizeof(double), cudaMemcpyHostToDevice, h->st));
    }
  CKC(cudaStreamSynchronize(h->st));
  return GDF_OK;
}

int download_cells(GdfCyHandle* h, const double* D, double* uh) {
  const size_t pl = (size_t)h->K.ncp;
  for (int n = 0; n < NE; ++n)
    for (int d = 0; d < NPC; ++d) {
      double* dst = uh + pl * (d + (size_t)NPC * n);
      const int s = slotc(n, d);
      if (s < 0) {
        std::memset(dst, 0, pl * sizeof(double));
        continue;
      }
      CKC(cudaMemcpyAsync(dst, D + pl * s, pl * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    }
  CKC(cudaStreamSynchronize(h->st));
  return GDF_OK;
}

int check_status(GdfCyHandle* h) {
  if (h->sc_host->status & 1)
    return fail(GDF_ERR_NUMERIC, "non-positive density, non-finite energy or non-positive dt at t = " +
                                     std::to_string(h->sc_host->t));
  return GDF_OK;
}

}  // namespace

extern "C" {

int gdf_cy_create(const GdfCyConfig* cfg, GdfCyHandle** out) {
  if (!out) return fail(GDF_ERR_ARG, "null handle pointer");
  *out = nullptr;
  int rc = check_config(cfg);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(GDF_ERR_CUDA, "no CUDA device available");
  }
  GdfCyHandle* h = new GdfCyHandle();
  h->cfg = *cfg;
  build_kc(*cfg, h->K);
  const KC& K = h->K;
  const size_t ub = cell_plane_bytes(K) * NSC;
  const long long ncell = (long long)K.nx * K.ny * K.nph;
  h->dt_blocks = (int)nblk(ncell, DT_BS);
  auto alloc = [&](double** p, size_t bytes) -> bool {
    if (cudaMalloc((void**)p, bytes) != cudaSuccess) return false;
    return cudaMemset(*p, 0, bytes) == cudaSuccess;
  };
  bool ok = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && alloc(&h->U, ub) && alloc(&h->X, ub) && alloc(&h->U0, ub) && alloc(&h->T, ub);
  ok = ok && alloc(&h->BP, cell_plane_bytes(K) * 2 * NQC);
  ok = ok && alloc(&h->BR, br_bytes(K)) && alloc(&h->BRX, br_bytes(K)) && alloc(&h->BR0, br_bytes(K));
  ok = ok && alloc(&h->BZ, bz_bytes(K)) && alloc(&h->BZX, bz_bytes(K)) && alloc(&h->BZ0, bz_bytes(K));
  ok = ok && alloc(&h->FXH, (size_t)K.nxf * NG * NFQ * sizeof(double)) &&
       alloc(&h->FYH, (size_t)K.nyf * NG * NFQ * sizeof(double));
  ok = ok && alloc(&h->EzV, (size_t)K.nvx * sizeof(double));
  ok = ok && alloc(&h->part, (size_t)h->dt_blocks * 2 * sizeof(double));
  ok = ok && alloc(&h->diag, (size_t)ncell * 3 * sizeof(double));
  ok = ok && cudaMalloc((void**)&h->sc, sizeof(ScalC)) == cudaSuccess;
  ok = ok && cudaMallocHost((void**)&h->sc_host, sizeof(ScalC)) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    gdf_cy_destroy(h);
    return fail(GDF_ERR_NOMEM, "device allocation failed for a " + std::to_string(cfg->nr) + "x" +
                                   std::to_string(cfg->nz) + "x" + std::to_string(2 * cfg->lphi) + " grid");
  }
  std::memset(h->sc_host, 0, sizeof(ScalC));
  h->sc_host->tend = 1e300;
  h->sc_host->active = 1;
  if (push_scal(h)) {
    gdf_cy_destroy(h);
    return GDF_ERR_CUDA;
  }
  *out = h;
  return GDF_OK;
}

int gdf_cy_destroy(GdfCyHandle* h) {
  if (!h) return GDF_OK;
  if (h->graph) cudaGraphExecDestroy(h->graph);
  for (double* p : {h->U, h->X, h->U0, h->T, h->BP, h->BR, h->BRX, h->BR0, h->BZ, h->BZX, h->BZ0, h->FXH, h->FYH,
                    h->EzV, h->part, h->diag})
    if (p) cudaFree(p);
  if (h->sc) cudaFree(h->sc);
  if (h->sc_host) cudaFreeHost(h->sc_host);
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
  return GDF_OK;
}

int gdf_cy_upload(GdfCyHandle* h, const double* uh, const double* br, const double* bz) {
  if (!h || !uh || !br || !bz) return fail(GDF_ERR_ARG, "null argument");
  int rc = upload_cells(h, uh, h->U);
  if (rc) return rc;
  CKC(cudaMemcpyAsync(h->BR, br, br_bytes(h->K), cudaMemcpyHostToDevice, h->st));
  CKC(cudaMemcpyAsync(h->BZ, bz, bz_bytes(h->K), cudaMemcpyHostToDevice, h->st));
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

int gdf_cy_download(GdfCyHandle* h, double* uh, double* br, double* bz) {
  if (!h || !uh || !br || !bz) return fail(GDF_ERR_ARG, "null argument");
  if (!h->uploaded) return fail(GDF_ERR_STATE, "no state uploaded");
  int rc = download_cells(h, h->U, uh);
  if (rc) return rc;
  CKC(cudaMemcpyAsync(br, h->BR, br_bytes(h->K), cudaMemcpyDeviceToHost, h->st));
  CKC(cudaMemcpyAsync(bz, h->BZ, bz_bytes(h->K), cudaMemcpyDeviceToHost, h->st));
  CKC(cudaStreamSynchronize(h->st));
  return GDF_OK;
}

int gdf_cy_set_time(GdfCyHandle* h, double t) {
  if (!h) return fail(GDF_ERR_ARG, "null handle");
  int rc = sync_scal(h);
  if (rc) return rc;
  h->sc_host->t = t;
  return push_scal(h);
}

int gdf_cy_get_time(GdfCyHandle* h, double* t) {
  if (!h || !t) return fail(GDF_ERR_ARG, "null argument");
  int rc = sync_scal(h);
  if (rc) return rc;
  *t = h->sc_host->t;
  return GDF_OK;
}

int gdf_cy_prepare(GdfCyHandle* h) {
  if (!h) return fail(GDF_ERR_ARG, "null handle");
  if (!h->uploaded) return fail(GDF_ERR_STATE, "no state uploaded");
  int rc = launch_limit(h, nullptr, nullptr);
  if (rc) return rc;
  CKC(cudaStreamSynchronize(h->st));
  return GDF_OK;
}

int gdf_cy_step(GdfCyHandle* h, double tend, double* t, double* dt) {
  if (!h) return fail(GDF_ERR_ARG, "null handle");
  if (!h->uploaded) return fail(GDF_ERR_STATE, "no state uploaded");
  int rc = sync_scal(h);
  if (rc) return rc;
  h->sc_host->tend = tend;
  h->sc_host->active = 1;
  if ((rc = push_scal(h))) return rc;
  if ((rc = ensure_graph(h))) return rc;
  CKC(cudaGraphLaunch(h->graph, h->st));
  h->launches += h->step_launches;
  if ((rc = sync_scal(h))) return rc;
  if (t) *t = h->sc_host->t;
  if (dt) *dt = h->sc_host->dt;
  return check_status(h);
}

static int advance_impl(GdfCyHandle* h, double tend, int32_t max_steps, double* t, int32_t* steps, double* ms,
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
    CKC(cudaEventCreate(&e0));
    CKC(cudaEventCreate(&e1));
    CKC(cudaEventRecord(e0, h->st));
  }
  int done = 0;
  const int chunk = exact_count ? std::max(max_steps, 1) : 16;
  while (done < max_steps) {
    const int n = std::min(chunk, max_steps - done);
    for (int k = 0; k < n; ++k) CKC(cudaGraphLaunch(h->graph, h->st));
    h->launches += (int64_t)n * h->step_launches;
    done += n;
    if (!exact_count) {
      if ((rc = sync_scal(h))) return rc;
      if (!h->sc_host->active || !(h->sc_host->t < tend) || (h->sc_host->status & 1)) break;
    }
  }
  if (ms) {
    CKC(cudaEventRecord(e1, h->st));
    CKC(cudaEventSynchronize(e1));
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

int gdf_cy_advance(GdfCyHandle* h, double tend, int32_t max_steps, double* t, int32_t* steps) {
  return advance_impl(h, tend, max_steps, t, steps, nullptr, false);
}

int gdf_cy_advance_timed(GdfCyHandle* h, double tend, int32_t steps, double* t, int32_t* steps_taken, double* ms) {
  if (!ms) return fail(GDF_ERR_ARG, "null ms");
  return advance_impl(h, tend, steps, t, steps_taken, ms, true);
}

int gdf_cy_lh(GdfCyHandle* h, const double* uh, const double* br, const double* bz, double t_rk, double* du,
              double* dbr, double* dbz) {
  if (!h || !uh || !br || !bz || !du || !dbr || !dbz) return fail(GDF_ERR_ARG, "null argument");
  const KC& K = h->K;
  int rc = upload_cells(h, uh, h->U);
  if (rc) return rc;
  CKC(cudaMemcpyAsync(h->BR, br, br_bytes(K), cudaMemcpyHostToDevice, h->st));
  CKC(cudaMemcpyAsync(h->BZ, bz, bz_bytes(K), cudaMemcpyHostToDevice, h->st));
  CKC(cudaMemsetAsync(h->T, 0, cell_plane_bytes(K) * NSC, h->st));
  if ((rc = sync_scal(h))) return rc;
  h->sc_host->trk[0] = t_rk;
  h->sc_host->active = 1;
  if ((rc = push_scal(h))) return rc;
  if ((rc = launch_lh(h, KIND_LH, h->sc))) return rc;
  if ((rc = download_cells(h, h->T, du))) return rc;
  CKC(cudaMemcpyAsync(dbr, h->BRX, br_bytes(K), cudaMemcpyDeviceToHost, h->st));
  CKC(cudaMemcpyAsync(dbz, h->BZX, bz_bytes(K), cudaMemcpyDeviceToHost, h->st));
  CKC(cudaStreamSynchronize(h->st));
  h->uploaded = 1;
  return GDF_OK;
}

int gdf_cy_limit(GdfCyHandle* h, double* uh, double* br, double* bz) {
  if (!h || !uh || !br || !bz) return fail(GDF_ERR_ARG, "null argument");
  const KC& K = h->K;
  int rc = upload_cells(h, uh, h->U);
  if (rc) return rc;
  CKC(cudaMemcpyAsync(h->BR, br, br_bytes(K), cudaMemcpyHostToDevice, h->st));
  CKC(cudaMemcpyAsync(h->BZ, bz, bz_bytes(K), cudaMemcpyHostToDevice, h->st));
  if ((rc = launch_limit(h, nullptr, nullptr))) return rc;
  if ((rc = download_cells(h, h->U, uh))) return rc;
  CKC(cudaMemcpyAsync(br, h->BR, br_bytes(K), cudaMemcpyDeviceToHost, h->st));
  CKC(cudaMemcpyAsync(bz, h->BZ, bz_bytes(K), cudaMemcpyDeviceToHost, h->st));
  CKC(cudaStreamSynchronize(h->st));
  h->uploaded = 1;
  return GDF_OK;
}

int gdf_cy_dt(GdfCyHandle* h, const double* uh, double* dt) {
  if (!h || !uh || !dt) return fail(GDF_ERR_ARG, "null argument");
  int rc = upload_cells(h, uh, h->U);
  if (rc) return rc;
  if ((rc = launch_dt(h, 0))) return rc;
  if ((rc = sync_scal(h))) return rc;
  *dt = h->sc_host->dt;
  return GDF_OK;
}

int gdf_cy_diagnostics(GdfCyHandle* h, double* umax, double* totaldiv, double* pmin) {
  if (!h) return fail(GDF_ERR_ARG, "null handle");
  if (!h->uploaded) return fail(GDF_ERR_STATE, "no state uploaded");
  const KC& K = h->K;
  const long long n = (long long)K.nx * K.ny * K.nph;
  int rc = run(h, [&] {
    switch (K.lphi) {
      case 1: k_cy_diag<1><<<nblk(n, 128), 128, 0, h->st>>>(K, h->U, h->diag); break;
      case 2: k_cy_diag<2><<<nblk(n, 128), 128, 0, h->st>>>(K, h->U, h->diag); break;
      case 4: k_cy_diag<4><<<nblk(n, 128), 128, 0, h->st>>>(K, h->U, h->diag); break;
      default: k_cy_diag<8><<<nblk(n, 128), 128, 0, h->st>>>(K, h->U, h->diag); break;
    }
  });
  if (rc) return rc;
  std::vector<double> v((size_t)n * 3);
  CKC(cudaMemcpyAsync(v.data(), h->diag, v.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CKC(cudaStreamSynchronize(h->st));
  // item q = kk + nph*((i-1) + nr*(j-1)); the reference's loops: j outer, i inner
  double um = 0, td = 0, pm = 1000000;
  for (long long q = 0; q < n; ++q) {
    if (v[q] > um) um = v[q];
    if (v[(size_t)n + q] < pm) pm = v[(size_t)n + q];
    td = td + v[(size_t)2 * n + q];
  }
  if (umax) *umax = um;
  if (totaldiv) *totaldiv = std::sqrt(0.25 * td / ((double)K.nx * K.ny * K.nph));
  if (pmin) *pmin = pm;
  return GDF_OK;
}

int gdf_cy_kernel_launches(GdfCyHandle* h, int64_t* n) {
  if (!h || !n) return fail(GDF_ERR_ARG, "null argument");
  *n = h->launches;
  return GDF_OK;
}

}  // extern "C"
