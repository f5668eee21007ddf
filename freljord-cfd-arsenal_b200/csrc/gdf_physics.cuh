// gdf_physics.cuh -- pointwise ideal-MHD physics of the GDF P2 step, FP64.
//
// Header-only, __host__ __device__: the kernels in gdf_kernels.cu use it on
// sm_100a, and the host build of tests/native/devcheck.cpp compiles the same
// code to compare it value-for-value with the CPU oracle.
//
// Every function keeps the reference's expression order (left-to-right
// evaluation of + - * /, x**2 as x*x, x**0.5 as sqrt, MAX/MIN as sequential
// NaN-skipping comparisons, SIGN as copysign) so that a build without FMA
// contraction reproduces the reference arithmetic. Functions are specialised
// by direction where the reference passes constant normals; terms that are
// products with those constant zeros are dropped, which leaves every
// nonzero value unchanged (x + (+-0) == x).
#pragma once

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define GDF_HD __host__ __device__ __forceinline__
#else
#define GDF_HD inline
#endif

namespace gdf {

constexpr int NG = 5;   // Gauss points per direction (com.txt NumGLP)
constexpr int NP = 10;  // modal slots per variable (dimPk, k = 2)
constexpr int NE = 8;   // conserved variables (NumEq)

// Modes carried by each variable (1-based mode numbers of the reference
// minus one): vars 0-4 and 7 carry modes 0-5; Bx (var 5) 0-6 and 8; By
// (var 6) 0-5, 7 and 9 (Lh.f90:59 mode mask, div_free_Balsara.f90:63-79).
GDF_HD bool live_mode(int n, int d) {
  return d <= 5 || (n == 5 && (d == 6 || d == 8)) || (n == 6 && (d == 7 || d == 9));
}

GDF_HD double sq(double x) { return x * x; }
// gfortran MAX/MIN: m = a; if (b > m .or. isnan(m)) m = b
GDF_HD double fmax2(double a, double b) { return (b > a || a != a) ? b : a; }
GDF_HD double fmin2(double a, double b) { return (b < a || a != a) ? b : a; }
GDF_HD double sgn1(double b) { return copysign(1.0, b); }

// x / y and sqrt(x) with their IEEE results. On the device a zero x is
// answered directly (the signed zero the operation would return), because
// the hardware sequences send a zero operand down their slow path; a 2-D run
// (w = Bz = 0 everywhere, u = v = 0 in quiet regions) feeds the face solvers
// a zero numerator in a large share of their divisions. Every other operand
// goes through the correctly rounded operation itself.
#ifndef GDF_DV_FAST
#define GDF_DV_FAST 1
#endif
GDF_HD double dv(double x, double y) {
#if defined(__CUDA_ARCH__) && GDF_DV_FAST
  if (x == 0.0 && y == y && y != 0.0)
    return __longlong_as_double((long long)(((unsigned long long)__double_as_longlong(x) ^
                                             (unsigned long long)__double_as_longlong(y)) & 0x8000000000000000ull));
#endif
  return x / y;
}
GDF_HD double sqrt0(double x) {
#if defined(__CUDA_ARCH__) && GDF_DV_FAST
  if (x == 0.0) return x;
#endif
  return sqrt(x);
}
// The face solvers take the shortcut (ZF); elsewhere the plain operation
// measured faster (the vertex solver and the limiter's eigenvectors meet
// few exact zeros and their code grows with the extra test).
template <bool ZF>
GDF_HD double dvz(double x, double y) {
  return ZF ? dv(x, y) : x / y;
}
template <bool ZF>
GDF_HD double sqz(double x) {
  return ZF ? sqrt0(x) : sqrt(x);
}

// Run-time physics constants shared by every kernel.
struct Phys {
  double gamma, gamma1;   // com.txt:7-8
  double gflux;           // MHD_flux.f90:7, eigenmatrix.f90:19
  double hlld_eps;        // HLLD_Flux.f90:126
  int flux;               // 1 LF, 2 HLL, 3 HLLC, 4 HLLD
  int kml_w;              // Lh.f90:126 w-term in KML
  int eig_p_typo;         // eigenmatrix.f90:21 DF form
  int eig_identity;       // eigenmatrix.f90:397-404
};

// ------------------------------------------------------------- state -----
// A conservative state with the primitives every routine of the reference
// derives from it (u = rhou/rho, ...; p with the com.txt gamma). Computing
// them once and sharing them gives the same values as recomputing them in
// each routine.
struct Side {
  double U[NE];
  double rho, u, v, w, E, B1, B2, B3, BB, p;
};

template <bool ZF = false>
GDF_HD void make_side(const Phys& P, const double* U, Side& s) {
#pragma unroll
  for (int n = 0; n < NE; ++n) s.U[n] = U[n];
  s.rho = U[0];
  s.u = dvz<ZF>(U[1], s.rho);
  s.v = dvz<ZF>(U[2], s.rho);
  s.w = dvz<ZF>(U[3], s.rho);
  s.E = U[4];
  s.B1 = U[5];
  s.B2 = U[6];
  s.B3 = U[7];
  s.BB = sq(s.B1) + sq(s.B2) + sq(s.B3);
  s.p = P.gamma1 * (s.E - 0.5 * s.rho * (sq(s.u) + sq(s.v) + sq(s.w)) - 0.5 * s.BB);
}

// Lh.f90:88-135 flux in x of a state (FR/FL arrays)
GDF_HD void side_flux_x(const Side& s, double* F, bool drop_w_in_k) {
  const double S = s.p + 0.5 * s.BB;
  const double T = s.E + S;
  const double K = drop_w_in_k ? (s.u * s.B1 + s.v * s.B2) : (s.u * s.B1 + s.v * s.B2 + s.w * s.B3);
  F[0] = s.U[1];
  F[1] = s.rho * sq(s.u) + S - sq(s.B1);
  F[2] = s.rho * s.u * s.v - s.B1 * s.B2;
  F[3] = s.rho * s.u * s.w - s.B1 * s.B3;
  F[4] = T * s.u - K * s.B1;
  F[5] = 0.0;
  F[6] = s.u * s.B2 - s.v * s.B1;
  F[7] = s.u * s.B3 - s.w * s.B1;
}

// Lh.f90:155-202 flux in y (FU/FD); the D side takes its pressure with
// +u^2+v^2-w^2 (Lh.f90:189)
GDF_HD void side_flux_y(const Phys& P, const Side& s, double* F, bool d_side) {
  const double p = d_side ? P.gamma1 * (s.E - 0.5 * s.rho * (sq(s.u) + sq(s.v) - sq(s.w)) - 0.5 * s.BB) : s.p;
  const double S = p + 0.5 * s.BB;
  const double T = s.E + S;
  const double K = s.u * s.B1 + s.v * s.B2 + s.w * s.B3;
  F[0] = s.U[2];
  F[1] = s.rho * s.u * s.v - s.B1 * s.B2;
  F[2] = s.rho * sq(s.v) + S - sq(s.B2);
  F[3] = s.rho * s.v * s.w - s.B2 * s.B3;
  F[4] = T * s.v - K * s.B2;
  F[5] = s.v * s.B1 - s.u * s.B2;
  F[6] = 0.0;
  F[7] = s.v * s.B3 - s.w * s.B2;
}

// MHD_flux.f90 (hard-coded gamma) from a state's primitives
GDF_HD void side_flux_hard(const Phys& P, const Side& s, double* Fx, double* Fy) {
  const double g1 = P.gflux - 1;
  const double p = g1 * (s.E - 0.5 * s.rho * (sq(s.u) + sq(s.v) + sq(s.w)) - 0.5 * s.BB);
  const double S = p + 0.5 * s.BB;
  const double T = s.E + S;
  const double K = s.u * s.B1 + s.v * s.B2 + s.w * s.B3;
  Fx[0] = s.U[1];
  Fx[1] = s.rho * sq(s.u) + S - sq(s.B1);
  Fx[2] = s.rho * s.u * s.v - s.B1 * s.B2;
  Fx[3] = s.rho * s.u * s.w - s.B1 * s.B3;
  Fx[4] = T * s.u - K * s.B1;
  Fx[5] = 0.0;
  Fx[6] = s.u * s.B2 - s.v * s.B1;
  Fx[7] = s.u * s.B3 - s.w * s.B1;
  Fy[0] = s.U[2];
  Fy[1] = s.rho * s.u * s.v - s.B1 * s.B2;
  Fy[2] = s.rho * sq(s.v) + S - sq(s.B2);
  Fy[3] = s.rho * s.w * s.v - s.B3 * s.B2;
  Fy[4] = T * s.v - K * s.B2;
  Fy[5] = s.v * s.B1 - s.u * s.B2;
  Fy[6] = 0.0;
  Fy[7] = s.v * s.B3 - s.w * s.B2;
}

// eigenvalueMm.f90 from a state's primitives (normal x: dir 0, y: dir 1)
template <bool ZF = false>
GDF_HD void side_speeds(const Phys& P, const Side& s, int dir, double& amax, double& amin) {
  const double Bn = dir == 0 ? s.B1 : s.B2;
  const double un = dir == 0 ? s.u : s.v;
  const double c = sqz<ZF>(fabs(dvz<ZF>(P.gamma * s.p, s.rho)));
  const double c2 = sq(c);
  const double br = dvz<ZF>(s.BB, s.rho);
  const double X = c2 + br;
  const double cf = sqz<ZF>(fabs(0.5 * (c2 + br + sqz<ZF>(sq(X) - dvz<ZF>(4 * c2 * sq(Bn), s.rho)))));
  amax = un + cf;
  amin = un - cf;
}

// -------------------------------------------------------- wave speeds ------
// eigenvalueMm.f90:1-25 for the normal (1,0) (dir 0) or (0,1) (dir 1).
GDF_HD void fast_speeds(const Phys& P, const double* U, int dir, double& amax, double& amin) {
  const double rho = U[0];
  const double u = dvz<false>(U[1], rho), v = dvz<false>(U[2], rho), w = dvz<false>(U[3], rho);
  const double B1 = U[5], B2 = U[6], B3 = U[7];
  const double BP = sq(B1) + sq(B2) + sq(B3);
  const double Bn = dir == 0 ? B1 : B2;
  const double un = dir == 0 ? u : v;
  const double p = P.gamma1 * (U[4] - 0.5 * rho * (sq(u) + sq(v) + sq(w)) - 0.5 * BP);
  const double c = sqz<false>(fabs(dvz<false>(P.gamma * p, rho)));
  const double c2 = sq(c);
  const double X = c2 + dvz<false>(BP, rho);
  const double cf = sqz<false>(fabs(0.5 * (c2 + dvz<false>(BP, rho) + sqz<false>(sq(X) - dvz<false>(4 * c2 * sq(Bn), rho)))));
  amax = un + cf;
  amin = un - cf;
}

// ------------------------------------------------------ 1-D Riemann --------
// HLLC_Flux.f90:9-106 and HLLD_Flux.f90:14-189 share the first stage.
// dir 0 = normal x (reference direction 1), 1 = normal y (direction 2).
// Fh gets the flux, Ust the star state (Ustar of the reference).
template <bool HLLD, bool ZF = false>
GDF_HD void hllcd_flux(const Phys& P, const Side& R, const Side& L, const double* FR, const double* FL, double SR,
                       double SL, int dir, double* Fh, double* Ust) {
  if (SR < 0) {
#pragma unroll
    for (int n = 0; n < NE; ++n) { Fh[n] = FR[n]; Ust[n] = R.U[n]; }
    return;
  }
  if (SL > 0) {
#pragma unroll
    for (int n = 0; n < NE; ++n) { Fh[n] = FL[n]; Ust[n] = L.U[n]; }
    return;
  }
  const double* UR1 = R.U;
  const double* UL1 = L.U;
  double Us[NE];
#pragma unroll
  for (int n = 0; n < NE; ++n) Us[n] = dvz<ZF>(SR * UR1[n] - SL * UL1[n] + FL[n] - FR[n], SR - SL);
  const double rhoR = R.rho, u1R = R.u, u2R = R.v, u3R = R.w, ER = R.E;
  const double B1R = R.B1, B2R = R.B2, B3R = R.B3;
  const double rhoL = L.rho, u1L = L.u, u2L = L.v, u3L = L.w, EL = L.E;
  const double B1L = L.B1, B2L = L.B2, B3L = L.B3;
  const double Sstar = dvz<ZF>(dir == 0 ? Us[1] : Us[2], Us[0]);
  const double uRbot = dir == 0 ? u1R : u2R, uLbot = dir == 0 ? u1L : u2L;
  const double BRbot = dir == 0 ? B1R : B2R, BLbot = dir == 0 ? B1L : B2L;
  const double Bsb = dir == 0 ? Us[5] : Us[6];
  const double dR = SR - uRbot, dL = SL - uLbot;      // (SR - uRbot), (SL - uLbot)
  const double eR = SR - Sstar, eL = SL - Sstar;      // (SR - Sstar), (SL - Sstar)
  const double rhoRs = dvz<ZF>(rhoR * dR, eR);
  const double rhoLs = dvz<ZF>(rhoL * dL, eL);
  const double PtotR = P.gamma1 * (ER - 0.5 * rhoR * (sq(u1R) + sq(u2R) + sq(u3R)));
  const double PtotL = P.gamma1 * (EL - 0.5 * rhoL * (sq(u1L) + sq(u2L) + sq(u3L)));
  const double PtotRs = PtotR + rhoR * dR * (Sstar - uRbot) + sq(Bsb) - sq(BRbot);
  const double PtotLs = PtotL + rhoL * dL * (Sstar - uLbot) + sq(Bsb) - sq(BLbot);
  double B1Rs, B1Ls, B2Rs, B2Ls, B3Rs, B3Ls;
  double SRs = 0, SLs = 0;
  if (HLLD) {
    SRs = Sstar + sqz<ZF>(dvz<ZF>(sq(Bsb), rhoRs));
    SLs = Sstar - sqz<ZF>(dvz<ZF>(sq(Bsb), rhoLs));
    const double AR = rhoR * sq(dR) - Bsb * BRbot;
    const double AL = rhoL * sq(dL) - Bsb * BLbot;
    const double CR = rhoR * dR * (BRbot - Bsb);
    const double CL = rhoL * dL * (BLbot - Bsb);
    const double DR = rhoR * dR * eR - sq(Bsb) + 1e-15;
    const double DL = rhoL * dL * eL - sq(Bsb) + 1e-15;
    if (dir == 0) {
      B1Rs = Bsb; B1Ls = Bsb;
      B2Rs = dvz<ZF>(AR * B2R + CR * u2R, DR);
      B2Ls = dvz<ZF>(AL * B2L + CL * u2L, DL);
    } else {
      B1Rs = dvz<ZF>(AR * B1R + CR * u1R, DR);
      B1Ls = dvz<ZF>(AL * B1L + CL * u1L, DL);
      B2Rs = Bsb; B2Ls = Bsb;
    }
    B3Rs = dvz<ZF>(AR * B3R + CR * u3R, DR);
    B3Ls = dvz<ZF>(AL * B3L + CL * u3L, DL);
  } else {
    B1Rs = Us[5]; B1Ls = Us[5]; B2Rs = Us[6]; B2Ls = Us[6]; B3Rs = Us[7]; B3Ls = Us[7];
  }
  double URs[NE], ULs[NE];
  if (dir == 0) {
    URs[1] = dvz<ZF>(UR1[1] * dR + PtotRs - PtotR + BRbot * B1R - Bsb * B1Rs, eR);
    URs[2] = dvz<ZF>(UR1[2] * dR + BRbot * B2R - Bsb * B2Rs, eR);
    ULs[1] = dvz<ZF>(UL1[1] * dL + PtotLs - PtotL + BLbot * B1L - Bsb * B1Ls, eL);
    ULs[2] = dvz<ZF>(UL1[2] * dL + BLbot * B2L - Bsb * B2Ls, eL);
  } else {
    URs[1] = dvz<ZF>(UR1[1] * dR + BRbot * B1R - Bsb * B1Rs, eR);
    URs[2] = dvz<ZF>(UR1[2] * dR + PtotRs - PtotR + BRbot * B2R - Bsb * B2Rs, eR);
    ULs[1] = dvz<ZF>(UL1[1] * dL + BLbot * B1L - Bsb * B1Ls, eL);
    ULs[2] = dvz<ZF>(UL1[2] * dL + PtotLs - PtotL + BLbot * B2L - Bsb * B2Ls, eL);
  }
  URs[3] = dvz<ZF>(UR1[3] * dR + BRbot * B3R - Bsb * B3Rs, eR);
  ULs[3] = dvz<ZF>(UL1[3] * dL + BLbot * B3L - Bsb * B3Ls, eL);
  const double u1Rs = dvz<ZF>(URs[1], rhoRs), u2Rs = dvz<ZF>(URs[2], rhoRs), u3Rs = dvz<ZF>(URs[3], rhoRs);
  const double u1Ls = dvz<ZF>(ULs[1], rhoLs), u2Ls = dvz<ZF>(ULs[2], rhoLs), u3Ls = dvz<ZF>(ULs[3], rhoLs);
  const double ERs = dvz<ZF>(dR * ER - PtotR * uRbot + PtotRs * Sstar + BRbot * (u1R * B1R + u2R * B2R + u3R * B3R) -
                            Bsb * (u1Rs * B1Rs + u2Rs * B2Rs + u3Rs * B3Rs), eR);
  const double ELs = dvz<ZF>(dL * EL - PtotL * uLbot + PtotLs * Sstar + BLbot * (u1L * B1L + u2L * B2L + u3L * B3L) -
                            Bsb * (u1Ls * B1Ls + u2Ls * B2Ls + u3Ls * B3Ls), eL);
  URs[0] = rhoRs; URs[4] = ERs;
  ULs[0] = rhoLs; ULs[4] = ELs;
#pragma unroll
  for (int n = 5; n < 8; ++n) { URs[n] = Us[n]; ULs[n] = Us[n]; }

  if (HLLD && (fabs(Bsb) > P.hlld_eps) && (SRs - SLs > P.hlld_eps)) {
    if (SLs > 0) {
#pragma unroll
      for (int n = 0; n < NE; ++n) { Fh[n] = FL[n] + SL * (ULs[n] - UL1[n]); Ust[n] = ULs[n]; }
    } else if (SRs < 0) {
#pragma unroll
      for (int n = 0; n < NE; ++n) { Fh[n] = FR[n] + SR * (URs[n] - UR1[n]); Ust[n] = URs[n]; }
    } else {
      // second stage (HLLD_Flux.f90:134-176)
      const double sL = sqrt(fabs(rhoLs)), sR = sqrt(fabs(rhoRs));
      const double sg = sgn1(Bsb);
      const double den = sL + sR;
      const double u1ss = dvz<ZF>(sL * u1Ls + sR * u1Rs + sg * (B1Rs - B1Ls), den);
      const double u2ss = dvz<ZF>(sL * u2Ls + sR * u2Rs + sg * (B2Rs - B2Ls), den);
      const double u3ss = dvz<ZF>(sL * u3Ls + sR * u3Rs + sg * (B3Rs - B3Ls), den);
      const double sLR = sqrt(fabs(rhoLs * rhoRs));
      const double B1ss = dvz<ZF>(sL * B1Ls + sR * B1Rs + sg * sLR * (u1Rs - u1Ls), den);
      const double B2ss = dvz<ZF>(sL * B2Ls + sR * B2Rs + sg * sLR * (u2Rs - u2Ls), den);
      const double B3ss = dvz<ZF>(sL * B3Ls + sR * B3Rs + sg * sLR * (u3Rs - u3Ls), den);
      if (Sstar > 0) {
        const double ELss = ELs - sL * (u1Ls * B1Ls + u2Ls * B2Ls + u3Ls * B3Ls - u1ss * B1ss - u2ss * B2ss -
                                        u3ss * B3ss) * sg;
        const double Uss[NE] = {rhoLs, rhoLs * u1ss, rhoLs * u2ss, rhoLs * u3ss, ELss, B1ss, B2ss, B3ss};
#pragma unroll
        for (int n = 0; n < NE; ++n) {
          const double FLm = FL[n] + SL * (ULs[n] - UL1[n]);
          Fh[n] = FLm + SLs * (Uss[n] - ULs[n]);
          Ust[n] = Uss[n];
        }
      } else {
        const double ERss = ERs + sR * (u1Rs * B1Rs + u2Rs * B2Rs + u3Rs * B3Rs - u1ss * B1ss - u2ss * B2ss -
                                        u3ss * B3ss) * sg;
        const double Uss[NE] = {rhoRs, rhoRs * u1ss, rhoRs * u2ss, rhoRs * u3ss, ERss, B1ss, B2ss, B3ss};
#pragma unroll
        for (int n = 0; n < NE; ++n) {
          const double FRm = FR[n] + SR * (URs[n] - UR1[n]);
          Fh[n] = FRm + SRs * (Uss[n] - URs[n]);
          Ust[n] = Uss[n];
        }
      }
    }
  } else {
    if (Sstar > 0) {
#pragma unroll
      for (int n = 0; n < NE; ++n) { Fh[n] = FL[n] + SL * (ULs[n] - UL1[n]); Ust[n] = ULs[n]; }
    } else {
#pragma unroll
      for (int n = 0; n < NE; ++n) { Fh[n] = FR[n] + SR * (URs[n] - UR1[n]); Ust[n] = URs[n]; }
    }
  }
}

// Riemann solve at one face point. uL = state on the -normal side (the
// reference's UL1), uR = +normal side (UR1); dir 0 = x, 1 = y. Writes the
// numerical flux Fh and returns the fluxes of both sides in fL / fR and the
// normal velocities of both sides in unL / unR (used by the face Ez).
template <bool ZF = false>
GDF_HD void face_flux_sides(const Phys& P, const Side& L, const Side& R, int dir, double* Fh, double* fL,
                            double* fR) {
  if (dir == 0) {
    side_flux_x(L, fL, false);
    side_flux_x(R, fR, !P.kml_w);
  } else {
    side_flux_y(P, L, fL, false);
    side_flux_y(P, R, fR, true);
  }
  double a1, a2, b1, b2;
  side_speeds<ZF>(P, L, dir, a1, a2);   // SRmax/SRmin of the reference (from UR(i) = left side)
  side_speeds<ZF>(P, R, dir, b1, b2);   // SLmax/SLmin (from UL(i+1) = right side)
  const double SR = fmax2(a1, b1);
  const double SL = fmin2(a2, b2);
  double Ust[NE];
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
      for (int n = 0; n < NE; ++n) Fh[n] = dvz<ZF>(SR * fL[n] - SL * fR[n] + sls * (R.U[n] - L.U[n]), den);
    }
  } else if (P.flux == 3) {
    hllcd_flux<false, ZF>(P, R, L, fR, fL, SR, SL, dir, Fh, Ust);
  } else {
    hllcd_flux<true, ZF>(P, R, L, fR, fL, SR, SL, dir, Fh, Ust);
  }
}

GDF_HD void face_flux(const Phys& P, const double* uL, const double* uR, int dir, double* Fh, double* fL,
                      double* fR) {
  Side L, R;
  make_side(P, uL, L);
  make_side(P, uR, R);
  face_flux_sides(P, L, R, dir, Fh, fL, fR);
}

// ------------------------------------------------------ 2-D vertex Ez -----
// HLL1.f90:1-15 restricted to what the vertex solver reads: component k of
// the HLL state and component m of the HLL flux.
GDF_HD void hll1_cm(const double* UR, const double* UL, const double* FR, const double* FL, double SR, double SL,
                    int k, int m, double& uk, double& fm) {
  if (SR < 0) {
    uk = UR[k]; fm = FR[m];
  } else if (SL > 0) {
    uk = UL[k]; fm = FL[m];
  } else {
    fm = dvz<false>(SR * FL[m] - SL * FR[m] + SL * SR * (UR[m] - UL[m]), SR - SL);
    uk = dvz<false>(SR * UR[k] - SL * UL[k] - (FR[k] - FL[k]), SR - SL);
  }
}

// LhEz.f90:50-69 for one vertex: states in the four quadrants around it
// (RU = upper right, ...). LF_Flux_2D.f90, HLL_Flux_2D.f90, HLLC/HLLD_Flux_2D.f90.
GDF_HD double vertex_ez(const Phys& P, const double* URU, const double* ULU, const double* URD, const double* ULD) {
  if (P.flux == 1) {
    const double ax = fmax2(fmax2(fmax2(fabs(URU[1] / URU[0]), fabs(ULU[1] / ULU[0])), fabs(URD[1] / URD[0])),
                            fabs(ULD[1] / ULD[0]));
    const double ay = fmax2(fmax2(fmax2(fabs(URU[2] / URU[0]), fabs(ULU[2] / ULU[0])), fabs(URD[2] / URD[0])),
                            fabs(ULD[2] / ULD[0]));
    // calculate_Ez.f90: Ez = u2*B1 - u1*B2
    const double EzRU = URU[2] / URU[0] * URU[5] - URU[1] / URU[0] * URU[6];
    const double EzLU = ULU[2] / ULU[0] * ULU[5] - ULU[1] / ULU[0] * ULU[6];
    const double EzRD = URD[2] / URD[0] * URD[5] - URD[1] / URD[0] * URD[6];
    const double EzLD = ULD[2] / ULD[0] * ULD[5] - ULD[1] / ULD[0] * ULD[6];
    return 0.25 * (EzRU + EzLU + EzRD + EzLD) - 0.25 * ay * (0.5 * (URU[5] + ULU[5]) - 0.5 * (URD[5] + ULD[5])) +
           0.25 * ax * (0.5 * (URU[6] + URD[6]) - 0.5 * (ULU[6] + ULD[6]));
  }
  Side sRU, sLU, sRD, sLD;
  make_side(P, URU, sRU);
  make_side(P, ULU, sLU);
  make_side(P, URD, sRD);
  make_side(P, ULD, sLD);
  double axRU, bxRU, ayRU, byRU, axLU, bxLU, ayLU, byLU, axRD, bxRD, ayRD, byRD, axLD, bxLD, ayLD, byLD;
  side_speeds(P, sRU, 0, axRU, bxRU);
  side_speeds(P, sRU, 1, ayRU, byRU);
  side_speeds(P, sLU, 0, axLU, bxLU);
  side_speeds(P, sLU, 1, ayLU, byLU);
  side_speeds(P, sRD, 0, axRD, bxRD);
  side_speeds(P, sRD, 1, ayRD, byRD);
  side_speeds(P, sLD, 0, axLD, bxLD);
  side_speeds(P, sLD, 1, ayLD, byLD);
  const double SR = fmax2(fmax2(fmax2(axRU, axLU), axRD), axLD);
  const double SL = fmin2(fmin2(fmin2(bxRU, bxLU), bxRD), bxLD);
  const double SU = fmax2(fmax2(fmax2(ayRU, ayLU), ayRD), ayLD);
  const double SD = fmin2(fmin2(fmin2(byRU, byLU), byRD), byLD);
  double FxRU[NE], FyRU[NE], FxLU[NE], FyLU[NE], FxRD[NE], FyRD[NE], FxLD[NE], FyLD[NE];
  side_flux_hard(P, sRU, FxRU, FyRU);
  side_flux_hard(P, sLU, FxLU, FyLU);
  side_flux_hard(P, sRD, FxRD, FyRD);
  side_flux_hard(P, sLD, FxLD, FyLD);
  double EzRs, EzLs, EzUs, EzDs;
  if (P.flux == 2) {
    double BxUs, BxDs, ByRs, ByLs, fU7, fD7;
    hll1_cm(URU, ULU, FxRU, FxLU, SR, SL, 5, 6, BxUs, fU7);
    hll1_cm(URD, ULD, FxRD, FxLD, SR, SL, 5, 6, BxDs, fD7);
    hll1_cm(URU, URD, FyRU, FyRD, SU, SD, 6, 5, ByRs, EzRs);
    hll1_cm(ULU, ULD, FyLU, FyLD, SU, SD, 6, 5, ByLs, EzLs);
    EzUs = -fU7;
    EzDs = -fD7;
    if (SL > 0) return EzLs;
    if (SR < 0) return EzRs;
    if (SD > 0) return EzDs;
    if (SU < 0) return EzUs;
    // HLL_Flux_2D.f90:61-64; the corner Ez values EzRU.. are never assigned
    // in the reference and are taken as 0.
    const double z = 0.0;
    const double BxRU = URU[5], BxLU = ULU[5], BxRD = URD[5], BxLD = ULD[5];
    const double ByRU = URU[6], ByLU = ULU[6], ByRD = URD[6], ByLD = ULD[6];
    const double den = 2 * (SR - SL) * (SU - SD);
    const double BxSS = dvz<false>(2 * SR * SU * BxRU - 2 * SL * SU * BxLU + 2 * SL * SD * BxLD - 2 * SR * SD * BxRD -
                               SR * (z - z) + SL * (z - z) - (SR - SL) * (EzUs - EzDs), den);
    const double BySS = dvz<false>(2 * SR * SU * ByRU - 2 * SL * SU * ByLU + 2 * SL * SD * ByLD - 2 * SR * SD * ByRD +
                               SU * (z - z) - SD * (z - z) + (SU - SD) * (EzRs - EzLs), den);
    return 0.25 * (EzRs + EzLs + EzUs + EzDs) - 0.25 * SU * (BxUs - BxSS) - 0.25 * SD * (BxDs - BxSS) +
           0.25 * SR * (ByRs - BySS) + 0.25 * SL * (ByLs - BySS);
  }
  // HLLC / HLLD vertex solvers: four 1-D solves, plain average for Ez**
  double Fh[NE], Us[NE];
  auto solve = [&](const Side& r, const Side& l, const double* Fr, const double* Fl, double sr, double sl, int dir) {
    if (P.flux == 3) hllcd_flux<false>(P, r, l, Fr, Fl, sr, sl, dir, Fh, Us);
    else hllcd_flux<true>(P, r, l, Fr, Fl, sr, sl, dir, Fh, Us);
  };
  solve(sRU, sLU, FxRU, FxLU, SR, SL, 0);
  EzUs = -Fh[6];
  solve(sRD, sLD, FxRD, FxLD, SR, SL, 0);
  EzDs = -Fh[6];
  solve(sRU, sRD, FyRU, FyRD, SU, SD, 1);
  EzRs = Fh[5];
  solve(sLU, sLD, FyLU, FyLD, SU, SD, 1);
  EzLs = Fh[5];
  if (SL > 0) return EzLs;
  if (SR < 0) return EzRs;
  if (SD > 0) return EzDs;
  if (SU < 0) return EzUs;
  return 0.25 * (EzRs + EzLs + EzUs + EzDs);
}

// ------------------------------------------------------- eigenmatrix ------
// eigenmatrix.f90:1-407 for the normal (1,0,0) (dir 0) or (0,1,0) (dir 1):
// right (R) and left (L) eigenvectors of the conservative ideal-MHD system,
// column-major R[r + 8*c]. The tangent t of compute_t_vector (:411-433)
// is kept general; products with the constant zero normal components are
// dropped. sin/cos(atan(1)) are the correctly rounded constants.
GDF_HD void tangent(int dir, double B1, double B2, double B3, double& t1, double& t2, double& t3) {
  // n x B and (n x B) x n for n = e_x / e_y; pick_orthogonal if |n x B|^2 < 1e-7
  double tp1, tp2, tp3;
  if (dir == 0) {
    // nB = (0, -B3, B2)
    if (sq(B3) + sq(B2) < 1e-7) { tp1 = -0.0; tp2 = 1.0; tp3 = 1.0; }
    else { tp1 = 0.0; tp2 = B2; tp3 = B3; }
  } else {
    // nB = (B3, 0, -B1)
    if (sq(B3) + sq(B1) < 1e-7) { tp1 = 1.0; tp2 = -0.0; tp3 = 1.0; }
    else { tp1 = B1; tp2 = 0.0; tp3 = B3; }
  }
  const double nrm = sqrt(sq(tp1) + sq(tp2) + sq(tp3));
  t1 = tp1 / nrm;
  t2 = tp2 / nrm;
  t3 = tp3 / nrm;
}

// The quantities both eigenvector sets of eigenmatrix.f90 start from: the
// pressure (:21), the tangent t of compute_t_vector (:411-433) and n x t.
struct EigFrame {
  double gm, g1, p, t1, t2, t3, TxN1, TxN2, TxN3;
};
GDF_HD void eigen_frame(const Phys& P, int dir, double rho, double u1, double u2, double u3, double E, double B1,
                        double B2, double B3, EigFrame& f) {
  f.gm = P.gflux;
  f.g1 = f.gm - 1.0;
  const double kin = sq(u1) + sq(u2) + sq(u3);
  f.p = P.eig_p_typo ? f.g1 * (E - 0.5 * kin - 0.5 * (sq(B1) + sq(B2) + sq(B3)))
                     : f.g1 * (E - 0.5 * rho * kin - 0.5 * (sq(B1) + sq(B2) + sq(B3)));
  tangent(dir, B1, B2, B3, f.t1, f.t2, f.t3);
  // normal components: n_d = 1, others 0
  // TxN = n x t rotated as in the reference: TxN1 = n3 t2 - n2 t3, ...
  f.TxN1 = dir == 0 ? 0.0 : -f.t3;
  f.TxN2 = dir == 0 ? f.t3 : 0.0;
  f.TxN3 = dir == 0 ? -f.t2 : f.t1;
}

#define GDF_EIG_UNPACK                                                   \
  const double gm = f.gm, g1 = f.g1, p = f.p, t1 = f.t1, t2 = f.t2, t3 = f.t3; \
  const double TxN1 = f.TxN1, TxN2 = f.TxN2, TxN3 = f.TxN3;              \
  (void)gm; (void)g1; (void)p; (void)t1; (void)t2; (void)t3;            \
  (void)TxN1; (void)TxN2; (void)TxN3;

// right eigenvectors (eigenmatrix.f90:21-180), column-major R[r + 8*c]
GDF_HD void eigen_right(int dir, const EigFrame& f, double rho, double u1, double u2, double u3, double B1, double B2,
                        double B3, double* R) {
  GDF_EIG_UNPACK
  {
    const double rhosq = sqrt(fabs(rho));
    const double a2 = fabs(gm * p / rho);
    const double a = sqrt(a2);
    const double sqg2 = sqrt(1.0 / (2.0 * gm));
    const double sq12 = sqrt(0.5);
    const double sqpr = sqrt(fabs(p)) / rho;
    const double sqpor = sqrt(fabs(p / rho));
    const double sq1og = sqrt(1.0 / gm);
    const double b1s = dvz<false>(B1, rhosq), b2s = dvz<false>(B2, rhosq), b3s = dvz<false>(B3, rhosq);
    const double bN = dir == 0 ? b1s : b2s;
    const double d = a2 + (sq(b1s) + sq(b2s) + sq(b3s));
    const double disc = sqrt(fabs(sq(d) - 4.0 * a2 * sq(bN)));
    const double cf = sqz<false>(0.5 * fabs(d + disc));
    const double cs = sqz<false>(0.5 * fabs(d - disc));
    const double bNsum = dir == 0 ? ((b1s + b2s * 0.0) + b3s * 0.0) : ((b1s * 0.0 + b2s) + b3s * 0.0);
    const double beta1 = sgn1(bNsum * 1.0);
    double alphaf, alphas;
    if (fabs(cf * cf - cs * cs) <= 1.0e-12) {
      alphaf = 0x1.6a09e667f3bccp-1;
      alphas = 0x1.6a09e667f3bcdp-1;
    } else {
      const double den = sqz<false>(fabs(cf * cf - cs * cs));
      alphaf = dvz<false>(sqz<false>(fabs(a2 - cs * cs)), den);
      alphas = dvz<false>(sqz<false>(fabs(cf * cf - a2)), den);
    }
    const double bst = (b1s * t1 + b2s * t2 + b3s * t3);
    const double rc = rhosq * cf;
    double ru[8][8];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
      for (int c = 0; c < 8; ++c) ru[r][c] = 0.0;
    ru[0][0] = sqrt(g1 / gm) * rhosq;
    // divergence wave: n components only
    ru[5 + dir][1] = sq1og * a;
    // Alfven waves
    ru[1][2] = -sq12 * (sqpr * TxN1);
    ru[2][2] = -sq12 * (sqpr * TxN2);
    ru[3][2] = -sq12 * (sqpr * TxN3);
    ru[5][2] = sq12 * sqpor * TxN1;
    ru[6][2] = sq12 * sqpor * TxN2;
    ru[7][2] = sq12 * sqpor * TxN3;
    // fast waves: alphaf*a2*n_k + alphas*a*(bst*n_k - bN*t_k)
    const double afa2 = alphaf * a2, asa = alphas * a;
    {
      const double m1 = dir == 0 ? (afa2 + asa * (bst - bN * t1)) : (asa * (-(bN * t1)));
      const double m2 = dir == 1 ? (afa2 + asa * (bst - bN * t2)) : (asa * (-(bN * t2)));
      const double m3 = asa * (-(bN * t3));
      ru[1][4] = dvz<false>(sqg2 * m1, rc);
      ru[2][4] = dvz<false>(sqg2 * m2, rc);
      ru[3][4] = dvz<false>(sqg2 * m3, rc);
    }
    ru[0][4] = sqg2 * alphaf * rhosq;
    ru[4][4] = sqg2 * alphaf * rhosq * a2;
    ru[5][4] = sqg2 * alphas * a * t1;
    ru[6][4] = sqg2 * alphas * a * t2;
    ru[7][4] = sqg2 * alphas * a * t3;
    // slow waves
    const double cf2 = sq(cf);
    {
      const double bs = beta1 * sqg2;
      const double k1 = dir == 0 ? (alphaf * cf2 * t1 + a * alphas * bN) : (alphaf * cf2 * t1);
      const double k2 = dir == 1 ? (alphaf * cf2 * t2 + alphas * a * bN) : (alphaf * cf2 * t2);
      const double k3 = alphaf * cf2 * t3;
      ru[1][6] = dvz<false>(bs * k1, rc);
      ru[2][6] = dvz<false>(bs * k2, rc);
      ru[3][6] = dvz<false>(bs * k3, rc);
    }
    ru[0][6] = sqg2 * alphas * rhosq;
    ru[4][6] = sq(a) * sqg2 * alphas * rhosq;
    ru[5][6] = -sqg2 * alphaf * a * t1;
    ru[6][6] = -sqg2 * alphaf * a * t2;
    ru[7][6] = -sqg2 * alphaf * a * t3;
    // paired columns (4 = 3 mirrored, 6 = 5, 8 = 7)
#pragma unroll
    for (int pcol = 2; pcol <= 6; pcol += 2) {
      ru[0][pcol + 1] = ru[0][pcol];
      ru[1][pcol + 1] = -ru[1][pcol];
      ru[2][pcol + 1] = -ru[2][pcol];
      ru[3][pcol + 1] = -ru[3][pcol];
      ru[4][pcol + 1] = ru[4][pcol];
      ru[5][pcol + 1] = ru[5][pcol];
      ru[6][pcol + 1] = ru[6][pcol];
      ru[7][pcol + 1] = ru[7][pcol];
    }
    const double k2 = sq(u1) + sq(u2) + sq(u3);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      R[0 + 8 * m] = dvz<false>(ru[0][m], g1);
      R[1 + 8 * m] = dvz<false>(ru[0][m] * u1 + ru[1][m] * rho, g1);
      R[2 + 8 * m] = dvz<false>(ru[0][m] * u2 + ru[2][m] * rho, g1);
      R[3 + 8 * m] = dvz<false>(ru[0][m] * u3 + ru[3][m] * rho, g1);
      R[4 + 8 * m] = dvz<false>(dvz<false>(ru[4][m], g1) + B1 * ru[5][m] + B2 * ru[6][m] + B3 * ru[7][m] + 0.5 * ru[0][m] * k2 +
                            ru[1][m] * u1 * rho + ru[2][m] * u2 * rho + ru[3][m] * u3 * rho, g1);
      R[5 + 8 * m] = dvz<false>(ru[5][m], g1);
      R[6 + 8 * m] = dvz<false>(ru[6][m], g1);
      R[7 + 8 * m] = dvz<false>(ru[7][m], g1);
    }
  }
}

// left eigenvectors (eigenmatrix.f90:185-394), column-major L[r + 8*c]
GDF_HD void eigen_left(int dir, const EigFrame& f, double rho, double u1, double u2, double u3, double B1, double B2,
                       double B3, double* L) {
  GDF_EIG_UNPACK
  {
    const double rhosq = sqrt(rho);
    const double a2 = fabs(gm * p / rho);
    const double a = sqrt(a2);
    const double b1s = dvz<false>(B1, rhosq), b2s = dvz<false>(B2, rhosq), b3s = dvz<false>(B3, rhosq);
    const double BNs = dir == 0 ? b1s : b2s;
    const double BN = dir == 0 ? B1 : B2;
    const double d = a2 + (sq(b1s) + sq(b2s) + sq(b3s));
    const double disc = sqrt(fabs(sq(d) - 4.0 * a2 * sq(BNs)));
    const double cf = sqz<false>(0.5 * fabs(d + disc));
    const double cs = sqz<false>(0.5 * fabs(d - disc));
    double alphaf, alphas;
    if (fabs(cf * cf - cs * cs) <= 1.0e-12) {
      alphaf = 0x1.6a09e667f3bccp-1;
      alphas = 0x1.6a09e667f3bcdp-1;
    } else {
      const double den = sqz<false>(fabs(cf * cf - cs * cs));
      alphaf = dvz<false>(sqz<false>(fabs(a2 - cs * cs)), den);
      alphas = dvz<false>(sqz<false>(fabs(cf * cf - a2)), den);
    }
    const double twosq = sqrt(2.0);
    // sign(1, BNs*1): BNs summed as (b1s*n1 + b2s*n2) + b3s*n3 so that the
    // sign of a zero matches
    const double BNsum = dir == 0 ? ((b1s + b2s * 0.0) + b3s * 0.0) : ((b1s * 0.0 + b2s) + b3s * 0.0);
    const double beta1 = sgn1(BNsum * 1.0);
    const double sqgam = sqrt(g1 / gm);
    const double BT = (B1 * t1 + B2 * t2 + B3 * t3);
    const double gu1sq = sqrt(1.0 / gm);
    double lu[8][8];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
      for (int c = 0; c < 8; ++c) lu[r][c] = 0.0;
    lu[0][0] = 1.0 / (sqgam * rhosq);
    lu[0][4] = -1.0 / (a2 * sqgam * rhosq);
    // nen of eigenmatrix.f90:246-247 for a unit normal: |t_perp|^2
    const double nen = dir == 0 ? (sq(t2) + sq(t3)) : (sq(t1) + sq(t3));
    const double nen2 = a * gu1sq * nen;
    if (dir == 0) {
      lu[1][5] = dvz<false>(sq(t2) + sq(t3), nen2);
      lu[1][6] = dvz<false>(-(t2 * t1), nen2);
      lu[1][7] = dvz<false>(-(t1 * t3), nen2);
    } else {
      lu[1][5] = dvz<false>(-(t1 * t2), nen2);
      lu[1][6] = dvz<false>(sq(t1) + sq(t3), nen2);
      lu[1][7] = dvz<false>(-(t2 * t3), nen2);
    }
    const double nen3 = sqrt(2.0) * sqrt(fabs(p)) * nen;
    const double nen31 = nen3 / sqrt(fabs(rho));
    lu[2][1] = dvz<false>(rho * (-TxN1), nen3);
    lu[2][2] = dvz<false>(rho * (-TxN2), nen3);
    lu[2][3] = dvz<false>(rho * (-TxN3), nen3);
    lu[2][5] = dvz<false>(TxN1, nen31);
    lu[2][6] = dvz<false>(TxN2, nen31);
    lu[2][7] = dvz<false>(TxN3, nen31);
    const double cf2 = sq(cf);
    const double q = a * sq(BN) * sq(alphas) + rhosq * cf2 * alphaf * (a * rhosq * alphaf + BT * alphas);
    const double nen51 = twosq * a * nen * gu1sq * q;
    const double nen52 = twosq * a * gu1sq * (sq(alphaf) + sq(alphas)) * nen;
    const double nen71 = twosq * beta1 * nen * gu1sq * q;
    const double rcf = rho * cf;
    const double Term54 = dvz<false>(alphaf, twosq * sq(a) * gu1sq * rhosq * (sq(alphaf) + sq(alphas)));
    const double Term74 = dvz<false>(alphas, twosq * sq(a) * gu1sq * rhosq * (sq(alphaf) + sq(alphas)));
    // Term51..Term77 of eigenmatrix.f90:287-351 with the zero normal
    // components removed
    double T51, T52, T53, T55, T56, T57, T71, T72, T73, T75, T76, T77;
    if (dir == 0) {
      T51 = rcf * ((-(sq(t2) + sq(t3))) * rhosq * cf2 * alphaf);
      T52 = rcf * ((-(t2 * t1)) * rhosq * cf2 * alphaf - a * BN * alphas * t2);
      T53 = rcf * ((-(t1 * t3)) * rhosq * cf2 * alphaf - a * t3 * BN * alphas);
      T55 = 0.0;
      T56 = alphas * t2;
      T57 = t3 * alphas;
      T71 = rcf * ((B1 * (sq(t2) + sq(t3))) * alphas);
      T72 = rcf * (((-t3) * (-(B3 * t2)) + B2 * sq(t2)) * alphas + a * rhosq * alphaf * t2);
      T73 = rcf * (a * t3 * rhosq * alphaf + alphas * (B3 * sq(t3) + B2 * (-t3) * TxN3));
      T75 = 0.0;
      T76 = -alphaf * t2;
      T77 = -alphaf * t3;
    } else {
      T51 = rcf * ((t1 * t2) * rhosq * cf2 * alphaf - a * BN * alphas * (-t1));
      T52 = rcf * ((sq(t1) + sq(t3)) * rhosq * cf2 * alphaf);
      T53 = rcf * ((-(t2 * t3)) * rhosq * cf2 * alphaf - a * t3 * BN * alphas);
      T55 = t1 * alphas;
      T56 = 0.0;
      T57 = t3 * alphas;
      T71 = rcf * (a * t1 * rhosq * alphaf + ((B3 * t1) * t3 + B1 * sq(t1)) * alphas);
      T72 = rcf * ((B2 * (sq(t1) + sq(t3))) * alphas);
      T73 = rcf * (a * t3 * rhosq * alphaf + alphas * (B3 * sq(t3) + B1 * t3 * TxN3));
      T75 = -alphaf * t1;
      T76 = 0.0;
      T77 = -alphaf * t3;
    }
    lu[4][1] = dvz<false>(-T51, nen51);
    lu[4][2] = dvz<false>(T52, nen51);
    lu[4][3] = dvz<false>(T53, nen51);
    lu[4][4] = Term54;
    lu[4][5] = dvz<false>(T55, nen52);
    lu[4][6] = dvz<false>(T56, nen52);
    lu[4][7] = dvz<false>(T57, nen52);
    lu[6][1] = dvz<false>(T71, nen71);
    lu[6][2] = dvz<false>(T72, nen71);
    lu[6][3] = dvz<false>(T73, nen71);
    lu[6][4] = Term74;
    lu[6][5] = dvz<false>(T75, nen52);
    lu[6][6] = dvz<false>(T76, nen52);
    lu[6][7] = dvz<false>(T77, nen52);
#pragma unroll
    for (int pr = 2; pr <= 6; pr += 2) {
      lu[pr + 1][0] = lu[pr][0];
      lu[pr + 1][1] = -lu[pr][1];
      lu[pr + 1][2] = -lu[pr][2];
      lu[pr + 1][3] = -lu[pr][3];
      lu[pr + 1][4] = lu[pr][4];
      lu[pr + 1][5] = lu[pr][5];
      lu[pr + 1][6] = lu[pr][6];
      lu[pr + 1][7] = lu[pr][7];
    }
    const double g12 = sq(g1);
    const double k2 = sq(u1) + sq(u2) + sq(u3);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const double* l = lu[m];
      L[m + 8 * 0] = l[0] * g1 - dvz<false>(l[1] * u1 * g1, rho) - dvz<false>(l[2] * u2 * g1, rho) - dvz<false>(l[3] * u3 * g1, rho) + l[4] * g12 * k2 * .5;
      L[m + 8 * 1] = -l[4] * u1 * g12 + dvz<false>(l[1] * g1, rho);
      L[m + 8 * 2] = -l[4] * u2 * g12 + dvz<false>(l[2] * g1, rho);
      L[m + 8 * 3] = -l[4] * u3 * g12 + dvz<false>(l[3] * g1, rho);
      L[m + 8 * 4] = l[4] * g12;
      L[m + 8 * 5] = l[5] * g1 - B1 * l[4] * g12;
      L[m + 8 * 6] = l[6] * g1 - B2 * l[4] * g12;
      L[m + 8 * 7] = l[7] * g1 - B3 * l[4] * g12;
    }
  }
}

GDF_HD void eigenmatrix(const Phys& P, int dir, double rho, double u1, double u2, double u3, double E, double B1,
                        double B2, double B3, double* R, double* L) {
  EigFrame f;
  eigen_frame(P, dir, rho, u1, u2, u3, E, B1, B2, B3, f);
  eigen_right(dir, f, rho, u1, u2, u3, B1, B2, B3, R);
  eigen_left(dir, f, rho, u1, u2, u3, B1, B2, B3, L);
  if (P.eig_identity) {
    double sr = 0, sl = 0;
#pragma unroll
    for (int q = 0; q < 64; ++q) sr = sr + fabs(R[q]);
#pragma unroll
    for (int q = 0; q < 64; ++q) sl = sl + fabs(L[q]);
    if (sr > 1e4 || sl > 1e4) {
#pragma unroll
      for (int q = 0; q < 64; ++q) { R[q] = 0.0; L[q] = 0.0; }
#pragma unroll
      for (int q = 0; q < 8; ++q) { R[q * 9] = 1.0; L[q * 9] = 1.0; }
    }
  }
}

// minmod.f90:5-27 for one component (TVB bound Mh2 = M*h**2)
GDF_HD double minmod1(double du, double dr, double dl, double Mh2) {
  if (fabs(du) <= Mh2) return du;
  const double s = (sgn1(du) + sgn1(dr) + sgn1(dl)) / 3.0;
  if (fabs(s) == 1) return s * fmin2(fmin2(fabs(du), fabs(dr)), fabs(dl));
  return 0.0;
}

// pressure.f90:1-8
GDF_HD double pressure(double g, const double* U) {
  return (g - 1) * (U[4] - 0.5 * (sq(U[1]) + sq(U[2]) + sq(U[3])) / U[0] - 0.5 * (sq(U[5]) + sq(U[6]) + sq(U[7])));
}

}  // namespace gdf
