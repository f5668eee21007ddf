// gdf_oracle.cpp -- CPU restatement of the GDF_Balsara_P2_0316 time step.
//
// TEST INFRASTRUCTURE ONLY. This file is the checker for the CUDA library:
// only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
// it, and nothing in the product links or calls it.
//
// What it restates: the reference's Fortran 90 hot path (paths relative to
// the reference project, GDF_Balsara_P2_0316/ unless another directory is
// named), subroutine by subroutine, keeping the Fortran evaluation order of
// every expression (left-to-right for + - * /, ** 2 as x*x, ** 0.5 as sqrt,
// MAX/MIN as gfortran's NaN-skipping sequential comparisons, SIGN via
// copysign, MATMUL/SUM as sequential sums from zero) and the reference's
// quirks (the Q-list in the project notes), with the variant lines of
// MHD_Globally_Divergence_Free/ as run-time switches.
//
// Parity status: UNPINNED by the reference itself. The reference ships no
// tests, no golden vectors and no fixtures, and it cannot be compiled here
// (no Fortran compiler in the image). The restatement is pinned instead by
// the invariants the reference's own diagnostics check (conservation,
// totaldiv at round-off, calculate_L2error convergence on init1.txt) and
// by known answers of the published methods for the pointwise routines
// (Rusanov, HLL, Toro's HLLC, Li's HLLC-C, Miyoshi-Kusano's HLLD, the
// ideal-MHD wave speeds of the eigensystem), with the reference's own
// departures from them written as closed-form terms, in tests/.
//
// Build: oracle/Makefile (g++ -O2 -ffp-contract=off, x86-64 baseline ISA,
// so no FMA is formed, as in a gfortran -O3 build without -march).

#include "../include/gdf.h"
#include "../include/gdf_p3.h"
#include "../include/gdf_cy.h"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <omp.h>

namespace {

// ---------------------------------------------------------------- helpers --
// gfortran expands MAX(a,b,...) as  m=a; if (b > m || isnan(m)) m=b; ...
inline double fmax2(double a, double b) { return (b > a || std::isnan(a)) ? b : a; }
inline double fmin2(double a, double b) { return (b < a || std::isnan(a)) ? b : a; }
inline double fmax4(double a, double b, double c, double d) { return fmax2(fmax2(fmax2(a, b), c), d); }
inline double fmin4(double a, double b, double c, double d) { return fmin2(fmin2(fmin2(a, b), c), d); }
inline double sgn1(double b) { return std::copysign(1.0, b); }  // sign(1d0,b)
inline double sq(double x) { return x * x; }                     // x**2

constexpr int NG = 5;     // NumGLP
constexpr int NP = 10;    // dimPk for k = 2
constexpr int NE = 8;     // NumEq

// sin(atan(1d0)), cos(atan(1d0)) as a Fortran compiler folds them
// (eigenmatrix.f90:55-56), correctly rounded.
const double SIN_ATAN1 = 0x1.6a09e667f3bccp-1;
const double COS_ATAN1 = 0x1.6a09e667f3bcdp-1;

struct Oracle {
  GdfConfig c{};
  int Nx = 0, Ny = 0;
  double hx = 0, hy = 0, hx1 = 0, hy1 = 0;
  double gamma = 0, gamma1 = 0;   // com.txt:7-8
  double gflux = 0;               // MHD_flux.f90:7 / eigenmatrix.f90:19

  // get_GLP.f90:38-56
  double lambda[NG], weight[NG], lambdaL[NG];
  // get_basis.f90 tables, 0-based: phiG[i1][j1][d]
  double phiG[NG][NG][NP], phixG[NG][NG][NP], phiyG[NG][NG][NP];
  double phiGLL[2][NG][NG][NP];
  double phiGR[NG][NP], phiGL[NG][NP], phiGU[NG][NP], phiGD[NG][NP];
  double phiRU[NP], phiLU[NP], phiRD[NP], phiLD[NP];
  double mm[NP];
  double EzG[NG][3], EzxG[NG][3], EzyG[NG][3], mmE[3], EzR[3], EzL[3], EzU[3], EzD[3];

  std::vector<int32_t> trouble;  // Is_Trouble_Cell(Nx,Ny)

  // work arrays of Lh / LhEz / RK3 / the limiter, allocated once
  std::vector<double> Fxhat, Fyhat, EzRL, EzUD, EzV;
  std::vector<double> w_du, w_uI, w_uII, w_uh0, w_uhmod;
  std::vector<double> w_dez1, w_dez2, w_BxI, w_ByI, w_BxII, w_ByII, w_Bx0, w_By0;
  std::vector<int32_t> w_f1, w_f2, w_f3;
  std::vector<double> cornRU, cornLU, cornRD, cornLD;

  // ------------------------------------------------------------- layout --
  size_t NX2() const { return (size_t)Nx + 2; }
  size_t NY2() const { return (size_t)Ny + 2; }
  size_t plane() const { return NX2() * NY2(); }
  size_t uhsize() const { return plane() * NP * NE; }
  // uh(i,j,d,n): i 0..Nx+1, j 0..Ny+1, d 1..10, n 1..8
  size_t U(int i, int j, int d, int n) const {
    return (size_t)i + NX2() * ((size_t)j + NY2() * ((size_t)(d - 1) + NP * (size_t)(n - 1)));
  }
  // Bx(i,j,d): i 0..Nx, j 1..Ny ; By(i,j,d): i 1..Nx, j 0..Ny
  size_t BXi(int i, int j, int d) const { return (size_t)i + (size_t)(Nx + 1) * ((size_t)(j - 1) + (size_t)Ny * (d - 1)); }
  size_t BYi(int i, int j, int d) const { return (size_t)(i - 1) + (size_t)Nx * ((size_t)j + (size_t)(Ny + 1) * (d - 1)); }
  size_t bxsize() const { return (size_t)(Nx + 1) * Ny * 3; }
  size_t bysize() const { return (size_t)Nx * (Ny + 1) * 3; }
  // Fxhat(i,j,g,n): i 0..Nx, j 1..Ny ; Fyhat(i,j,g,n): i 1..Nx, j 0..Ny
  size_t FX(int i, int j, int g, int n) const { return (((size_t)(j - 1) * (Nx + 1) + i) * NG + g) * NE + (n - 1); }
  size_t FY(int i, int j, int g, int n) const { return (((size_t)j * Nx + (i - 1)) * NG + g) * NE + (n - 1); }
  size_t EX(int i, int j, int g) const { return ((size_t)(j - 1) * (Nx + 1) + i) * NG + g; }
  size_t EY(int i, int j, int g) const { return ((size_t)j * Nx + (i - 1)) * NG + g; }
  size_t VX(int i, int j) const { return (size_t)j * (Nx + 1) + i; }       // EzVertex(0:Nx,0:Ny)
  size_t CN(int i, int j) const { return ((size_t)j * NX2() + i) * NE; }   // corner traces, all cells

  static void par_copy(const double* src, double* dst, size_t n) {
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < n; ++q) dst[q] = src[q];
  }

  // ------------------------------------------------------------- set-up --
  void setup(const GdfConfig& cfg) {
    c = cfg;
    Nx = c.nx; Ny = c.ny;
    gamma = c.gamma; gamma1 = gamma - 1;
    gflux = c.gamma_flux;
    // init_data.f90:21-24
    hx = (c.xb - c.xa) / Nx;
    hy = (c.yb - c.ya) / Ny;
    hx1 = 0.5 * hx;
    hy1 = 0.5 * hy;
    get_GLP();
    get_basis();
    trouble.assign((size_t)Nx * Ny, 0);
    Fxhat.assign((size_t)(Nx + 1) * Ny * NG * NE, 0.0);
    Fyhat.assign((size_t)Nx * (Ny + 1) * NG * NE, 0.0);
    EzRL.assign((size_t)(Nx + 1) * Ny * NG, 0.0);
    EzUD.assign((size_t)Nx * (Ny + 1) * NG, 0.0);
    EzV.assign((size_t)(Nx + 1) * (Ny + 1), 0.0);
    cornRU.assign(plane() * NE, 0.0);
    cornLU.assign(plane() * NE, 0.0);
    cornRD.assign(plane() * NE, 0.0);
    cornLD.assign(plane() * NE, 0.0);
  }

  // get_GLP.f90:38-56 (NumGLP = 5 branch)
  void get_GLP() {
    lambda[0] = -0.9061798459386639927976269;
    lambda[1] = -0.5384693101056830910363144;
    lambda[2] = 0;
    lambda[3] = 0.5384693101056830910363144;
    lambda[4] = 0.9061798459386639927976269;
    weight[0] = 0.2369268850561890875142640;
    weight[1] = 0.4786286704993664680412915;
    weight[2] = 0.5688888888888888888888889;
    weight[3] = 0.4786286704993664680412915;
    weight[4] = 0.2369268850561890875142640;
    lambdaL[0] = -1;
    lambdaL[1] = -0.6546536707079771437983;
    lambdaL[2] = 0;
    lambdaL[3] = 0.654653670707977143798;
    lambdaL[4] = 1;
  }

  // get_basis.f90:5-189
  void get_basis() {
    const double c23 = 2.0 / 3.0, c25 = 2.0 / 5.0, c13 = 1.0 / 3.0, c35 = 3.0 / 5.0;
    const double ru[NP] = {1, 1, 1, c23, 1, c23, c25, c23, c23, c25};
    const double lu[NP] = {1, -1, 1, c23, -1, c23, -c25, c23, -c23, c25};
    const double rd[NP] = {1, 1, -1, c23, -1, c23, c25, -c23, c23, -c25};
    const double ld[NP] = {1, -1, -1, c23, 1, c23, -c25, -c23, -c23, -c25};
    for (int d = 0; d < NP; ++d) { phiRU[d] = ru[d]; phiLU[d] = lu[d]; phiRD[d] = rd[d]; phiLD[d] = ld[d]; }
    const double mmv[NP] = {1, 1.0 / 3.0, 1.0 / 3.0, 4.0 / 45.0, 1.0 / 9.0, 4.0 / 45.0,
                            4.0 / 175.0, 4.0 / 135.0, 4.0 / 135.0, 4.0 / 175.0};
    for (int d = 0; d < NP; ++d) mm[d] = mmv[d];
    for (int i = 0; i < NG; ++i) {
      const double li = lambda[i], lj_dummy = 0; (void)lj_dummy;
      const double Li = lambdaL[i];
      for (int j = 0; j < NG; ++j) {
        const double lj = lambda[j], Lj = lambdaL[j];
        double* G = phiG[i][j];
        double* X = phixG[i][j];
        double* Y = phiyG[i][j];
        double* G1 = phiGLL[0][i][j];
        double* G2 = phiGLL[1][i][j];
        G[0] = 1; G1[0] = 1; G2[0] = 1; X[0] = 0; Y[0] = 0;
        G[1] = li; G1[1] = Li; G2[1] = li; X[1] = 1.0 / hx1; Y[1] = 0;
        G[2] = lj; G1[2] = lj; G2[2] = Lj; X[2] = 0; Y[2] = 1.0 / hy1;
        G[3] = sq(li) - c13; G1[3] = sq(Li) - c13; G2[3] = sq(li) - c13; X[3] = 2.0 * li / hx1; Y[3] = 0;
        G[4] = li * lj; G1[4] = Li * lj; G2[4] = li * Lj; X[4] = lj / hx1; Y[4] = li / hy1;
        G[5] = sq(lj) - c13; G1[5] = sq(lj) - c13; G2[5] = sq(Lj) - c13; X[5] = 0; Y[5] = 2.0 * lj / hy1;
        G[6] = li * li * li - 3.0 * li / 5.0;
        G1[6] = Li * Li * Li - 3.0 * Li / 5.0;
        G2[6] = li * li * li - 3.0 * li / 5.0;
        X[6] = (3 * sq(li) - c35) / hx1; Y[6] = 0;
        G[7] = (sq(li) - c13) * (lj);
        G1[7] = (sq(Li) - c13) * (lj);
        G2[7] = (sq(li) - c13) * (Lj);
        X[7] = 2.0 * li * lj / hx1; Y[7] = (sq(li) - c13) / hy1;
        G[8] = (li) * (sq(lj) - c13);
        G1[8] = (Li) * (sq(lj) - c13);
        G2[8] = (li) * (sq(Lj) - c13);
        X[8] = (sq(lj) - c13) / hx1; Y[8] = 2.0 * li * lj / hy1;
        G[9] = lj * lj * lj - 3.0 * lj / 5.0;
        G1[9] = lj * lj * lj - 3.0 * lj / 5.0;
        G2[9] = Lj * Lj * Lj - 3.0 * Lj / 5.0;
        X[9] = 0; Y[9] = (3 * sq(lj) - c35) / hy1;
      }
      // face tables (index by the face quadrature point i)
      phiGR[i][0] = 1; phiGL[i][0] = 1; phiGU[i][0] = 1; phiGD[i][0] = 1;
      phiGR[i][1] = 1; phiGL[i][1] = -1; phiGU[i][1] = li; phiGD[i][1] = li;
      phiGR[i][2] = li; phiGL[i][2] = li; phiGU[i][2] = 1; phiGD[i][2] = -1;
      phiGR[i][3] = c23; phiGL[i][3] = c23; phiGU[i][3] = sq(li) - c13; phiGD[i][3] = sq(li) - c13;
      phiGR[i][4] = li; phiGL[i][4] = -li; phiGU[i][4] = li; phiGD[i][4] = -li;
      phiGR[i][5] = sq(li) - c13; phiGL[i][5] = sq(li) - c13; phiGU[i][5] = c23; phiGD[i][5] = c23;
      phiGR[i][6] = c25; phiGL[i][6] = -c25;
      phiGU[i][6] = li * li * li - 3.0 * li / 5.0; phiGD[i][6] = li * li * li - 3.0 * li / 5.0;
      phiGR[i][7] = c23 * (li); phiGL[i][7] = c23 * (li);
      phiGU[i][7] = (sq(li) - c13); phiGD[i][7] = -(sq(li) - c13);
      phiGR[i][8] = (sq(li) - c13); phiGL[i][8] = -(sq(li) - c13);
      phiGU[i][8] = li * c23; phiGD[i][8] = li * c23;
      phiGR[i][9] = li * li * li - 3.0 * li / 5.0; phiGL[i][9] = li * li * li - 3.0 * li / 5.0;
      phiGU[i][9] = c25; phiGD[i][9] = -c25;
      // Ez basis (get_basis.f90:162-172)
      EzG[i][0] = 1; EzG[i][1] = li; EzG[i][2] = sq(li) - c13;
      EzxG[i][0] = 0; EzxG[i][1] = 1 / hx1; EzxG[i][2] = 2 * li / hx1;
      EzyG[i][0] = 0; EzyG[i][1] = 1 / hy1; EzyG[i][2] = 2 * li / hy1;
    }
    EzR[0] = 1; EzR[1] = 1; EzR[2] = c23;
    EzL[0] = 1; EzL[1] = -1; EzL[2] = c23;
    for (int d = 0; d < 3; ++d) { EzU[d] = EzR[d]; EzD[d] = EzL[d]; }
    mmE[0] = 1; mmE[1] = 1.0 / 3.0; mmE[2] = 4.0 / 45.0;
  }

  // ----------------------------------------------------------- set_bc ----
  // set_bc.f90:5-27: x ghosts first, then y ghosts over full rows
  void set_bc(double* uh) const {
    for (int n = 1; n <= NE; ++n)
      for (int d = 1; d <= NP; ++d)
        for (int j = 0; j <= Ny + 1; ++j) {
          if (c.bc_r == 1) uh[U(Nx + 1, j, d, n)] = uh[U(1, j, d, n)];
          else if (c.bc_r == 2) uh[U(Nx + 1, j, d, n)] = uh[U(Nx, j, d, n)];
        }
    for (int n = 1; n <= NE; ++n)
      for (int d = 1; d <= NP; ++d)
        for (int j = 0; j <= Ny + 1; ++j) {
          if (c.bc_l == 1) uh[U(0, j, d, n)] = uh[U(Nx, j, d, n)];
          else if (c.bc_l == 2) uh[U(0, j, d, n)] = uh[U(1, j, d, n)];
        }
    for (int n = 1; n <= NE; ++n)
      for (int d = 1; d <= NP; ++d)
        for (int i = 0; i <= Nx + 1; ++i) {
          if (c.bc_u == 1) uh[U(i, Ny + 1, d, n)] = uh[U(i, 1, d, n)];
          else if (c.bc_u == 2) uh[U(i, Ny + 1, d, n)] = uh[U(i, Ny, d, n)];
        }
    for (int n = 1; n <= NE; ++n)
      for (int d = 1; d <= NP; ++d)
        for (int i = 0; i <= Nx + 1; ++i) {
          if (c.bc_d == 1) uh[U(i, 0, d, n)] = uh[U(i, Ny, d, n)];
          else if (c.bc_d == 2) uh[U(i, 0, d, n)] = uh[U(i, 1, d, n)];
        }
  }

  // ---------------------------------------------------- pointwise physics --
  // eigenvalueMm.f90:1-25 (n1, n2 are INTEGER dummies; gamma of com.txt)
  void eigenvalueMm(double& Amax, double& Amin, double rho, double rhou, double rhov, double rhow,
                    double E, double B1, double B2, double B3, int n1i, int n2i) const {
    const double n1 = n1i, n2 = n2i, n3 = 0;
    double u = rhou / rho, v = rhov / rho, w = rhow / rho;
    double BP = sq(B1) + sq(B2) + sq(B3);
    double Bn = B1 * n1 + B2 * n2 + B3 * n3;
    double un = u * n1 + v * n2 + w * n3;
    double p = gamma1 * (E - 0.5 * rho * (sq(u) + sq(v) + sq(w)) - 0.5 * BP);
    double cc = std::sqrt(std::fabs(gamma * p / rho));
    double X = sq(cc) + BP / rho;
    double cf = std::sqrt(std::fabs(0.5 * (sq(cc) + BP / rho + std::sqrt(sq(X) - 4 * sq(cc) * sq(Bn) / rho))));
    Amax = un + cf;
    Amin = un - cf;
  }

  // Lh.f90:88-135 (x faces) / :155-202 (y faces): conservative state at a
  // point -> flux. dir 0: x flux, 1: y flux. pMD quirk (Lh.f90:189) for the
  // D-side traces and the KML w-term switch (Lh.f90:126) for the L side.
  void point_flux(const double* Uv, double* F, int dir, bool d_side_quirk, bool l_side) const {
    double rho = Uv[0];
    double u = Uv[1] / rho, v = Uv[2] / rho, w = Uv[3] / rho;
    double E = Uv[4], B1 = Uv[5], B2 = Uv[6], B3 = Uv[7];
    double p;
    if (d_side_quirk)
      p = gamma1 * (E - 0.5 * rho * (sq(u) + sq(v) - sq(w)) - 0.5 * (sq(B1) + sq(B2) + sq(B3)));
    else
      p = gamma1 * (E - 0.5 * rho * (sq(u) + sq(v) + sq(w)) - 0.5 * (sq(B1) + sq(B2) + sq(B3)));
    double S = p + 0.5 * (sq(B1) + sq(B2) + sq(B3));
    double T = E + S;
    double K = (l_side && !c.kml_w_term) ? (u * B1 + v * B2) : (u * B1 + v * B2 + w * B3);
    if (dir == 0) {
      F[0] = Uv[1];
      F[1] = rho * sq(u) + S - sq(B1);
      F[2] = rho * u * v - B1 * B2;
      F[3] = rho * u * w - B1 * B3;
      F[4] = T * u - K * B1;
      F[5] = 0;
      F[6] = u * B2 - v * B1;
      F[7] = u * B3 - w * B1;
    } else {
      F[0] = Uv[2];
      F[1] = rho * u * v - B1 * B2;
      F[2] = rho * sq(v) + S - sq(B2);
      F[3] = rho * v * w - B2 * B3;
      F[4] = T * v - K * B2;
      F[5] = v * B1 - u * B2;
      F[6] = 0;
      F[7] = v * B3 - w * B2;
    }
  }

  // MHD_flux.f90:1-42 (gamma hard-coded 5/3, quirk Q1; Fy(4) = rho*w*v - B3*B2)
  void MHD_flux(const double* Uh, double* Fx, double* Fy) const {
    const double g = gflux, g1 = g - 1;
    double rho = Uh[0];
    double u = Uh[1] / rho, v = Uh[2] / rho, w = Uh[3] / rho;
    double E = Uh[4], B1 = Uh[5], B2 = Uh[6], B3 = Uh[7];
    double p = g1 * (E - 0.5 * rho * (sq(u) + sq(v) + sq(w)) - 0.5 * (sq(B1) + sq(B2) + sq(B3)));
    double S = p + 0.5 * (sq(B1) + sq(B2) + sq(B3));
    double T = E + S;
    double K = u * B1 + v * B2 + w * B3;
    Fx[0] = Uh[1];
    Fx[1] = rho * sq(u) + S - sq(B1);
    Fx[2] = rho * u * v - B1 * B2;
    Fx[3] = rho * u * w - B1 * B3;
    Fx[4] = T * u - K * B1;
    Fx[5] = 0;
    Fx[6] = u * B2 - v * B1;
    Fx[7] = u * B3 - w * B1;
    Fy[0] = Uh[2];
    Fy[1] = rho * u * v - B1 * B2;
    Fy[2] = rho * sq(v) + S - sq(B2);
    Fy[3] = rho * w * v - B3 * B2;
    Fy[4] = T * v - K * B2;
    Fy[5] = v * B1 - u * B2;
    Fy[6] = 0;
    Fy[7] = v * B3 - w * B2;
  }

  // Riemann-solver context: the COMMON /flux4/,/flux5/ variables.
  struct RS {
    double FR1[NE], FL1[NE], UR1[NE], UL1[NE], Fhat1[NE], Ustar[NE];
    double SR, SL;
    int direction;
  };

  // LF_Flux.f90:5
  static void LF_Flux(RS& s) {
    double a = fmax2(std::fabs(s.SR), std::fabs(s.SL));
    for (int n = 0; n < NE; ++n) s.Fhat1[n] = 0.5 * (s.FR1[n] + s.FL1[n] - a * (s.UR1[n] - s.UL1[n]));
  }

  // HLL_Flux.f90:5-11
  static void HLL_Flux(RS& s) {
    if (s.SR < 0) {
      for (int n = 0; n < NE; ++n) s.Fhat1[n] = s.FR1[n];
    } else if (s.SL > 0) {
      for (int n = 0; n < NE; ++n) s.Fhat1[n] = s.FL1[n];
    } else {
      for (int n = 0; n < NE; ++n)
        s.Fhat1[n] = (s.SR * s.FL1[n] - s.SL * s.FR1[n] + s.SL * s.SR * (s.UR1[n] - s.UL1[n])) / (s.SR - s.SL);
    }
  }

  // HLL1.f90:1-15
  static void HLL1(const double* UR, const double* UL, const double* FR, const double* FL, double SR, double SL,
                   double* Uhat, double* Fhat) {
    if (SR < 0) {
      for (int n = 0; n < NE; ++n) { Fhat[n] = FR[n]; Uhat[n] = UR[n]; }
    } else if (SL > 0) {
      for (int n = 0; n < NE; ++n) { Fhat[n] = FL[n]; Uhat[n] = UL[n]; }
    } else {
      for (int n = 0; n < NE; ++n) {
        Fhat[n] = (SR * FL[n] - SL * FR[n] + SL * SR * (UR[n] - UL[n])) / (SR - SL);
        Uhat[n] = (SR * UR[n] - SL * UL[n] - (FR[n] - FL[n])) / (SR - SL);
      }
    }
  }

  // HLLC_Flux.f90:9-106
  void HLLC_Flux(RS& s) const {
    double* UR1 = s.UR1; double* UL1 = s.UL1; double* FR1 = s.FR1; double* FL1 = s.FL1;
    const double SR = s.SR, SL = s.SL;
    if (SR < 0) {
      for (int n = 0; n < NE; ++n) { s.Fhat1[n] = FR1[n]; s.Ustar[n] = UR1[n]; }
      return;
    }
    if (SL > 0) {
      for (int n = 0; n < NE; ++n) { s.Fhat1[n] = FL1[n]; s.Ustar[n] = UL1[n]; }
      return;
    }
    double Ust[NE];
    for (int n = 0; n < NE; ++n) Ust[n] = (SR * UR1[n] - SL * UL1[n] + FL1[n] - FR1[n]) / (SR - SL);
    double rhoR = UR1[0], u1R = UR1[1] / rhoR, u2R = UR1[2] / rhoR, u3R = UR1[3] / rhoR, ER = UR1[4];
    double B1R = UR1[5], B2R = UR1[6], B3R = UR1[7];
    double rhoL = UL1[0], u1L = UL1[1] / rhoL, u2L = UL1[2] / rhoL, u3L = UL1[3] / rhoL, EL = UL1[4];
    double B1L = UL1[5], B2L = UL1[6], B3L = UL1[7];
    double B1star = Ust[5], B2star = Ust[6], B3star = Ust[7];
    double Sstar = 0, uRbot = 0, uLbot = 0, BRbot = 0, BLbot = 0, Bstarbot = 0;
    if (s.direction == 1) {
      Sstar = Ust[1] / Ust[0]; uRbot = u1R; uLbot = u1L; BRbot = B1R; BLbot = B1L; Bstarbot = B1star;
    } else if (s.direction == 2) {
      Sstar = Ust[2] / Ust[0]; uRbot = u2R; uLbot = u2L; BRbot = B2R; BLbot = B2L; Bstarbot = B2star;
    }
    double rhoRstar = rhoR * (SR - uRbot) / (SR - Sstar);
    double rhoLstar = rhoL * (SL - uLbot) / (SL - Sstar);
    double PtotR = gamma1 * (ER - 0.5 * rhoR * (sq(u1R) + sq(u2R) + sq(u3R)));
    double PtotL = gamma1 * (EL - 0.5 * rhoL * (sq(u1L) + sq(u2L) + sq(u3L)));
    double PtotRstar = PtotR + rhoR * (SR - uRbot) * (Sstar - uRbot) + sq(Bstarbot) - sq(BRbot);
    double PtotLstar = PtotL + rhoL * (SL - uLbot) * (Sstar - uLbot) + sq(Bstarbot) - sq(BLbot);
    double URs[NE], ULs[NE];
    if (s.direction == 1) {
      URs[1] = (UR1[1] * (SR - uRbot) + PtotRstar - PtotR + BRbot * B1R - Bstarbot * B1star) / (SR - Sstar);
      URs[2] = (UR1[2] * (SR - uRbot) + BRbot * B2R - Bstarbot * B2star) / (SR - Sstar);
      ULs[1] = (UL1[1] * (SL - uLbot) + PtotLstar - PtotL + BLbot * B1L - Bstarbot * B1star) / (SL - Sstar);
      ULs[2] = (UL1[2] * (SL - uLbot) + BLbot * B2L - Bstarbot * B2star) / (SL - Sstar);
    } else {
      URs[1] = (UR1[1] * (SR - uRbot) + BRbot * B1R - Bstarbot * B1star) / (SR - Sstar);
      URs[2] = (UR1[2] * (SR - uRbot) + PtotRstar - PtotR + BRbot * B2R - Bstarbot * B2star) / (SR - Sstar);
      ULs[1] = (UL1[1] * (SL - uLbot) + BLbot * B1L - Bstarbot * B1star) / (SL - Sstar);
      ULs[2] = (UL1[2] * (SL - uLbot) + PtotLstar - PtotL + BLbot * B2L - Bstarbot * B2star) / (SL - Sstar);
    }
    URs[3] = (UR1[3] * (SR - uRbot) + BRbot * B3R - Bstarbot * B3star) / (SR - Sstar);
    ULs[3] = (UL1[3] * (SL - uLbot) + BLbot * B3L - Bstarbot * B3star) / (SL - Sstar);
    double u1Rstar = URs[1] / rhoRstar, u2Rstar = URs[2] / rhoRstar, u3Rstar = URs[3] / rhoRstar;
    double u1Lstar = ULs[1] / rhoLstar, u2Lstar = ULs[2] / rhoLstar, u3Lstar = ULs[3] / rhoLstar;
    double ERstar = ((SR - uRbot) * ER - PtotR * uRbot + PtotRstar * Sstar + BRbot * (u1R * B1R + u2R * B2R + u3R * B3R) -
                     Bstarbot * (u1Rstar * B1star + u2Rstar * B2star + u3Rstar * B3star)) / (SR - Sstar);
    double ELstar = ((SL - uLbot) * EL - PtotL * uLbot + PtotLstar * Sstar + BLbot * (u1L * B1L + u2L * B2L + u3L * B3L) -
                     Bstarbot * (u1Lstar * B1star + u2Lstar * B2star + u3Lstar * B3star)) / (SL - Sstar);
    URs[0] = rhoRstar; URs[4] = ERstar;
    ULs[0] = rhoLstar; ULs[4] = ELstar;
    for (int n = 5; n < 8; ++n) { URs[n] = Ust[n]; ULs[n] = Ust[n]; }
    if (Sstar > 0) {
      for (int n = 0; n < NE; ++n) { s.Fhat1[n] = FL1[n] + SL * (ULs[n] - UL1[n]); s.Ustar[n] = ULs[n]; }
    } else {
      for (int n = 0; n < NE; ++n) { s.Fhat1[n] = FR1[n] + SR * (URs[n] - UR1[n]); s.Ustar[n] = URs[n]; }
    }
  }

  // HLLD_Flux.f90:14-189 (Ptot without magnetic pressure, quirk Q4;
  // +1e-15 in D; two-stage switch on |B*|, SR*-SL* > hlld_eps)
  void HLLD_Flux(RS& s) const {
    double* UR1 = s.UR1; double* UL1 = s.UL1; double* FR1 = s.FR1; double* FL1 = s.FL1;
    const double SR = s.SR, SL = s.SL;
    if (SR < 0) {
      for (int n = 0; n < NE; ++n) { s.Fhat1[n] = FR1[n]; s.Ustar[n] = UR1[n]; }
      return;
    }
    if (SL > 0) {
      for (int n = 0; n < NE; ++n) { s.Fhat1[n] = FL1[n]; s.Ustar[n] = UL1[n]; }
      return;
    }
    double Ust[NE];
    for (int n = 0; n < NE; ++n) Ust[n] = (SR * UR1[n] - SL * UL1[n] + FL1[n] - FR1[n]) / (SR - SL);
    double rhoR = UR1[0], u1R = UR1[1] / rhoR, u2R = UR1[2] / rhoR, u3R = UR1[3] / rhoR, ER = UR1[4];
    double B1R = UR1[5], B2R = UR1[6], B3R = UR1[7];
    double rhoL = UL1[0], u1L = UL1[1] / rhoL, u2L = UL1[2] / rhoL, u3L = UL1[3] / rhoL, EL = UL1[4];
    double B1L = UL1[5], B2L = UL1[6], B3L = UL1[7];
    double Sstar = 0, uRbot = 0, uLbot = 0, BRbot = 0, BLbot = 0, Bstarbot = 0;
    if (s.direction == 1) {
      Sstar = Ust[1] / Ust[0]; uRbot = u1R; uLbot = u1L; BRbot = B1R; BLbot = B1L; Bstarbot = Ust[5];
    } else if (s.direction == 2) {
      Sstar = Ust[2] / Ust[0]; uRbot = u2R; uLbot = u2L; BRbot = B2R; BLbot = B2L; Bstarbot = Ust[6];
    }
    double rhoRstar = rhoR * (SR - uRbot) / (SR - Sstar);
    double rhoLstar = rhoL * (SL - uLbot) / (SL - Sstar);
    double SRstar = Sstar + std::sqrt(sq(Bstarbot) / rhoRstar);
    double SLstar = Sstar - std::sqrt(sq(Bstarbot) / rhoLstar);
    double PtotR = gamma1 * (ER - 0.5 * rhoR * (sq(u1R) + sq(u2R) + sq(u3R)));
    double PtotL = gamma1 * (EL - 0.5 * rhoL * (sq(u1L) + sq(u2L) + sq(u3L)));
    double PtotRstar = PtotR + rhoR * (SR - uRbot) * (Sstar - uRbot) + sq(Bstarbot) - sq(BRbot);
    double PtotLstar = PtotL + rhoL * (SL - uLbot) * (Sstar - uLbot) + sq(Bstarbot) - sq(BLbot);
    double AR = rhoR * sq(SR - uRbot) - Bstarbot * BRbot;
    double AL = rhoL * sq(SL - uLbot) - Bstarbot * BLbot;
    double CR = rhoR * (SR - uRbot) * (BRbot - Bstarbot);
    double CL = rhoL * (SL - uLbot) * (BLbot - Bstarbot);
    double DR = rhoR * (SR - uRbot) * (SR - Sstar) - sq(Bstarbot) + 1e-15;
    double DL = rhoL * (SL - uLbot) * (SL - Sstar) - sq(Bstarbot) + 1e-15;
    double B1Rstar, B1Lstar, B2Rstar, B2Lstar;
    if (s.direction == 1) {
      B1Rstar = Bstarbot; B1Lstar = Bstarbot;
      B2Rstar = (AR * B2R + CR * u2R) / DR;
      B2Lstar = (AL * B2L + CL * u2L) / DL;
    } else {
      B1Rstar = (AR * B1R + CR * u1R) / DR;
      B1Lstar = (AL * B1L + CL * u1L) / DL;
      B2Rstar = Bstarbot; B2Lstar = Bstarbot;
    }
    double B3Rstar = (AR * B3R + CR * u3R) / DR;
    double B3Lstar = (AL * B3L + CL * u3L) / DL;
    double URs[NE], ULs[NE];
    if (s.direction == 1) {
      URs[1] = (UR1[1] * (SR - uRbot) + PtotRstar - PtotR + BRbot * B1R - Bstarbot * B1Rstar) / (SR - Sstar);
      URs[2] = (UR1[2] * (SR - uRbot) + BRbot * B2R - Bstarbot * B2Rstar) / (SR - Sstar);
      ULs[1] = (UL1[1] * (SL - uLbot) + PtotLstar - PtotL + BLbot * B1L - Bstarbot * B1Lstar) / (SL - Sstar);
      ULs[2] = (UL1[2] * (SL - uLbot) + BLbot * B2L - Bstarbot * B2Lstar) / (SL - Sstar);
    } else {
      URs[1] = (UR1[1] * (SR - uRbot) + BRbot * B1R - Bstarbot * B1Rstar) / (SR - Sstar);
      URs[2] = (UR1[2] * (SR - uRbot) + PtotRstar - PtotR + BRbot * B2R - Bstarbot * B2Rstar) / (SR - Sstar);
      ULs[1] = (UL1[1] * (SL - uLbot) + BLbot * B1L - Bstarbot * B1Lstar) / (SL - Sstar);
      ULs[2] = (UL1[2] * (SL - uLbot) + PtotLstar - PtotL + BLbot * B2L - Bstarbot * B2Lstar) / (SL - Sstar);
    }
    URs[3] = (UR1[3] * (SR - uRbot) + BRbot * B3R - Bstarbot * B3Rstar) / (SR - Sstar);
    ULs[3] = (UL1[3] * (SL - uLbot) + BLbot * B3L - Bstarbot * B3Lstar) / (SL - Sstar);
    double u1Rstar = URs[1] / rhoRstar, u2Rstar = URs[2] / rhoRstar, u3Rstar = URs[3] / rhoRstar;
    double u1Lstar = ULs[1] / rhoLstar, u2Lstar = ULs[2] / rhoLstar, u3Lstar = ULs[3] / rhoLstar;
    double ERstar = ((SR - uRbot) * ER - PtotR * uRbot + PtotRstar * Sstar + BRbot * (u1R * B1R + u2R * B2R + u3R * B3R) -
                     Bstarbot * (u1Rstar * B1Rstar + u2Rstar * B2Rstar + u3Rstar * B3Rstar)) / (SR - Sstar);
    double ELstar = ((SL - uLbot) * EL - PtotL * uLbot + PtotLstar * Sstar + BLbot * (u1L * B1L + u2L * B2L + u3L * B3L) -
                     Bstarbot * (u1Lstar * B1Lstar + u2Lstar * B2Lstar + u3Lstar * B3Lstar)) / (SL - Sstar);
    URs[0] = rhoRstar; URs[4] = ERstar;
    ULs[0] = rhoLstar; ULs[4] = ELstar;
    for (int n = 5; n < 8; ++n) { URs[n] = Ust[n]; ULs[n] = Ust[n]; }
    const double eps = c.hlld_eps;
    if ((std::fabs(Bstarbot) > eps) && (SRstar - SLstar > eps)) {
      if (SLstar > 0) {
        for (int n = 0; n < NE; ++n) { s.Fhat1[n] = FL1[n] + SL * (ULs[n] - UL1[n]); s.Ustar[n] = ULs[n]; }
      } else if (SRstar < 0) {
        for (int n = 0; n < NE; ++n) { s.Fhat1[n] = FR1[n] + SR * (URs[n] - UR1[n]); s.Ustar[n] = URs[n]; }
      } else {
        // Stage 2 (HLLD_Flux.f90:134-176); FR1/FL1 are overwritten as in the reference
        for (int n = 0; n < NE; ++n) {
          FR1[n] = FR1[n] + SR * (URs[n] - UR1[n]);
          FL1[n] = FL1[n] + SL * (ULs[n] - UL1[n]);
        }
        double sL = std::sqrt(std::fabs(rhoLstar)), sR = std::sqrt(std::fabs(rhoRstar));
        double sg = sgn1(Bstarbot);
        double u1ss = (sL * u1Lstar + sR * u1Rstar + sg * (B1Rstar - B1Lstar)) / (sL + sR);
        double u2ss = (sL * u2Lstar + sR * u2Rstar + sg * (B2Rstar - B2Lstar)) / (sL + sR);
        double u3ss = (sL * u3Lstar + sR * u3Rstar + sg * (B3Rstar - B3Lstar)) / (sL + sR);
        double sLR = std::sqrt(std::fabs(rhoLstar * rhoRstar));
        double B1ss = (sL * B1Lstar + sR * B1Rstar + sg * sLR * (u1Rstar - u1Lstar)) / (sL + sR);
        double B2ss = (sL * B2Lstar + sR * B2Rstar + sg * sLR * (u2Rstar - u2Lstar)) / (sL + sR);
        double B3ss = (sL * B3Lstar + sR * B3Rstar + sg * sLR * (u3Rstar - u3Lstar)) / (sL + sR);
        double ERss = ERstar + sR * (u1Rstar * B1Rstar + u2Rstar * B2Rstar + u3Rstar * B3Rstar - u1ss * B1ss -
                                     u2ss * B2ss - u3ss * B3ss) * sg;
        double ELss = ELstar - sL * (u1Lstar * B1Lstar + u2Lstar * B2Lstar + u3Lstar * B3Lstar - u1ss * B1ss -
                                     u2ss * B2ss - u3ss * B3ss) * sg;
        double URss[NE] = {rhoRstar, rhoRstar * u1ss, rhoRstar * u2ss, rhoRstar * u3ss, ERss, B1ss, B2ss, B3ss};
        double ULss[NE] = {rhoLstar, rhoLstar * u1ss, rhoLstar * u2ss, rhoLstar * u3ss, ELss, B1ss, B2ss, B3ss};
        if (Sstar > 0) {
          for (int n = 0; n < NE; ++n) { s.Fhat1[n] = FL1[n] + SLstar * (ULss[n] - ULs[n]); s.Ustar[n] = ULss[n]; }
        } else {
          for (int n = 0; n < NE; ++n) { s.Fhat1[n] = FR1[n] + SRstar * (URss[n] - URs[n]); s.Ustar[n] = URss[n]; }
        }
      }
    } else {
      if (Sstar > 0) {
        for (int n = 0; n < NE; ++n) { s.Fhat1[n] = FL1[n] + SL * (ULs[n] - UL1[n]); s.Ustar[n] = ULs[n]; }
      } else {
        for (int n = 0; n < NE; ++n) { s.Fhat1[n] = FR1[n] + SR * (URs[n] - UR1[n]); s.Ustar[n] = URs[n]; }
      }
    }
  }

  void riemann1d(RS& s) const {
    switch (c.flux_type) {
      case 1: LF_Flux(s); break;
      case 2: HLL_Flux(s); break;
      case 3: HLLC_Flux(s); break;
      default: HLLD_Flux(s); break;
    }
  }

  // calculate_Ez.f90:5
  static double calculate_Ez(double u1, double u2, double B1, double B2) { return u2 * B1 - u1 * B2; }

  // LF_Flux_2D.f90:15-60
  double LF_Flux_2D(const double* URU1, const double* ULU1, const double* URD1, const double* ULD1) const {
    double ax = fmax4(std::fabs(URU1[1] / URU1[0]), std::fabs(ULU1[1] / ULU1[0]), std::fabs(URD1[1] / URD1[0]),
                      std::fabs(ULD1[1] / ULD1[0]));
    double ay = fmax4(std::fabs(URU1[2] / URU1[0]), std::fabs(ULU1[2] / ULU1[0]), std::fabs(URD1[2] / URD1[0]),
                      std::fabs(ULD1[2] / ULD1[0]));
    double EzRU = calculate_Ez(URU1[1] / URU1[0], URU1[2] / URU1[0], URU1[5], URU1[6]);
    double EzLU = calculate_Ez(ULU1[1] / ULU1[0], ULU1[2] / ULU1[0], ULU1[5], ULU1[6]);
    double EzRD = calculate_Ez(URD1[1] / URD1[0], URD1[2] / URD1[0], URD1[5], URD1[6]);
    double EzLD = calculate_Ez(ULD1[1] / ULD1[0], ULD1[2] / ULD1[0], ULD1[5], ULD1[6]);
    double B1RU = URU1[5], B1LU = ULU1[5], B1RD = URD1[5], B1LD = ULD1[5];
    double B2RU = URU1[6], B2LU = ULU1[6], B2RD = URD1[6], B2LD = ULD1[6];
    return 0.25 * (EzRU + EzLU + EzRD + EzLD) - 0.25 * ay * (0.5 * (B1RU + B1LU) - 0.5 * (B1RD + B1LD)) +
           0.25 * ax * (0.5 * (B2RU + B2RD) - 0.5 * (B2LU + B2LD));
  }

  // HLL_Flux_2D.f90:17-109. EzRU/EzLU/EzRD/EzLD are never assigned in the
  // reference (uninitialised locals at :8, used at :61-62); taken as 0.
  double HLL_Flux_2D(const double* URU1, const double* ULU1, const double* URD1, const double* ULD1) const {
    double axRU, bxRU, ayRU, byRU, axLU, bxLU, ayLU, byLU, axRD, bxRD, ayRD, byRD, axLD, bxLD, ayLD, byLD;
    eigenvalueMm(axRU, bxRU, URU1[0], URU1[1], URU1[2], URU1[3], URU1[4], URU1[5], URU1[6], URU1[7], 1, 0);
    eigenvalueMm(ayRU, byRU, URU1[0], URU1[1], URU1[2], URU1[3], URU1[4], URU1[5], URU1[6], URU1[7], 0, 1);
    eigenvalueMm(axLU, bxLU, ULU1[0], ULU1[1], ULU1[2], ULU1[3], ULU1[4], ULU1[5], ULU1[6], ULU1[7], 1, 0);
    eigenvalueMm(ayLU, byLU, ULU1[0], ULU1[1], ULU1[2], ULU1[3], ULU1[4], ULU1[5], ULU1[6], ULU1[7], 0, 1);
    eigenvalueMm(axRD, bxRD, URD1[0], URD1[1], URD1[2], URD1[3], URD1[4], URD1[5], URD1[6], URD1[7], 1, 0);
    eigenvalueMm(ayRD, byRD, URD1[0], URD1[1], URD1[2], URD1[3], URD1[4], URD1[5], URD1[6], URD1[7], 0, 1);
    eigenvalueMm(axLD, bxLD, ULD1[0], ULD1[1], ULD1[2], ULD1[3], ULD1[4], ULD1[5], ULD1[6], ULD1[7], 1, 0);
    eigenvalueMm(ayLD, byLD, ULD1[0], ULD1[1], ULD1[2], ULD1[3], ULD1[4], ULD1[5], ULD1[6], ULD1[7], 0, 1);
    double SR = fmax4(axRU, axLU, axRD, axLD);
    double SL = fmin4(bxRU, bxLU, bxRD, bxLD);
    double SU = fmax4(ayRU, ayLU, ayRD, ayLD);
    double SD = fmin4(byRU, byLU, byRD, byLD);
    double FxRU[NE], FyRU[NE], FxLU[NE], FyLU[NE], FxRD[NE], FyRD[NE], FxLD[NE], FyLD[NE];
    MHD_flux(URU1, FxRU, FyRU);
    MHD_flux(ULU1, FxLU, FyLU);
    MHD_flux(URD1, FxRD, FyRD);
    MHD_flux(ULD1, FxLD, FyLD);
    double BxRU = URU1[5], BxLU = ULU1[5], BxRD = URD1[5], BxLD = ULD1[5];
    double ByRU = URU1[6], ByLU = ULU1[6], ByRD = URD1[6], ByLD = ULD1[6];
    double UUs[NE], FUs[NE], UDs[NE], FDs[NE], URs[NE], FRs[NE], ULs[NE], FLs[NE];
    HLL1(URU1, ULU1, FxRU, FxLU, SR, SL, UUs, FUs);
    HLL1(URD1, ULD1, FxRD, FxLD, SR, SL, UDs, FDs);
    HLL1(URU1, URD1, FyRU, FyRD, SU, SD, URs, FRs);
    HLL1(ULU1, ULD1, FyLU, FyLD, SU, SD, ULs, FLs);
    double BxUstar = UUs[5], BxDstar = UDs[5], ByRstar = URs[6], ByLstar = ULs[6];
    double EzRstar = FRs[5], EzLstar = FLs[5], EzUstar = -FUs[6], EzDstar = -FDs[6];
    const double EzRU = 0, EzLU = 0, EzRD = 0, EzLD = 0;
    double BxSS = (2 * SR * SU * BxRU - 2 * SL * SU * BxLU + 2 * SL * SD * BxLD - 2 * SR * SD * BxRD - SR * (EzRU - EzRD) +
                   SL * (EzLU - EzLD) - (SR - SL) * (EzUstar - EzDstar)) / (2 * (SR - SL) * (SU - SD));
    double BySS = (2 * SR * SU * ByRU - 2 * SL * SU * ByLU + 2 * SL * SD * ByLD - 2 * SR * SD * ByRD + SU * (EzRU - EzLU) -
                   SD * (EzRD - EzLD) + (SU - SD) * (EzRstar - EzLstar)) / (2 * (SR - SL) * (SU - SD));
    double EzSS = 0.25 * (EzRstar + EzLstar + EzUstar + EzDstar) - 0.25 * SU * (BxUstar - BxSS) -
                  0.25 * SD * (BxDstar - BxSS) + 0.25 * SR * (ByRstar - BySS) + 0.25 * SL * (ByLstar - BySS);
    if (SL > 0) return EzLstar;
    if (SR < 0) return EzRstar;
    if (SD > 0) return EzDstar;
    if (SU < 0) return EzUstar;
    return EzSS;
  }

  // HLLD_Flux_2D.f90:17-114 and HLLC_Flux_2D.f90:17-114 (same structure;
  // Ez** is the plain average of the four star fluxes)
  double HLLDC_Flux_2D(const double* URU1, const double* ULU1, const double* URD1, const double* ULD1, bool hlld) const {
    double axRU, bxRU, ayRU, byRU, axLU, bxLU, ayLU, byLU, axRD, bxRD, ayRD, byRD, axLD, bxLD, ayLD, byLD;
    eigenvalueMm(axRU, bxRU, URU1[0], URU1[1], URU1[2], URU1[3], URU1[4], URU1[5], URU1[6], URU1[7], 1, 0);
    eigenvalueMm(ayRU, byRU, URU1[0], URU1[1], URU1[2], URU1[3], URU1[4], URU1[5], URU1[6], URU1[7], 0, 1);
    eigenvalueMm(axLU, bxLU, ULU1[0], ULU1[1], ULU1[2], ULU1[3], ULU1[4], ULU1[5], ULU1[6], ULU1[7], 1, 0);
    eigenvalueMm(ayLU, byLU, ULU1[0], ULU1[1], ULU1[2], ULU1[3], ULU1[4], ULU1[5], ULU1[6], ULU1[7], 0, 1);
    eigenvalueMm(axRD, bxRD, URD1[0], URD1[1], URD1[2], URD1[3], URD1[4], URD1[5], URD1[6], URD1[7], 1, 0);
    eigenvalueMm(ayRD, byRD, URD1[0], URD1[1], URD1[2], URD1[3], URD1[4], URD1[5], URD1[6], URD1[7], 0, 1);
    eigenvalueMm(axLD, bxLD, ULD1[0], ULD1[1], ULD1[2], ULD1[3], ULD1[4], ULD1[5], ULD1[6], ULD1[7], 1, 0);
    eigenvalueMm(ayLD, byLD, ULD1[0], ULD1[1], ULD1[2], ULD1[3], ULD1[4], ULD1[5], ULD1[6], ULD1[7], 0, 1);
    double SR = fmax4(axRU, axLU, axRD, axLD);
    double SL = fmin4(bxRU, bxLU, bxRD, bxLD);
    double SU = fmax4(ayRU, ayLU, ayRD, ayLD);
    double SD = fmin4(byRU, byLU, byRD, byLD);
    double FxRU[NE], FyRU[NE], FxLU[NE], FyLU[NE], FxRD[NE], FyRD[NE], FxLD[NE], FyLD[NE];
    MHD_flux(URU1, FxRU, FyRU);
    MHD_flux(ULU1, FxLU, FyLU);
    MHD_flux(URD1, FxRD, FyRD);
    MHD_flux(ULD1, FxLD, FyLD);
    RS s;
    double FUs[NE], FDs[NE], FRs[NE], FLs[NE];
    auto call = [&](const double* Ur, const double* Ul, const double* Fr, const double* Fl, double sr, double sl,
                    int dir, double* Fout) {
      for (int n = 0; n < NE; ++n) { s.UR1[n] = Ur[n]; s.UL1[n] = Ul[n]; s.FR1[n] = Fr[n]; s.FL1[n] = Fl[n]; }
      s.SR = sr; s.SL = sl; s.direction = dir;
      if (hlld) HLLD_Flux(s); else HLLC_Flux(s);
      for (int n = 0; n < NE; ++n) Fout[n] = s.Fhat1[n];
    };
    call(URU1, ULU1, FxRU, FxLU, SR, SL, 1, FUs);
    call(URD1, ULD1, FxRD, FxLD, SR, SL, 1, FDs);
    call(URU1, URD1, FyRU, FyRD, SU, SD, 2, FRs);
    call(ULU1, ULD1, FyLU, FyLD, SU, SD, 2, FLs);
    double EzRstar = FRs[5], EzLstar = FLs[5], EzUstar = -FUs[6], EzDstar = -FDs[6];
    double EzSS = 0.25 * (EzRstar + EzLstar + EzUstar + EzDstar);
    if (SL > 0) return EzLstar;
    if (SR < 0) return EzRstar;
    if (SD > 0) return EzDstar;
    if (SU < 0) return EzUstar;
    return EzSS;
  }

  double vertex_Ez(const double* URU1, const double* ULU1, const double* URD1, const double* ULD1) const {
    switch (c.flux_type) {
      case 1: return LF_Flux_2D(URU1, ULU1, URD1, ULD1);
      case 2: return HLL_Flux_2D(URU1, ULU1, URD1, ULD1);
      case 3: return HLLDC_Flux_2D(URU1, ULU1, URD1, ULD1, false);
      default: return HLLDC_Flux_2D(URU1, ULU1, URD1, ULD1, true);
    }
  }

  // ------------------------------------------------------------------ Lh --
  // Lh.f90:1-306. du is written for every cell (ghost entries 0). Face
  // traces and fluxes are recomputed per face point instead of stored in
  // whole-grid arrays; EzRL/EzUD of LhEz.f90:6-28 (which read Lh's trace
  // and flux arrays) are computed in the same face loops.
  void Lh(const double* uh, double* du) {
    const size_t usz = uhsize();
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < usz; ++q) du[q] = 0.0;
    auto live = [](int d, int n) {
      return d <= 6 || (n == 6 && (d == 7 || d == 9)) || (n == 7 && (d == 8 || d == 10));
    };
    // volume term, Lh.f90:11-68
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 1; j <= Ny; ++j)
      for (int i = 1; i <= Nx; ++i) {
        double uG[NG][NG][NE];
        for (int a = 0; a < NG; ++a)
          for (int b = 0; b < NG; ++b)
            for (int n = 0; n < NE; ++n) uG[a][b][n] = 0;
        for (int n = 1; n <= NE; ++n)
          for (int d = 1; d <= NP; ++d) {
            double ud = uh[U(i, j, d, n)];
            for (int b = 0; b < NG; ++b)
              for (int a = 0; a < NG; ++a) uG[a][b][n - 1] = uG[a][b][n - 1] + ud * phiG[a][b][d - 1];
          }
        double Fx[NG][NG][NE], Fy[NG][NG][NE];
        for (int a = 0; a < NG; ++a)
          for (int b = 0; b < NG; ++b) {
            double rho = uG[a][b][0];
            double u = uG[a][b][1] / rho, v = uG[a][b][2] / rho, w = uG[a][b][3] / rho;
            double E = uG[a][b][4], B1 = uG[a][b][5], B2 = uG[a][b][6], B3 = uG[a][b][7];
            double p = gamma1 * (E - 0.5 * rho * (sq(u) + sq(v) + sq(w)) - 0.5 * (sq(B1) + sq(B2) + sq(B3)));
            double S = p + 0.5 * (sq(B1) + sq(B2) + sq(B3));
            double T = E + S;
            double K = u * B1 + v * B2 + w * B3;
            double* fx = Fx[a][b];
            double* fy = Fy[a][b];
            fx[0] = uG[a][b][1];
            fx[1] = rho * sq(u) + S - sq(B1);
            fx[2] = rho * u * v - B1 * B2;
            fx[3] = rho * u * w - B1 * B3;
            fx[4] = T * u - K * B1;
            fx[5] = 0;
            fx[6] = u * B2 - v * B1;
            fx[7] = u * B3 - w * B1;
            fy[0] = uG[a][b][2];
            fy[1] = rho * u * v - B1 * B2;
            fy[2] = rho * sq(v) + S - sq(B2);
            fy[3] = rho * v * w - B2 * B3;
            fy[4] = T * v - K * B2;
            fy[5] = v * B1 - u * B2;
            fy[6] = 0;
            fy[7] = v * B3 - w * B2;
          }
        for (int d = 2; d <= NP; ++d)
          for (int n = 1; n <= NE; ++n) {
            if (!live(d, n)) continue;
            double acc = du[U(i, j, d, n)];
            for (int a = 0; a < NG; ++a)
              for (int b = 0; b < NG; ++b)
                acc = acc + 0.25 * weight[a] * weight[b] *
                                (Fx[a][b][n - 1] * phixG[a][b][d - 1] + Fy[a][b][n - 1] * phiyG[a][b][d - 1]);
            du[U(i, j, d, n)] = acc;
          }
      }

    // x faces: traces (Lh.f90:72-86), fluxes (:88-136), Riemann (:206-234),
    // and LhEz face Ez (LhEz.f90:6-16)
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 1; j <= Ny; ++j)
      for (int i = 0; i <= Nx; ++i)
        for (int g = 0; g < NG; ++g) {
          double URv[NE], ULv[NE], FRv[NE], FLv[NE];
          for (int n = 1; n <= NE; ++n) {
            double a = 0, b = 0;
            for (int d = 1; d <= NP; ++d) {
              a = a + uh[U(i, j, d, n)] * phiGR[g][d - 1];
              b = b + uh[U(i + 1, j, d, n)] * phiGL[g][d - 1];
            }
            URv[n - 1] = a;
            ULv[n - 1] = b;
          }
          point_flux(URv, FRv, 0, false, false);
          point_flux(ULv, FLv, 0, false, true);
          double SRmax, SRmin, SLmax, SLmin;
          eigenvalueMm(SRmax, SRmin, URv[0], URv[1], URv[2], URv[3], URv[4], URv[5], URv[6], URv[7], 1, 0);
          eigenvalueMm(SLmax, SLmin, ULv[0], ULv[1], ULv[2], ULv[3], ULv[4], ULv[5], ULv[6], ULv[7], 1, 0);
          RS s;
          s.SR = fmax2(SRmax, SLmax);
          s.SL = fmin2(SRmin, SLmin);
          s.direction = 1;
          for (int n = 0; n < NE; ++n) { s.FR1[n] = FLv[n]; s.FL1[n] = FRv[n]; s.UR1[n] = ULv[n]; s.UL1[n] = URv[n]; }
          riemann1d(s);
          for (int n = 1; n <= NE; ++n) Fxhat[FX(i, j, g, n)] = s.Fhat1[n - 1];
          if (c.ez_face_fhat) {
            EzRL[EX(i, j, g)] = -s.Fhat1[6];
          } else {
            double a = URv[1] / URv[0];
            double b = ULv[1] / ULv[0];
            double S = fmax2(std::fabs(a), std::fabs(b));
            EzRL[EX(i, j, g)] = -0.5 * (FRv[6] + FLv[6] - S * (ULv[6] - URv[6]));
          }
        }

    // y faces (Lh.f90:139-203, :237-264; LhEz.f90:18-28)
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 0; j <= Ny; ++j)
      for (int i = 1; i <= Nx; ++i)
        for (int g = 0; g < NG; ++g) {
          double UUv[NE], UDv[NE], FUv[NE], FDv[NE];
          for (int n = 1; n <= NE; ++n) {
            double a = 0, b = 0;
            for (int d = 1; d <= NP; ++d) {
              a = a + uh[U(i, j, d, n)] * phiGU[g][d - 1];
              b = b + uh[U(i, j + 1, d, n)] * phiGD[g][d - 1];
            }
            UUv[n - 1] = a;
            UDv[n - 1] = b;
          }
          point_flux(UUv, FUv, 1, false, false);
          point_flux(UDv, FDv, 1, true, false);
          double SRmax, SRmin, SLmax, SLmin;
          eigenvalueMm(SRmax, SRmin, UUv[0], UUv[1], UUv[2], UUv[3], UUv[4], UUv[5], UUv[6], UUv[7], 0, 1);
          eigenvalueMm(SLmax, SLmin, UDv[0], UDv[1], UDv[2], UDv[3], UDv[4], UDv[5], UDv[6], UDv[7], 0, 1);
          RS s;
          s.SR = fmax2(SRmax, SLmax);
          s.SL = fmin2(SRmin, SLmin);
          s.direction = 2;
          for (int n = 0; n < NE; ++n) { s.FR1[n] = FDv[n]; s.FL1[n] = FUv[n]; s.UR1[n] = UDv[n]; s.UL1[n] = UUv[n]; }
          riemann1d(s);
          for (int n = 1; n <= NE; ++n) Fyhat[FY(i, j, g, n)] = s.Fhat1[n - 1];
          if (c.ez_face_fhat) {
            EzUD[EY(i, j, g)] = s.Fhat1[5];
          } else {
            double a = UUv[2] / UUv[0];
            double b = UDv[2] / UDv[0];
            double S = fmax2(std::fabs(a), std::fabs(b));
            EzUD[EY(i, j, g)] = 0.5 * (FUv[5] + FDv[5] - S * (UDv[5] - UUv[5]));
          }
        }

    // surface integrals in the serial order (Lh.f90:268-298), then mass
    // matrix (:302-304)
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 1; j <= Ny; ++j)
      for (int i = 1; i <= Nx; ++i)
        for (int d = 1; d <= NP; ++d)
          for (int n = 1; n <= NE; ++n) {
            if (!live(d, n)) continue;
            double acc = du[U(i, j, d, n)];
            for (int g = 0; g < NG; ++g)
              acc = acc - (0.5 / hx) * weight[g] *
                              (Fxhat[FX(i, j, g, n)] * phiGR[g][d - 1] - Fxhat[FX(i - 1, j, g, n)] * phiGL[g][d - 1]);
            for (int g = 0; g < NG; ++g)
              acc = acc - (0.5 / hy) * weight[g] *
                              (Fyhat[FY(i, j, g, n)] * phiGU[g][d - 1] - Fyhat[FY(i, j - 1, g, n)] * phiGD[g][d - 1]);
            du[U(i, j, d, n)] = acc / mm[d - 1];
          }
  }

  // ---------------------------------------------------------------- LhEz --
  // LhEz.f90:34-96 (EzRL/EzUD were filled by Lh from the same uh)
  void LhEz(const double* uh, double* dez1, double* dez2) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 0; j <= Ny + 1; ++j)
      for (int i = 0; i <= Nx + 1; ++i)
        for (int n = 1; n <= NE; ++n) {
          double ru = 0, lu = 0, rd = 0, ld = 0;
          for (int d = 1; d <= NP; ++d) {
            double v = uh[U(i, j, d, n)];
            ru = ru + v * phiRU[d - 1];
            lu = lu + v * phiLU[d - 1];
            rd = rd + v * phiRD[d - 1];
            ld = ld + v * phiLD[d - 1];
          }
          cornRU[CN(i, j) + n - 1] = ru;
          cornLU[CN(i, j) + n - 1] = lu;
          cornRD[CN(i, j) + n - 1] = rd;
          cornLD[CN(i, j) + n - 1] = ld;
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 0; j <= Ny; ++j)
      for (int i = 0; i <= Nx; ++i) {
        const double* URU1 = &cornLD[CN(i + 1, j + 1)];
        const double* ULU1 = &cornRD[CN(i, j + 1)];
        const double* URD1 = &cornLU[CN(i + 1, j)];
        const double* ULD1 = &cornRU[CN(i, j)];
        EzV[VX(i, j)] = vertex_Ez(URU1, ULU1, URD1, ULD1);
      }
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 1; j <= Ny; ++j)
      for (int i = 0; i <= Nx; ++i)
        for (int d = 1; d <= 3; ++d) {
          double acc = 0;
          for (int g = 0; g < NG; ++g) acc = acc + 0.5 * weight[g] * EzRL[EX(i, j, g)] * EzyG[g][d - 1];
          dez1[BXi(i, j, d)] = (acc - EzV[VX(i, j)] * EzU[d - 1] / hy + EzV[VX(i, j - 1)] * EzD[d - 1] / hy) / mmE[d - 1];
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 0; j <= Ny; ++j)
      for (int i = 1; i <= Nx; ++i)
        for (int d = 1; d <= 3; ++d) {
          double acc = 0;
          for (int g = 0; g < NG; ++g) acc = acc - 0.5 * weight[g] * EzUD[EY(i, j, g)] * EzxG[g][d - 1];
          dez2[BYi(i, j, d)] = (acc + EzV[VX(i, j)] * EzR[d - 1] / hx - EzV[VX(i - 1, j)] * EzL[d - 1] / hx) / mmE[d - 1];
        }
  }

  // ---------------------------------------------------------- eigenmatrix --
  // eigenmatrix.f90:1-407 with compute_t_vector/compute_cross/pick_orthogonal
  // (:411-469). gamma is the hard-coded 5/3 (quirk Q1). evr/evl column-major
  // evr[(r-1) + 8*(c-1)].
  static void compute_cross(double a1, double a2, double a3, double b1, double b2, double b3, double& c1, double& c2,
                            double& c3) {
    c1 = a2 * b3 - a3 * b2;
    c2 = a3 * b1 - a1 * b3;
    c3 = a1 * b2 - a2 * b1;
  }
  static void pick_orthogonal(double v1, double v2, double v3, double& r1, double& r2, double& r3) {
    if (std::fabs(v1) >= std::fabs(v2) && std::fabs(v1) >= std::fabs(v3)) {
      r2 = 1.0; r3 = 1.0; r1 = (-v2 - v3) / v1;
    } else if (std::fabs(v2) >= std::fabs(v1) && std::fabs(v2) >= std::fabs(v3)) {
      r1 = 1.0; r3 = 1.0; r2 = (-v1 - v3) / v2;
    } else if (std::fabs(v3) >= std::fabs(v1) && std::fabs(v3) >= std::fabs(v1)) {
      r1 = 1.0; r2 = 1.0; r3 = (-v1 - v2) / v3;
    }
  }
  static void compute_t_vector(double n1, double n2, double n3, double B1, double B2, double B3, double& t1,
                               double& t2, double& t3) {
    const double eps = 1e-7;
    double nB1, nB2, nB3, tp1 = 0, tp2 = 0, tp3 = 0;
    compute_cross(n1, n2, n3, B1, B2, B3, nB1, nB2, nB3);
    if (sq(nB1) + sq(nB2) + sq(nB3) < eps)
      pick_orthogonal(n1, n2, n3, tp1, tp2, tp3);
    else
      compute_cross(nB1, nB2, nB3, n1, n2, n3, tp1, tp2, tp3);
    double tpnorm = std::sqrt(sq(tp1) + sq(tp2) + sq(tp3));
    t1 = tp1 / tpnorm;
    t2 = tp2 / tpnorm;
    t3 = tp3 / tpnorm;
  }

  void eigenmatrix(double* evr, double* evl, double rho, double u1, double u2, double u3, double E, double B1,
                   double B2, double B3, double n1, double n2, double n3) const {
    const double gm = gflux;
    double ru[8][8], lu[8][8];  // ru[r][c] = ru(r+1,c+1)
    double p;
    if (c.eig_p_typo)
      p = (gm - 1.0) * (E - 0.5 * (sq(u1) + sq(u2) + sq(u3)) - 0.5 * (sq(B1) + sq(B2) + sq(B3)));
    else
      p = (gm - 1.0) * (E - 0.5 * rho * (sq(u1) + sq(u2) + sq(u3)) - 0.5 * (sq(B1) + sq(B2) + sq(B3)));
    double t1, t2, t3;
    compute_t_vector(n1, n2, n3, B1, B2, B3, t1, t2, t3);
    double rhosq = std::sqrt(std::fabs(rho));
    double g1 = gm - 1.0;
    double a2 = std::fabs(gm * p / rho);
    double a = std::sqrt(a2);
    double sqg2 = std::sqrt(1.0 / (2.0 * gm));
    double sq12 = std::sqrt(0.5);
    double sqpr = std::sqrt(std::fabs(p)) / rho;
    double sqpor = std::sqrt(std::fabs(p / rho));
    double sq1og = std::sqrt(1.0 / gm);
    double b1s = B1 / rhosq, b2s = B2 / rhosq, b3s = B3 / rhosq;
    double bN = b1s * n1 + b2s * n2 + b3s * n3;
    double d = a2 + (sq(b1s) + sq(b2s) + sq(b3s));
    double cf = std::sqrt(0.5 * std::fabs(d + std::sqrt(std::fabs(sq(d) - 4.0 * a2 * sq(bN)))));
    double cs = std::sqrt(0.5 * std::fabs(d - std::sqrt(std::fabs(sq(d) - 4.0 * a2 * sq(bN)))));
    double beta1 = sgn1((b1s * n1 + b2s * n2 + b3s * n3) * 1.0);
    double alphaf, alphas;
    if (std::fabs(cf * cf - cs * cs) <= 1.0e-12) {
      alphaf = SIN_ATAN1;
      alphas = COS_ATAN1;
    } else {
      alphaf = std::sqrt(std::fabs(a2 - cs * cs)) / std::sqrt(std::fabs(cf * cf - cs * cs));
      alphas = std::sqrt(std::fabs(cf * cf - a2)) / std::sqrt(std::fabs(cf * cf - cs * cs));
    }
    double TxN1 = n3 * t2 - n2 * t3;
    double TxN2 = n1 * t3 - n3 * t1;
    double TxN3 = n2 * t1 - n1 * t2;
    for (int r = 0; r < 8; ++r)
      for (int cc = 0; cc < 8; ++cc) ru[r][cc] = 0.0;
    ru[0][0] = std::sqrt(g1 / gm) * rhosq;
    ru[5][1] = sq1og * a * n1;
    ru[6][1] = sq1og * a * n2;
    ru[7][1] = sq1og * a * n3;
    ru[0][2] = 0.0;
    ru[1][2] = -sq12 * (sqpr * (TxN1));
    ru[2][2] = -sq12 * (sqpr * (TxN2));
    ru[3][2] = -sq12 * (sqpr * (TxN3));
    ru[4][2] = 0.0;
    ru[5][2] = sq12 * sqpor * (TxN1);
    ru[6][2] = sq12 * sqpor * (TxN2);
    ru[7][2] = sq12 * sqpor * (TxN3);
    ru[0][3] = ru[0][2];
    ru[1][3] = -ru[1][2];
    ru[2][3] = -ru[2][2];
    ru[3][3] = -ru[3][2];
    ru[4][3] = ru[4][2];
    ru[5][3] = ru[5][2];
    ru[6][3] = ru[6][2];
    ru[7][3] = ru[7][2];
    double bst = (b1s * t1 + b2s * t2 + b3s * t3);
    ru[0][4] = sqg2 * alphaf * rhosq;
    ru[1][4] = sqg2 * ((alphaf * a2 * n1 + alphas * a * ((bst)*n1 - (bN)*t1))) / (rhosq * cf);
    ru[2][4] = sqg2 * ((alphaf * a2 * n2 + alphas * a * ((bst)*n2 - (bN)*t2))) / (rhosq * cf);
    ru[3][4] = sqg2 * ((alphaf * a2 * n3 + alphas * a * ((bst)*n3 - (bN)*t3))) / (rhosq * cf);
    ru[4][4] = sqg2 * alphaf * rhosq * a2;
    ru[5][4] = sqg2 * alphas * a * t1;
    ru[6][4] = sqg2 * alphas * a * t2;
    ru[7][4] = sqg2 * alphas * a * t3;
    ru[0][5] = ru[0][4];
    ru[1][5] = -ru[1][4];
    ru[2][5] = -ru[2][4];
    ru[3][5] = -ru[3][4];
    ru[4][5] = ru[4][4];
    ru[5][5] = ru[5][4];
    ru[6][5] = ru[6][4];
    ru[7][5] = ru[7][4];
    ru[0][6] = sqg2 * alphas * rhosq;
    ru[1][6] = beta1 * sqg2 * (alphaf * sq(cf) * t1 + a * n1 * alphas * (bN)) / (rhosq * cf);
    ru[2][6] = beta1 * sqg2 * (alphaf * sq(cf) * t2 + alphas * a * (bN)*n2) / (rhosq * cf);
    ru[3][6] = beta1 * sqg2 * (alphaf * sq(cf) * t3 + alphas * a * (bN)*n3) / (rhosq * cf);
    ru[4][6] = sq(a) * sqg2 * alphas * rhosq;
    ru[5][6] = -sqg2 * alphaf * a * t1;
    ru[6][6] = -sqg2 * alphaf * a * t2;
    ru[7][6] = -sqg2 * alphaf * a * t3;
    ru[0][7] = ru[0][6];
    ru[1][7] = -ru[1][6];
    ru[2][7] = -ru[2][6];
    ru[3][7] = -ru[3][6];
    ru[4][7] = ru[4][6];
    ru[5][7] = ru[5][6];
    ru[6][7] = ru[6][6];
    ru[7][7] = ru[7][6];
    for (int m = 0; m < 8; ++m) {
      evr[0 + 8 * m] = ru[0][m] / g1;
      evr[1 + 8 * m] = (ru[0][m] * u1 + ru[1][m] * rho) / g1;
      evr[2 + 8 * m] = (ru[0][m] * u2 + ru[2][m] * rho) / g1;
      evr[3 + 8 * m] = (ru[0][m] * u3 + ru[3][m] * rho) / g1;
      evr[4 + 8 * m] = (ru[4][m] / g1 + B1 * ru[5][m] + B2 * ru[6][m] + B3 * ru[7][m] +
                        0.5 * ru[0][m] * (sq(u1) + sq(u2) + sq(u3)) + ru[1][m] * u1 * rho + ru[2][m] * u2 * rho +
                        ru[3][m] * u3 * rho) / g1;
      evr[5 + 8 * m] = ru[5][m] / g1;
      evr[6 + 8 * m] = ru[6][m] / g1;
      evr[7 + 8 * m] = ru[7][m] / g1;
    }

    // left eigenvectors (eigenmatrix.f90:185-394)
    compute_t_vector(n1, n2, n3, B1, B2, B3, t1, t2, t3);
    rhosq = std::sqrt(rho);
    g1 = gm - 1.0;
    a2 = std::fabs(gm * p / rho);
    a = std::sqrt(a2);
    b1s = B1 / rhosq; b2s = B2 / rhosq; b3s = B3 / rhosq;
    double BNs = b1s * n1 + b2s * n2 + b3s * n3;
    double BN = (B1 * n1 + B2 * n2 + B3 * n3);
    d = a2 + (sq(b1s) + sq(b2s) + sq(b3s));
    cf = std::sqrt(0.5 * std::fabs(d + std::sqrt(std::fabs(sq(d) - 4.0 * a2 * sq(BNs)))));
    cs = std::sqrt(0.5 * std::fabs(d - std::sqrt(std::fabs(sq(d) - 4.0 * a2 * sq(BNs)))));
    if (std::fabs(cf * cf - cs * cs) <= 1.0e-12) {
      alphaf = SIN_ATAN1;
      alphas = COS_ATAN1;
    } else {
      alphaf = std::sqrt(std::fabs(a2 - cs * cs)) / std::sqrt(std::fabs(cf * cf - cs * cs));
      alphas = std::sqrt(std::fabs(cf * cf - a2)) / std::sqrt(std::fabs(cf * cf - cs * cs));
    }
    double twosq = std::sqrt(2.0);
    beta1 = sgn1((BNs)*1.0);
    double sqgam = std::sqrt(g1 / gm);
    TxN1 = n3 * t2 - n2 * t3;
    TxN2 = n1 * t3 - n3 * t1;
    TxN3 = n2 * t1 - n1 * t2;
    double BT = (B1 * t1 + B2 * t2 + B3 * t3);
    double gu1sq = std::sqrt(1.0 / gm);
    for (int r = 0; r < 8; ++r)
      for (int cc = 0; cc < 8; ++cc) lu[r][cc] = 0.0;
    lu[0][0] = 1.0 / (sqgam * rhosq);
    lu[0][4] = -1.0 / (a2 * sqgam * rhosq);
    double nen = (sq(n3) * (sq(t1) + sq(t2)) - 2.0 * n1 * n3 * t1 * t3 - 2.0 * n2 * t2 * (n1 * t1 + n3 * t3) +
                  sq(n2) * (sq(t1) + sq(t3)) + sq(n1) * (sq(t2) + sq(t3)));
    double nen2 = a * gu1sq * nen;
    lu[1][5] = (-n2 * t1 * t2 - n3 * t1 * t3 + n1 * (sq(t2) + sq(t3))) / nen2;
    lu[1][6] = (-t2 * (n1 * t1 + n3 * t3) + n2 * (sq(t1) + sq(t3))) / nen2;
    lu[1][7] = (n3 * (sq(t1) + sq(t2)) - (n1 * t1 + n2 * t2) * t3) / nen2;
    double nen3 = std::sqrt(2.0) * std::sqrt(std::fabs(p)) * nen;
    double nen31 = nen3 / std::sqrt(std::fabs(rho));
    lu[2][1] = rho * (-TxN1) / nen3;
    lu[2][2] = rho * (-TxN2) / nen3;
    lu[2][3] = rho * (-TxN3) / nen3;
    lu[2][5] = TxN1 / nen31;
    lu[2][6] = TxN2 / nen31;
    lu[2][7] = TxN3 / nen31;
    lu[3][0] = lu[2][0];
    lu[3][1] = -lu[2][1];
    lu[3][2] = -lu[2][2];
    lu[3][3] = -lu[2][3];
    lu[3][4] = lu[2][4];
    lu[3][5] = lu[2][5];
    lu[3][6] = lu[2][6];
    lu[3][7] = lu[2][7];
    double Term51 = rho * cf *
                    ((n2 * t1 * t2 + n3 * t1 * t3 - n1 * (sq(t2) + sq(t3))) * rhosq * sq(cf) * alphaf -
                     a * BN * alphas * (-sq(n2) * t1 + n1 * n2 * t2 + n3 * TxN2));
    double Term52 = rho * cf *
                    ((-t2 * (n1 * t1 + n3 * t3) + n2 * (sq(t1) + sq(t3))) * rhosq * sq(cf) * alphaf -
                     a * BN * alphas * (-n1 * n2 * t1 + sq(n1) * t2 + n3 * TxN1));
    double Term53 = rho * cf *
                    ((n3 * (sq(t1) + sq(t2)) - (n1 * t1 + n2 * t2) * t3) * rhosq * sq(cf) * alphaf -
                     a * (-n1 * n3 * t1 + sq(n1) * t3 + n2 * (-n3 * t2 + n2 * t3)) * BN * alphas);
    double Term54 = alphaf / (twosq * sq(a) * gu1sq * rhosq * (sq(alphaf) + sq(alphas)));
    double Term55 = (sq(n2) * t1 - n1 * n2 * t2 + n3 * (n3 * t1 - n1 * t3)) * alphas;
    double Term56 = alphas * (-n1 * n2 * t1 + sq(n1) * t2 + n3 * TxN1);
    double Term57 = (-n1 * n3 * t1 + sq(n1) * t3 + n2 * (-n3 * t2 + n2 * t3)) * alphas;
    double nen51 = twosq * a * nen * gu1sq *
                   (a * sq(BN) * sq(alphas) + rhosq * sq(cf) * alphaf * (a * rhosq * alphaf + BT * alphas));
    double nen52 = twosq * a * gu1sq * (sq(alphaf) + sq(alphas)) * nen;
    lu[4][0] = 0.0;
    lu[4][1] = -Term51 / nen51;
    lu[4][2] = Term52 / nen51;
    lu[4][3] = Term53 / nen51;
    lu[4][4] = Term54;
    lu[4][5] = Term55 / nen52;
    lu[4][6] = Term56 / nen52;
    lu[4][7] = Term57 / nen52;
    lu[5][0] = lu[4][0];
    lu[5][1] = -lu[4][1];
    lu[5][2] = -lu[4][2];
    lu[5][3] = -lu[4][3];
    lu[5][4] = lu[4][4];
    lu[5][5] = lu[4][5];
    lu[5][6] = lu[4][6];
    lu[5][7] = lu[4][7];
    double Term71 =
        rho * cf *
        (a * (sq(n2) * t1 - n1 * n2 * t2 + n3 * (n3 * t1 - n1 * t3)) * rhosq * alphaf +
         ((B3 * n2 * t1 - B2 * n3 * t1 - B3 * n1 * t2 + B2 * n1 * t3) * (-n3 * t2 + n2 * t3) +
          B1 * (sq(n2) * sq(t1) + sq(n3) * sq(t1) - 2.0 * n1 * n2 * t1 * t2 - 2.0 * n1 * n3 * t1 * t3 +
                sq(n1) * (sq(t2) + sq(t3)))) *
             alphas);
    double Term72 =
        rho * cf *
        (((n3 * t1 - n1 * t3) * (B3 * n2 * t1 - B3 * n1 * t2 + B1 * n3 * t2 - B1 * n2 * t3) +
          B2 * ((sq(n1) + sq(n3)) * sq(t2) - 2.0 * n2 * t2 * (n1 * t1 + n3 * t3) + sq(n2) * (sq(t1) + sq(t3)))) *
             alphas +
         a * rhosq * alphaf * (-n1 * n2 * t1 + sq(n1) * t2 + n3 * TxN1));
    double Term73 =
        rho * cf *
        (a * (-n1 * n3 * t1 + sq(n1) * t3 + n2 * (-n3 * t2 + n2 * t3)) * rhosq * alphaf +
         alphas * (B3 * (sq(n3) * (sq(t1) + sq(t2)) - 2.0 * n3 * (n1 * t1 + n2 * t2) * t3 + (sq(n1) + sq(n2)) * sq(t3)) +
                   B2 * (n3 * t1 - n1 * t3) * TxN3 + B1 * (-n3 * t2 + n2 * t3) * TxN3));
    double Term74 = alphas / (twosq * sq(a) * gu1sq * rhosq * (sq(alphaf) + sq(alphas)));
    double Term75 = -alphaf * (sq(n2) * t1 - n1 * n2 * t2 + n3 * (n3 * t1 - n1 * t3));
    double Term76 = -alphaf * (-n1 * n2 * t1 + sq(n1) * t2 + n3 * TxN1);
    double Term77 = -alphaf * (-n1 * n3 * t1 + sq(n1) * t3 + n2 * (-n3 * t2 + n2 * t3));
    double nen71 = twosq * beta1 * nen * gu1sq *
                   (a * sq(BN) * sq(alphas) + rhosq * sq(cf) * alphaf * (a * rhosq * alphaf + BT * alphas));
    double nen72 = nen52;
    lu[6][0] = 0.0;
    lu[6][1] = Term71 / nen71;
    lu[6][2] = Term72 / nen71;
    lu[6][3] = Term73 / nen71;
    lu[6][4] = Term74;
    lu[6][5] = Term75 / nen72;
    lu[6][6] = Term76 / nen72;
    lu[6][7] = Term77 / nen72;
    lu[7][0] = lu[6][0];
    lu[7][1] = -lu[6][1];
    lu[7][2] = -lu[6][2];
    lu[7][3] = -lu[6][3];
    lu[7][4] = lu[6][4];
    lu[7][5] = lu[6][5];
    lu[7][6] = lu[6][6];
    lu[7][7] = lu[6][7];
    for (int m = 0; m < 8; ++m) {
      const double* l = lu[m];
      evl[m + 8 * 0] = l[0] * g1 - l[1] * u1 * g1 / rho - l[2] * u2 * g1 / rho - l[3] * u3 * g1 / rho +
                       l[4] * sq(g1) * (sq(u1) + sq(u2) + sq(u3)) * .5;
      evl[m + 8 * 1] = -l[4] * u1 * sq(g1) + l[1] * g1 / rho;
      evl[m + 8 * 2] = -l[4] * u2 * sq(g1) + l[2] * g1 / rho;
      evl[m + 8 * 3] = -l[4] * u3 * sq(g1) + l[3] * g1 / rho;
      evl[m + 8 * 4] = l[4] * sq(g1);
      evl[m + 8 * 5] = l[5] * g1 - B1 * l[4] * sq(g1);
      evl[m + 8 * 6] = l[6] * g1 - B2 * l[4] * sq(g1);
      evl[m + 8 * 7] = l[7] * g1 - B3 * l[4] * sq(g1);
    }
    if (c.eig_identity) {
      double sr = 0, sl = 0;
      for (int q = 0; q < 64; ++q) sr = sr + std::fabs(evr[q]);
      for (int q = 0; q < 64; ++q) sl = sl + std::fabs(evl[q]);
      if (sr > 1e4 || sl > 1e4) {
        for (int q = 0; q < 64; ++q) { evl[q] = 0; evr[q] = 0; }
        for (int q = 0; q < 8; ++q) { evl[q + 8 * q] = 1; evr[q + 8 * q] = 1; }
      }
    }
  }

  // matmul(A, x) for an 8x8 column-major A, summed from zero in k order
  static void matvec(const double* A, const double* x, double* y) {
    for (int r = 0; r < 8; ++r) {
      double acc = 0;
      for (int k = 0; k < 8; ++k) acc = acc + A[r + 8 * k] * x[k];
      y[r] = acc;
    }
  }

  // minmod.f90:5-27 (TVB: keep a if |a| <= M h^2)
  static void minmod(const double* DU, const double* DR, const double* DL, double M, double hd, double* out) {
    for (int i = 0; i < 8; ++i) {
      if (std::fabs(DU[i]) <= M * sq(hd)) {
        out[i] = DU[i];
      } else {
        double a = sgn1(DU[i]), b = sgn1(DR[i]), cc = sgn1(DL[i]);
        double s = (a + b + cc) / 3.0;
        if (std::fabs(s) == 1)
          out[i] = s * fmin2(fmin2(std::fabs(DU[i]), std::fabs(DR[i])), std::fabs(DL[i]));
        else
          out[i] = 0;
      }
    }
  }

  // minmodB.f90:5-21
  static double minmodB(double a, double b, double cc, double M, double hd) {
    if (std::fabs(a) <= M * sq(hd)) return a;
    double as = sgn1(a), bs = sgn1(b), cs = sgn1(cc);
    double s = (as + bs + cs) / 3.0;
    if (std::fabs(s) == 1) return s * fmin2(fmin2(std::fabs(a), std::fabs(b)), std::fabs(cc));
    return 0;
  }

  // pressure.f90:1-8
  static double pressure(double rho, double rhou, double rhov, double rhow, double E, double B1, double B2, double B3,
                         double g) {
    return (g - 1) * (E - 0.5 * (sq(rhou) + sq(rhov) + sq(rhow)) / rho - 0.5 * (sq(B1) + sq(B2) + sq(B3)));
  }

  // ------------------------------------------------------- KXRCF detector --
  // KXRCF_Detector.f90:1-109. Ck and stickiness are configuration.
  void kxrcf(const double* uh) {
    const double P = std::pow(hx * hy, 0.25 * (2 + 1));
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 1; j <= Ny; ++j)
      for (int i = 1; i <= Nx; ++i) {
        auto trace = [&](int ci, int cj, const double (*phi)[NP], int g, double* out) {
          for (int n = 1; n <= NE; ++n) {
            double a = 0;
            for (int d = 1; d <= NP; ++d) a = a + uh[U(ci, cj, d, n)] * phi[g][d - 1];
            out[n - 1] = a;
          }
        };
        double Iij[NE] = {0, 0, 0, 0, 0, 0, 0, 0};
        double Lij = 1e-12;
        double A[NE], B[NE];
        if (uh[U(i + 1, j, 1, 2)] < 0) {
          for (int g = 0; g < NG; ++g) {
            trace(i, j, phiGR, g, A);
            trace(i + 1, j, phiGL, g, B);
            for (int n = 0; n < NE; ++n) Iij[n] = Iij[n] + hy1 * weight[g] * (A[n] - B[n]);
            Lij = Lij + hy;
          }
        }
        if (uh[U(i - 1, j, 1, 2)] > 0) {
          for (int g = 0; g < NG; ++g) {
            trace(i, j, phiGL, g, A);
            trace(i - 1, j, phiGR, g, B);
            for (int n = 0; n < NE; ++n) Iij[n] = Iij[n] + hy1 * weight[g] * (A[n] - B[n]);
            Lij = Lij + hy;
          }
        }
        if (uh[U(i, j + 1, 1, 3)] < 0) {
          for (int g = 0; g < NG; ++g) {
            trace(i, j, phiGU, g, A);
            trace(i, j + 1, phiGD, g, B);
            for (int n = 0; n < NE; ++n) Iij[n] = Iij[n] + hx1 * weight[g] * (A[n] - B[n]);
            Lij = Lij + hx;
          }
        }
        if (uh[U(i, j - 1, 1, 3)] > 0) {
          for (int g = 0; g < NG; ++g) {
            trace(i, j, phiGD, g, A);
            trace(i, j - 1, phiGU, g, B);
            for (int n = 0; n < NE; ++n) Iij[n] = Iij[n] + hx1 * weight[g] * (A[n] - B[n]);
            Lij = Lij + hx;
          }
        }
        double uinf[NE] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int a = 0; a < NG; ++a)
          for (int b = 0; b < NG; ++b)
            for (int n = 1; n <= NE; ++n) {
              double v = 0;
              for (int d = 1; d <= NP; ++d) v = v + uh[U(i, j, d, n)] * phiG[a][b][d - 1];
              if (std::fabs(v) + 1e-12 > uinf[n - 1]) uinf[n - 1] = std::fabs(v) + 1e-12;
            }
        int flag = c.kxrcf_sticky ? trouble[(size_t)(i - 1) + (size_t)Nx * (j - 1)] : 0;
        for (int n = 0; n < NE; ++n) {
          double r = std::fabs(Iij[n]) / (P * Lij * uinf[n]);
          if (r >= c.kxrcf_ck) flag = 1;
        }
        trouble[(size_t)(i - 1) + (size_t)Nx * (j - 1)] = flag;
      }
  }

  // ---------------------------------------------------------- pp_Limiter --
  // pp_Limiter.f90:1-126 (density: eta = last eta1 < 1, quirk; pressure:
  // bisection calculate_tq)
  void calculate_tq(const double* ubar, const double* uq, double& tq) const {
    double ta = 0, tb = 1;
    double ut[NE];
    while (tb - ta > 1e-14) {
      tq = 0.5 * (ta + tb);
      for (int n = 0; n < NE; ++n) ut[n] = tq * uq[n] + (1 - tq) * ubar[n];
      if (pressure(ut[0], ut[1], ut[2], ut[3], ut[4], ut[5], ut[6], ut[7], gamma) < 1e-12)
        tb = tq;
      else
        ta = tq;
    }
    tq = ta;
  }
  static double norm8(const double* x) {
    double d = 0;
    for (int i = 0; i < 8; ++i) d = d + sq(x[i]);
    return std::sqrt(d);
  }
  void uhGLL_cell(const double* uh, int i, int j, double (*G)[NG][NG][NE]) const {
    for (int s = 0; s < 2; ++s)
      for (int a = 0; a < NG; ++a)
        for (int b = 0; b < NG; ++b)
          for (int n = 0; n < NE; ++n) G[s][a][b][n] = 0;
    for (int d = 1; d <= NP; ++d)
      for (int n = 1; n <= NE; ++n) {
        double v = uh[U(i, j, d, n)];
        for (int s = 0; s < 2; ++s)
          for (int b = 0; b < NG; ++b)
            for (int a = 0; a < NG; ++a) G[s][a][b][n - 1] = G[s][a][b][n - 1] + v * phiGLL[s][a][b][d - 1];
      }
  }
  void pp_limiter(double* uh) const {
    const double epsilon = 1e-13;
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 1; j <= Ny; ++j)
      for (int i = 1; i <= Nx; ++i) {
        double G[2][NG][NG][NE];
        uhGLL_cell(uh, i, j, G);
        double eta = 1;
        for (int a = 0; a < NG; ++a)
          for (int b = 0; b < NG; ++b)
            for (int s = 0; s < 2; ++s) {
              double rb = uh[U(i, j, 1, 1)];
              double eta1 = std::fabs((rb - epsilon) / (rb - G[s][a][b][0]));
              if (eta1 < 1) eta = eta1;
            }
        if (eta < 1)
          for (int d = 2; d <= NP; ++d) uh[U(i, j, d, 1)] = 0.5 * eta * uh[U(i, j, d, 1)];
      }
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 1; j <= Ny; ++j)
      for (int i = 1; i <= Nx; ++i) {
        double G[2][NG][NG][NE];
        uhGLL_cell(uh, i, j, G);
        double ubar[NE];
        for (int n = 1; n <= NE; ++n) ubar[n - 1] = uh[U(i, j, 1, n)];
        double eta = 1, eta1 = 1;
        for (int a = 0; a < NG; ++a)
          for (int b = 0; b < NG; ++b)
            for (int s = 0; s < 2; ++s) {
              const double* uq = G[s][a][b];
              double pq = pressure(uq[0], uq[1], uq[2], uq[3], uq[4], uq[5], uq[6], uq[7], gamma);
              if (pq < 0) {
                double tq = 0;
                calculate_tq(ubar, uq, tq);
                double sqv[NE], d1[NE], d2[NE];
                for (int n = 0; n < NE; ++n) sqv[n] = tq * uq[n] + (1 - tq) * ubar[n];
                for (int n = 0; n < NE; ++n) { d1[n] = sqv[n] - ubar[n]; d2[n] = uq[n] - ubar[n]; }
                eta1 = norm8(d1) / norm8(d2);
              }
              if (eta1 < eta) eta = eta1;
            }
        if (eta < 1) eta = 0.5 * eta;
        for (int n = 1; n <= NE; ++n)
          for (int d = 2; d <= NP; ++d) uh[U(i, j, d, n)] = eta * uh[U(i, j, d, n)];
      }
  }

  // ----------------------------------------------------- TVB_Limiter_P2 --
  // TVB_Limiter_P2.f90:1-191, then div_free_Balsara.f90:13-79. flags gets
  // per interior cell the changed-variable mask (bits 0-7) and the KXRCF
  // flag (bit 24).
  void limit(double* uh, double* bx, double* by, int32_t* flags) {
    const bool gate = (c.detector == GDF_DETECT_KXRCF);
    if (gate) kxrcf(uh);
    std::vector<double>& uhmod = w_uhmod;
    uhmod.resize(uhsize());
    par_copy(uh, uhmod.data(), uhsize());
    const double c23 = 2.0 / 3.0;
    const double M = c.tvb_m;
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 1; j <= Ny; ++j)
      for (int i = 1; i <= Nx; ++i) {
        const size_t cell = (size_t)(i - 1) + (size_t)Nx * (j - 1);
        int32_t word = 0;
        if (gate && trouble[cell]) word |= (1 << 24);
        if (!gate || trouble[cell]) {
          int change[NE] = {0, 0, 0, 0, 0, 0, 0, 0};
          double rhoij = uh[U(i, j, 1, 1)];
          double u1ij = uh[U(i, j, 1, 2)] / rhoij;
          double u2ij = uh[U(i, j, 1, 3)] / rhoij;
          double u3ij = uh[U(i, j, 1, 4)] / rhoij;
          double Eij = uh[U(i, j, 1, 5)];
          double B1ij = uh[U(i, j, 1, 6)], B2ij = uh[U(i, j, 1, 7)], B3ij = uh[U(i, j, 1, 8)];
          double R[64], L[64];
          double DR[NE], DL[NE], D1p[NE], D1m[NE], t1[NE], t2[NE], tU[NE], mod[NE];
          double Rp[NE], Rm[NE], Up[NE], Um[NE];
          if (c.tvb_p1) {
            // TVB_Limiter_P1.f90:19-90: slopes only; a changed variable keeps
            // its limited slopes and loses every higher mode
            double Xm[NE], Ym[NE], D1[NE];
            eigenmatrix(R, L, rhoij, u1ij, u2ij, u3ij, Eij, B1ij, B2ij, B3ij, 1.0, 0.0, 0.0);
            for (int n = 1; n <= NE; ++n) {
              DR[n - 1] = uh[U(i + 1, j, 1, n)] - uh[U(i, j, 1, n)];
              DL[n - 1] = uh[U(i, j, 1, n)] - uh[U(i - 1, j, 1, n)];
              D1[n - 1] = uh[U(i, j, 2, n)];
            }
            matvec(L, DR, t1);
            matvec(L, DL, t2);
            matvec(L, D1, tU);
            minmod(tU, t1, t2, M, hx, mod);
            matvec(R, mod, Xm);
            for (int d = 0; d < NE; ++d)
              if (std::fabs(Xm[d] - D1[d]) > 1e-6) change[d] = 1;
            eigenmatrix(R, L, rhoij, u1ij, u2ij, u3ij, Eij, B1ij, B2ij, B3ij, 0.0, 1.0, 0.0);
            for (int n = 1; n <= NE; ++n) {
              DR[n - 1] = uh[U(i, j + 1, 1, n)] - uh[U(i, j, 1, n)];
              DL[n - 1] = uh[U(i, j, 1, n)] - uh[U(i, j - 1, 1, n)];
              D1[n - 1] = uh[U(i, j, 3, n)];
            }
            matvec(L, DR, t1);
            matvec(L, DL, t2);
            matvec(L, D1, tU);
            minmod(tU, t1, t2, M, hy, mod);
            matvec(R, mod, Ym);
            for (int d = 0; d < NE; ++d)
              if (std::fabs(Ym[d] - D1[d]) > 1e-6) change[d] = 1;
            for (int d = 1; d <= NE; ++d) {
              if (change[d - 1] == 1) {
                word |= (1 << (d - 1));
                for (int q = 4; q <= NP; ++q) uhmod[U(i, j, q, d)] = 0;
                uhmod[U(i, j, 2, d)] = Xm[d - 1];
                uhmod[U(i, j, 3, d)] = Ym[d - 1];
              }
            }
            if (flags) flags[cell] = word;
            continue;
          }
          // x direction (:35-68)
          eigenmatrix(R, L, rhoij, u1ij, u2ij, u3ij, Eij, B1ij, B2ij, B3ij, 1.0, 0.0, 0.0);
          for (int n = 1; n <= NE; ++n) {
            DR[n - 1] = uh[U(i + 1, j, 1, n)] - uh[U(i, j, 1, n)];
            DL[n - 1] = uh[U(i, j, 1, n)] - uh[U(i - 1, j, 1, n)];
            D1p[n - 1] = uh[U(i, j, 2, n)] + c23 * uh[U(i, j, 4, n)];
            D1m[n - 1] = uh[U(i, j, 2, n)] - c23 * uh[U(i, j, 4, n)];
          }
          matvec(L, DR, t1);
          matvec(L, DL, t2);
          matvec(L, D1p, tU);
          minmod(tU, t1, t2, M, hx, mod);
          matvec(R, mod, Rp);
          for (int d = 0; d < NE; ++d)
            if (std::fabs(Rp[d] - D1p[d]) > 1e-6) change[d] = 1;
          matvec(L, D1m, tU);
          minmod(tU, t1, t2, M, hx, mod);
          matvec(R, mod, Rm);
          for (int d = 0; d < NE; ++d)
            if (std::fabs(Rm[d] - D1m[d]) > 1e-6) change[d] = 1;
          // y direction (:70-103)
          if (c.eig_y_zero_w)
            eigenmatrix(R, L, rhoij, u1ij, u2ij, 0.0, Eij, B1ij, B2ij, 0.0, 0.0, 1.0, 0.0);
          else
            eigenmatrix(R, L, rhoij, u1ij, u2ij, u3ij, Eij, B1ij, B2ij, B3ij, 0.0, 1.0, 0.0);
          for (int n = 1; n <= NE; ++n) {
            DR[n - 1] = uh[U(i, j + 1, 1, n)] - uh[U(i, j, 1, n)];
            DL[n - 1] = uh[U(i, j, 1, n)] - uh[U(i, j - 1, 1, n)];
            D1p[n - 1] = uh[U(i, j, 3, n)] + c23 * uh[U(i, j, 6, n)];
            D1m[n - 1] = uh[U(i, j, 3, n)] - c23 * uh[U(i, j, 6, n)];
          }
          matvec(L, DR, t1);
          matvec(L, DL, t2);
          matvec(L, D1p, tU);
          minmod(tU, t1, t2, M, hy, mod);
          matvec(R, mod, Up);
          for (int d = 0; d < NE; ++d)
            if (std::fabs(Up[d] - D1p[d]) > 1e-6) change[d] = 1;
          matvec(L, D1m, tU);
          minmod(tU, t1, t2, M, hy, mod);
          matvec(R, mod, Um);
          for (int d = 0; d < NE; ++d)
            if (std::fabs(Um[d] - D1m[d]) > 1e-6) change[d] = 1;
          // rewrite (:105-114)
          for (int d = 1; d <= NE; ++d) {
            if (change[d - 1] == 1) {
              word |= (1 << (d - 1));
              for (int q = 7; q <= NP; ++q) uhmod[U(i, j, q, d)] = 0;
              uhmod[U(i, j, 5, d)] = 0;
              uhmod[U(i, j, 2, d)] = 0.5 * (Rp[d - 1] + Rm[d - 1]);
              uhmod[U(i, j, 3, d)] = 0.5 * (Up[d - 1] + Um[d - 1]);
              uhmod[U(i, j, 4, d)] = c.tvb_slope * (Rp[d - 1] - Rm[d - 1]);
              uhmod[U(i, j, 6, d)] = c.tvb_slope * (Up[d - 1] - Um[d - 1]);
            }
          }
        }
        if (flags) flags[cell] = word;
      }
    par_copy(uhmod.data(), uh, uhsize());
    if (c.pp_limiter) pp_limiter(uh);
    set_bc(uh);
    if (c.faceb_limiter || c.tvb_p1) {   // TVB_Limiter_P1 applies it always
      // TVB_Limiter_P2.f90:128-187 (face traces of cell B from both sides,
      // minmodB of face modes 2..3, applied)
      const double c25 = 2.0 / 5.0;
      auto aRM = [&](int i, int j, int d) {
        double a00 = uh[U(i, j, 1, 6)], a10 = uh[U(i, j, 2, 6)], a01 = uh[U(i, j, 3, 6)], a20 = uh[U(i, j, 4, 6)];
        double a11 = uh[U(i, j, 5, 6)], a02 = uh[U(i, j, 6, 6)], a30 = uh[U(i, j, 7, 6)], a12 = uh[U(i, j, 9, 6)];
        (void)a00; (void)a10; (void)a20; (void)a30;
        if (d == 1) return a00 + a10 + c23 * a20 + c25 * a30;
        if (d == 2) return a01 + a11;
        return a02 + a12;
      };
      auto aLM = [&](int i, int j, int d) {
        double a00 = uh[U(i, j, 1, 6)], a10 = uh[U(i, j, 2, 6)], a01 = uh[U(i, j, 3, 6)], a20 = uh[U(i, j, 4, 6)];
        double a11 = uh[U(i, j, 5, 6)], a02 = uh[U(i, j, 6, 6)], a30 = uh[U(i, j, 7, 6)], a12 = uh[U(i, j, 9, 6)];
        if (d == 1) return a00 - a10 + c23 * a20 - c25 * a30;
        if (d == 2) return a01 - a11;
        return a02 - a12;
      };
      auto bUM = [&](int i, int j, int d) {
        double b00 = uh[U(i, j, 1, 7)], b10 = uh[U(i, j, 2, 7)], b01 = uh[U(i, j, 3, 7)], b20 = uh[U(i, j, 4, 7)];
        double b11 = uh[U(i, j, 5, 7)], b02 = uh[U(i, j, 6, 7)], b21 = uh[U(i, j, 8, 7)], b03 = uh[U(i, j, 10, 7)];
        if (d == 1) return b00 + b01 + c23 * b02 + c25 * b03;
        if (d == 2) return b10 + b11;
        return b20 + b21;
      };
      auto bDM = [&](int i, int j, int d) {
        double b00 = uh[U(i, j, 1, 7)], b10 = uh[U(i, j, 2, 7)], b01 = uh[U(i, j, 3, 7)], b20 = uh[U(i, j, 4, 7)];
        double b11 = uh[U(i, j, 5, 7)], b02 = uh[U(i, j, 6, 7)], b21 = uh[U(i, j, 8, 7)], b03 = uh[U(i, j, 10, 7)];
        if (d == 1) return b00 - b01 + c23 * b02 - c25 * b03;
        if (d == 2) return b10 - b11;
        return b20 - b21;
      };
      std::vector<double> bxm(bx, bx + bxsize()), bym(by, by + bysize());
      for (int i = 0; i <= Nx; ++i)
        for (int j = 1; j <= Ny; ++j)
          for (int d = 2; d <= 3; ++d)
            bxm[BXi(i, j, d)] = minmodB(bx[BXi(i, j, d)], aRM(i, j, d), aLM(i + 1, j, d), M, hy);
      for (int i = 1; i <= Nx; ++i)
        for (int j = 0; j <= Ny; ++j)
          for (int d = 2; d <= 3; ++d)
            bym[BYi(i, j, d)] = minmodB(by[BYi(i, j, d)], bUM(i, j, d), bDM(i, j + 1, d), M, hx);
      std::copy(bxm.begin(), bxm.end(), bx);
      std::copy(bym.begin(), bym.end(), by);
    }
    div_free(uh, bx, by);
  }

  // div_free_Balsara.f90:13-79
  void div_free(double* uh, const double* bx, const double* by) const {
    for (int n = 6; n <= 7; ++n)
      for (int d = 1; d <= NP; ++d)
        for (int j = 0; j <= Ny + 1; ++j)
          for (int i = 0; i <= Nx + 1; ++i) uh[U(i, j, d, n)] = 0;
    const double c16 = 1.0 / 6.0, c115 = 1.0 / 15.0, c14 = 1.0 / 4.0, c12 = 1.0 / 2.0;
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 1; j <= Ny; ++j)
      for (int i = 1; i <= Nx; ++i) {
        double a0R = bx[BXi(i, j, 1)], a1R = bx[BXi(i, j, 2)], a2R = bx[BXi(i, j, 3)];
        double a0L = bx[BXi(i - 1, j, 1)], a1L = bx[BXi(i - 1, j, 2)], a2L = bx[BXi(i - 1, j, 3)];
        double b0U = by[BYi(i, j, 1)], b1U = by[BYi(i, j, 2)], b2U = by[BYi(i, j, 3)];
        double b0D = by[BYi(i, j - 1, 1)], b1D = by[BYi(i, j - 1, 2)], b2D = by[BYi(i, j - 1, 3)];
        double rxy = hx / hy, ryx = hy / hx;
        double a00 = c12 * (a0R + a0L) + c16 * rxy * (b1U - b1D);
        double a10 = c12 * (a0R - a0L) + c115 * rxy * (b2U - b2D);
        double a01 = c12 * (a1R + a1L);
        double a20 = -c14 * rxy * (b1U - b1D);
        double a11 = c12 * (a1R - a1L);
        double a02 = c12 * (a2R + a2L);
        double a30 = -c16 * rxy * (b2U - b2D);
        double a12 = c12 * (a2R - a2L);
        double b00 = c12 * (b0U + b0D) + c16 * ryx * (a1R - a1L);
        double b01 = c12 * (b0U - b0D) + c115 * ryx * (a2R - a2L);
        double b10 = c12 * (b1U + b1D);
        double b02 = -c14 * ryx * (a1R - a1L);
        double b11 = c12 * (b1U - b1D);
        double b20 = c12 * (b2U + b2D);
        double b03 = -c16 * ryx * (a2R - a2L);
        double b21 = c12 * (b2U - b2D);
        uh[U(i, j, 1, 6)] = a00; uh[U(i, j, 2, 6)] = a10; uh[U(i, j, 3, 6)] = a01; uh[U(i, j, 4, 6)] = a20;
        uh[U(i, j, 5, 6)] = a11; uh[U(i, j, 6, 6)] = a02; uh[U(i, j, 7, 6)] = a30; uh[U(i, j, 9, 6)] = a12;
        uh[U(i, j, 1, 7)] = b00; uh[U(i, j, 2, 7)] = b10; uh[U(i, j, 3, 7)] = b01; uh[U(i, j, 4, 7)] = b20;
        uh[U(i, j, 5, 7)] = b11; uh[U(i, j, 6, 7)] = b02; uh[U(i, j, 8, 7)] = b21; uh[U(i, j, 10, 7)] = b03;
      }
  }

  // ------------------------------------------------------- calculate_dt --
  // calculate_dt.f90:5-27
  double calc_dt(const double* uh) const {
    double ax = 0, ay = 0;
    for (int i = 1; i <= Nx; ++i)
      for (int j = 1; j <= Ny; ++j) {
        double a1, a2;
        const double r = uh[U(i, j, 1, 1)], m1 = uh[U(i, j, 1, 2)], m2 = uh[U(i, j, 1, 3)], m3 = uh[U(i, j, 1, 4)];
        const double E = uh[U(i, j, 1, 5)], B1 = uh[U(i, j, 1, 6)], B2 = uh[U(i, j, 1, 7)], B3 = uh[U(i, j, 1, 8)];
        eigenvalueMm(a1, a2, r, m1, m2, m3, E, B1, B2, B3, 1, 0);
        if (std::fabs(a1) > ax || std::fabs(a2) > ax) ax = fmax2(std::fabs(a1), std::fabs(a2));
        eigenvalueMm(a1, a2, r, m1, m2, m3, E, B1, B2, B3, 0, 1);
        if (std::fabs(a1) > ay || std::fabs(a2) > ay) ay = fmax2(std::fabs(a1), std::fabs(a2));
      }
    return c.cfl / (ax / hx + ay / hy);
  }

  // ---------------------------------------------------------- RK3 step --
  // RK3.f90:58-151 (one pass of the loop body). Combines use the pre-limit
  // stage arrays uI / uII as the reference does.
  int step(double* uh, double* bx, double* by, double* t, double tend, double* dt_out, int32_t* flags) {
    const size_t usz = uhsize(), bxs = bxsize(), bys = bysize();
    for (auto* v : {&w_du, &w_uI, &w_uII, &w_uh0}) v->resize(usz);
    for (auto* v : {&w_dez1, &w_BxI, &w_BxII, &w_Bx0}) v->resize(bxs);
    for (auto* v : {&w_dez2, &w_ByI, &w_ByII, &w_By0}) v->resize(bys);
    for (auto* v : {&w_f1, &w_f2, &w_f3}) v->resize((size_t)Nx * Ny);
    std::vector<double>&du = w_du, &uI = w_uI, &uII = w_uII, &uh0 = w_uh0;
    std::vector<double>&dez1 = w_dez1, &dez2 = w_dez2, &BxI = w_BxI, &ByI = w_ByI, &BxII = w_BxII, &ByII = w_ByII,
                       &Bx0 = w_Bx0, &By0 = w_By0;
    std::vector<int32_t>&f1 = w_f1, &f2 = w_f2, &f3 = w_f3;
    double dt = calc_dt(uh);
    double tt = *t;
    if (tt + dt >= tend) {
      dt = tend - tt;
      tt = tend;
    } else {
      tt = tt + dt;
    }
    if (c.dt_floor_stop && dt < 1e-7) tt = tend;
    // stage 1 (:74-97)
    set_bc(uh);
    Lh(uh, du.data());
    LhEz(uh, dez1.data(), dez2.data());
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < usz; ++q) uI[q] = uh[q] + dt * du[q];
    for (size_t q = 0; q < bxs; ++q) BxI[q] = bx[q] + dt * dez1[q];
    for (size_t q = 0; q < bys; ++q) ByI[q] = by[q] + dt * dez2[q];
    par_copy(uh, uh0.data(), usz);
    std::copy(bx, bx + bxs, Bx0.begin());
    std::copy(by, by + bys, By0.begin());
    par_copy(uI.data(), uh, usz);
    std::copy(BxI.begin(), BxI.end(), bx);
    std::copy(ByI.begin(), ByI.end(), by);
    limit(uh, bx, by, f1.data());
    set_bc(uh);
    // stage 2 (:102-120)
    Lh(uh, du.data());
    LhEz(uh, dez1.data(), dez2.data());
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < usz; ++q) uh[q] = uI[q] + dt * du[q];
    for (size_t q = 0; q < bxs; ++q) bx[q] = BxI[q] + dt * dez1[q];
    for (size_t q = 0; q < bys; ++q) by[q] = ByI[q] + dt * dez2[q];
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < usz; ++q) uII[q] = (3.0 / 4.0) * uh0[q] + (1.0 / 4.0) * uh[q];
    for (size_t q = 0; q < bxs; ++q) BxII[q] = (3.0 / 4.0) * Bx0[q] + (1.0 / 4.0) * bx[q];
    for (size_t q = 0; q < bys; ++q) ByII[q] = (3.0 / 4.0) * By0[q] + (1.0 / 4.0) * by[q];
    par_copy(uII.data(), uh, usz);
    std::copy(BxII.begin(), BxII.end(), bx);
    std::copy(ByII.begin(), ByII.end(), by);
    limit(uh, bx, by, f2.data());
    // stage 3 (:123-139)
    set_bc(uh);
    Lh(uh, du.data());
    LhEz(uh, dez1.data(), dez2.data());
    for (size_t q = 0; q < bxs; ++q) bx[q] = BxII[q] + dt * dez1[q];
    for (size_t q = 0; q < bys; ++q) by[q] = ByII[q] + dt * dez2[q];
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < usz; ++q) uh[q] = uII[q] + dt * du[q];
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < usz; ++q) uh[q] = (1.0 / 3.0) * uh0[q] + (2.0 / 3.0) * uh[q];
    for (size_t q = 0; q < bxs; ++q) bx[q] = (1.0 / 3.0) * Bx0[q] + (2.0 / 3.0) * bx[q];
    for (size_t q = 0; q < bys; ++q) by[q] = (1.0 / 3.0) * By0[q] + (2.0 / 3.0) * by[q];
    limit(uh, bx, by, f3.data());
    if (flags) {
      for (size_t q = 0; q < (size_t)Nx * Ny; ++q) {
        int32_t w = (f1[q] & 0xff) | ((f2[q] & 0xff) << 8) | ((f3[q] & 0xff) << 16);
        if (f1[q] & (1 << 24)) w |= (1 << 24);
        if (f2[q] & (1 << 24)) w |= (1 << 25);
        if (f3[q] & (1 << 24)) w |= (1 << 26);
        flags[q] = w;
      }
    }
    *t = tt;
    if (dt_out) *dt_out = dt;
    return 0;
  }

  // ------------------------------------------------------- diagnostics --
  // calculate_umax.f90, calculate_totaldiv.f90, calculate_pmin.f90
  void diagnostics(const double* uh, double* umax, double* totaldiv, double* pmin) const {
    double um = 0;
    for (int i = 1; i <= Nx; ++i)
      for (int j = 1; j <= Ny; ++j) {
        if (c.umax_all_vars) {
          for (int n = 1; n <= NE; ++n)
            if (std::fabs(uh[U(i, j, 1, n)]) > um) um = std::fabs(uh[U(i, j, 1, n)]);
        } else if (std::fabs(uh[U(i, j, 1, 1)]) > um) {
          um = std::fabs(uh[U(i, j, 1, 1)]);
        }
      }
    double td = 0;
    double pm = 1000000;
    for (int i = 1; i <= Nx; ++i)
      for (int j = 1; j <= Ny; ++j) {
        double gd[NG][NG];
        for (int a = 0; a < NG; ++a)
          for (int b = 0; b < NG; ++b) gd[a][b] = 0;
        for (int d = 1; d <= NP; ++d)
          for (int b = 0; b < NG; ++b)
            for (int a = 0; a < NG; ++a)
              gd[a][b] = gd[a][b] + uh[U(i, j, d, 6)] * phixG[a][b][d - 1] + uh[U(i, j, d, 7)] * phiyG[a][b][d - 1];
        for (int a = 0; a < NG; ++a)
          for (int b = 0; b < NG; ++b) td = td + weight[a] * weight[b] * sq(gd[a][b]);
        double uG[NG][NG][NE];
        for (int a = 0; a < NG; ++a)
          for (int b = 0; b < NG; ++b)
            for (int n = 0; n < NE; ++n) uG[a][b][n] = 0;
        for (int n = 1; n <= NE; ++n)
          for (int d = 1; d <= NP; ++d)
            for (int b = 0; b < NG; ++b)
              for (int a = 0; a < NG; ++a) uG[a][b][n - 1] = uG[a][b][n - 1] + uh[U(i, j, d, n)] * phiG[a][b][d - 1];
        for (int a = 0; a < NG; ++a)
          for (int b = 0; b < NG; ++b) {
            const double* q = uG[a][b];
            double p1 = pressure(q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], gamma);
            if (p1 < pm) pm = p1;
          }
      }
    *umax = um;
    *totaldiv = std::sqrt(td * hx1 * hy1);
    *pmin = pm;
  }
};

// -------------------------------------------------------- initial data --
// init_data.f90:1-123 with the problem functions of init1/3/4/5/6.txt.
// Benchmark problems follow the benchmark definitions (rotor speed 2 at
// r0 with the Rotor_functions.f90 taper; blast with caller parameters).
struct Problem {
  int id;
  double g;   // gamma of com.txt
  double prm[8];
  void eval(double x, double y, double* Uv) const {
    const double pi = 4 * std::atan(1.0);
    double rho = 0, v1 = 0, v2 = 0, v3 = 0, p = 0, B1 = 0, B2 = 0, B3 = 0;
    const double g1 = g - 1;
    switch (id) {
      case GDF_PROB_VORTEX: {  // init1.txt:3-20
        double r2 = x * x + y * y;
        p = 1 - r2 / (8.0 * (pi * pi)) * std::exp(1 - r2);
        rho = 1;
        v1 = 1 - 1.0 / (2.0 * pi) * y * std::exp(0.5 * (1 - r2));
        v2 = 1 + 1.0 / (2.0 * pi) * x * std::exp(0.5 * (1 - r2));
        B1 = -1.0 / (2.0 * pi) * y * std::exp(0.5 * (1 - r2));
        B2 = 1.0 / (2.0 * pi) * x * std::exp(0.5 * (1 - r2));
        break;
      }
      case GDF_PROB_ORSZAG_TANG: {  // init3.txt:3-16
        p = g; rho = g * g; v1 = -std::sin(y); v2 = std::sin(x); B1 = -std::sin(y); B2 = std::sin(2.0 * x);
        break;
      }
      case GDF_PROB_ROTOR: {  // Rotor_functions.f90:1-70 shape, speed u0 at r0
        const double cx = prm[0], cy = prm[1], r0 = prm[2], r1 = prm[3], rin = prm[4], u0 = prm[5];
        double r = std::sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy));
        double f = (r1 - r) / (r1 - r0);
        if (r < r0) { rho = rin; v1 = -u0 * (y - cy) / r0; v2 = u0 * (x - cx) / r0; }
        else if (r < r1) { rho = 1.0 + (rin - 1.0) * f; v1 = -f * u0 * (y - cy) / r; v2 = f * u0 * (x - cx) / r; }
        else { rho = 1.0; v1 = 0; v2 = 0; }
        p = prm[6]; B1 = prm[7]; B2 = 0;
        break;
      }
      case GDF_PROB_BLAST: {  // init5.txt / p0.f90 shape
        double dx = x - prm[0], dy = y - prm[1];
        double r = std::sqrt(dx * dx + dy * dy);
        p = (r <= prm[2]) ? prm[3] : prm[4];
        rho = prm[5]; B1 = prm[6]; B2 = prm[7];
        break;
      }
      default: {  // GDF_PROB_CLOUD_SHOCK, Cloud_Shock_functions.f90
        double r = std::sqrt((x - 1.4) * (x - 1.4) + (y - 0.5) * (y - 0.5));
        const double r0 = 0.18;
        if (x <= 1.2) { rho = 3.88968; v1 = 0; v2 = 0; v3 = -0.05234; p = 14.2641; B1 = 1; B2 = 0; B3 = 3.9353; }
        else { rho = (r >= r0) ? 1.0 : 5.0; v1 = -3.3156; v2 = 0; v3 = 0; p = 0.04; B1 = 1; B2 = 0; B3 = 1; }
        break;
      }
    }
    Uv[0] = rho;
    Uv[1] = rho * v1;
    Uv[2] = rho * v2;
    Uv[3] = rho * v3;
    if (id == GDF_PROB_CLOUD_SHOCK)
      Uv[4] = p / g1 + 0.5 * rho * (v1 * v1 + v2 * v2 + v3 * v3) + 0.5 * (B1 * B1 + B2 * B2 + B3 * B3);
    else
      Uv[4] = p / g1 + 0.5 * rho * (v1 * v1 + v2 * v2) + 0.5 * (B1 * B1 + B2 * B2);
    Uv[5] = B1;
    Uv[6] = B2;
    Uv[7] = B3;
  }
};

void default_params(int problem, double* prm) {
  const double pi = 4 * std::atan(1.0);
  for (int q = 0; q < 8; ++q) prm[q] = 0;
  if (problem == GDF_PROB_ROTOR) {
    prm[0] = 0.5; prm[1] = 0.5; prm[2] = 0.1; prm[3] = 0.115; prm[4] = 10.0; prm[5] = 2.0;
    prm[6] = 1.0; prm[7] = 5.0 / std::sqrt(4 * pi);
  } else if (problem == GDF_PROB_BLAST) {
    prm[0] = 0; prm[1] = 0; prm[2] = 0.1; prm[3] = 1000; prm[4] = 0.1; prm[5] = 1.0;
    prm[6] = 100.0 / std::sqrt(8 * pi); prm[7] = 100.0 / std::sqrt(8 * pi);
  }
}

#ifndef GDF_ORACLE_NO_P3
#include "gdf_oracle_p3.inc"
#include "gdf_oracle_cy.inc"
#endif

}  // namespace

// ----------------------------------------------------------------- C ABI --
extern "C" {

void* orc_create(const GdfConfig* cfg) {
  if (!cfg || cfg->nx < 1 || cfg->ny < 1) return nullptr;
  Oracle* o = new Oracle();
  o->setup(*cfg);
  return o;
}
void orc_destroy(void* h) { delete static_cast<Oracle*>(h); }
int orc_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
}

int orc_init_data(void* h, int problem, const double* params, double* uh, double* bx, double* by) {
  Oracle& o = *static_cast<Oracle*>(h);
  Problem P;
  P.id = problem;
  P.g = o.gamma;
  double prm[8];
  default_params(problem, prm);
  if (params) for (int q = 0; q < 8; ++q) prm[q] = params[q];
  for (int q = 0; q < 8; ++q) P.prm[q] = prm[q];
  const int shock = (problem == GDF_PROB_BLAST || problem == GDF_PROB_CLOUD_SHOCK) ? 1 : 0;
  std::fill(uh, uh + o.uhsize(), 0.0);
  std::fill(bx, bx + o.bxsize(), 0.0);
  std::fill(by, by + o.bysize(), 0.0);
  std::vector<double> Xc(o.Nx + 1), Yc(o.Ny + 1);
  for (int i = 1; i <= o.Nx; ++i) Xc[i] = o.c.xa + (i - 0.5) * o.hx;
  for (int j = 1; j <= o.Ny; ++j) Yc[j] = o.c.ya + (j - 0.5) * o.hy;
  double Uv[8];
  for (int i = 1; i <= o.Nx; ++i)
    for (int j = 1; j <= o.Ny; ++j) {
      for (int d = 1; d <= 6; ++d)  // mask d <= 6 (init_data.f90:43, quirk Q9)
        for (int a = 0; a < NG; ++a)
          for (int b = 0; b < NG; ++b) {
            P.eval(Xc[i] + o.hx1 * o.lambda[a], Yc[j] + o.hy1 * o.lambda[b], Uv);
            for (int n = 1; n <= NE; ++n)
              uh[o.U(i, j, d, n)] = uh[o.U(i, j, d, n)] + o.weight[a] * o.weight[b] * o.phiG[a][b][d - 1] * Uv[n - 1];
          }
      for (int d = 1; d <= NP; ++d)
        for (int n = 1; n <= NE; ++n) uh[o.U(i, j, d, n)] = 0.25 * uh[o.U(i, j, d, n)] / o.mm[d - 1];
    }
  for (int i = 0; i <= o.Nx; ++i)
    for (int j = 1; j <= o.Ny; ++j)
      for (int d = 1; d <= 3; ++d) {
        double acc = 0;
        for (int b = 0; b < NG; ++b) {
          P.eval(o.c.xa + i * o.hx, Yc[j] + o.hy1 * o.lambda[b], Uv);
          acc = acc + 0.5 * o.weight[b] * o.EzG[b][d - 1] * Uv[5];
        }
        bx[o.BXi(i, j, d)] = acc / o.mmE[d - 1];
      }
  for (int i = 1; i <= o.Nx; ++i)
    for (int j = 0; j <= o.Ny; ++j)
      for (int d = 1; d <= 3; ++d) {
        double acc = 0;
        for (int a = 0; a < NG; ++a) {
          P.eval(Xc[i] + o.hx1 * o.lambda[a], o.c.ya + j * o.hy, Uv);
          acc = acc + 0.5 * o.weight[a] * o.EzG[a][d - 1] * Uv[6];
        }
        by[o.BYi(i, j, d)] = acc / o.mmE[d - 1];
      }
  if (shock) {
    for (int i = 1; i <= o.Nx; ++i)
      for (int j = 1; j <= o.Ny; ++j) {
        P.eval(Xc[i], Yc[j], Uv);
        for (int n = 1; n <= NE; ++n) {
          for (int d = 2; d <= NP; ++d) uh[o.U(i, j, d, n)] = 0;
          uh[o.U(i, j, 1, n)] = Uv[n - 1];
        }
      }
    for (int i = 0; i <= o.Nx; ++i)
      for (int j = 1; j <= o.Ny; ++j) {
        P.eval(o.c.xa + i * o.hx, Yc[j], Uv);
        bx[o.BXi(i, j, 2)] = 0; bx[o.BXi(i, j, 3)] = 0;
        bx[o.BXi(i, j, 1)] = Uv[5];
      }
    for (int i = 1; i <= o.Nx; ++i)
      for (int j = 0; j <= o.Ny; ++j) {
        P.eval(Xc[i], o.c.ya + j * o.hy, Uv);
        by[o.BYi(i, j, 2)] = 0; by[o.BYi(i, j, 3)] = 0;
        by[o.BYi(i, j, 1)] = Uv[6];
      }
  }
  return 0;
}

int orc_set_bc(void* h, double* uh) { static_cast<Oracle*>(h)->set_bc(uh); return 0; }

int orc_lh(void* h, const double* uh, double* du) { static_cast<Oracle*>(h)->Lh(uh, du); return 0; }

int orc_lhez(void* h, const double* uh, double* dez1, double* dez2) {
  Oracle& o = *static_cast<Oracle*>(h);
  std::vector<double> du(o.uhsize());
  o.Lh(uh, du.data());
  o.LhEz(uh, dez1, dez2);
  return 0;
}

int orc_limit(void* h, double* uh, double* bx, double* by, int32_t* flags) {
  static_cast<Oracle*>(h)->limit(uh, bx, by, flags);
  return 0;
}

int orc_div_free(void* h, double* uh, const double* bx, const double* by) {
  static_cast<Oracle*>(h)->div_free(uh, bx, by);
  return 0;
}

int orc_dt(void* h, const double* uh, double* dt) { *dt = static_cast<Oracle*>(h)->calc_dt(uh); return 0; }

int orc_prepare(void* h, double* uh, double* bx, double* by, int32_t* flags) {
  Oracle& o = *static_cast<Oracle*>(h);
  o.set_bc(uh);
  o.limit(uh, bx, by, flags);
  return 0;
}

int orc_step(void* h, double* uh, double* bx, double* by, double* t, double tend, double* dt, int32_t* flags) {
  return static_cast<Oracle*>(h)->step(uh, bx, by, t, tend, dt, flags);
}

int orc_diagnostics(void* h, const double* uh, double* umax, double* totaldiv, double* pmin) {
  static_cast<Oracle*>(h)->diagnostics(uh, umax, totaldiv, pmin);
  return 0;
}

void orc_reset_trouble(void* h) {
  Oracle& o = *static_cast<Oracle*>(h);
  std::fill(o.trouble.begin(), o.trouble.end(), 0);
}

// Pointwise entry points for the known-answer tests.
void orc_eigenvalue(void* h, const double* Uv, int n1, int n2, double* amax, double* amin) {
  static_cast<Oracle*>(h)->eigenvalueMm(*amax, *amin, Uv[0], Uv[1], Uv[2], Uv[3], Uv[4], Uv[5], Uv[6], Uv[7], n1, n2);
}
void orc_eigenmatrix(void* h, const double* prim8, const double* n3v, double* evr, double* evl) {
  static_cast<Oracle*>(h)->eigenmatrix(evr, evl, prim8[0], prim8[1], prim8[2], prim8[3], prim8[4], prim8[5], prim8[6],
                                       prim8[7], n3v[0], n3v[1], n3v[2]);
}
// 1-D Riemann solve with the reference calling convention of Lh.f90:207-231
// (ul = left state of the face, ur = right state; dir 1 = x, 2 = y).
void orc_riemann(void* h, const double* ul, const double* ur, int dir, double* fhat) {
  Oracle& o = *static_cast<Oracle*>(h);
  double FL[8], FR[8];
  o.point_flux(ul, FL, dir - 1, false, false);
  o.point_flux(ur, FR, dir - 1, dir == 2, dir == 1);
  double a1, a2, b1, b2;
  o.eigenvalueMm(a1, a2, ul[0], ul[1], ul[2], ul[3], ul[4], ul[5], ul[6], ul[7], dir == 1 ? 1 : 0, dir == 2 ? 1 : 0);
  o.eigenvalueMm(b1, b2, ur[0], ur[1], ur[2], ur[3], ur[4], ur[5], ur[6], ur[7], dir == 1 ? 1 : 0, dir == 2 ? 1 : 0);
  Oracle::RS s;
  s.SR = fmax2(a1, b1);
  s.SL = fmin2(a2, b2);
  s.direction = dir;
  for (int n = 0; n < 8; ++n) { s.FR1[n] = FR[n]; s.FL1[n] = FL[n]; s.UR1[n] = ur[n]; s.UL1[n] = ul[n]; }
  o.riemann1d(s);
  for (int n = 0; n < 8; ++n) fhat[n] = s.Fhat1[n];
}
double orc_vertex_ez(void* h, const double* uru, const double* ulu, const double* urd, const double* uld) {
  return static_cast<Oracle*>(h)->vertex_Ez(uru, ulu, urd, uld);
}
double orc_pow_hxhy(void* h) {
  Oracle& o = *static_cast<Oracle*>(h);
  return std::pow(o.hx * o.hy, 0.75);
}

#ifndef GDF_ORACLE_NO_P3
// ------------------------------------------------ the k = 3 variant (P3) --
void* orc_p3_create(const GdfP3Config* cfg) {
  if (!cfg || cfg->nx < 1 || cfg->ny < 1) return nullptr;
  OracleP3* o = new OracleP3();
  o->setup(*cfg);
  return o;
}
void orc_p3_destroy(void* h) { delete static_cast<OracleP3*>(h); }
int orc_p3_init_data(void* h, int problem, double* uh, double* bx, double* by) {
  static_cast<OracleP3*>(h)->init_data(problem, uh, bx, by);
  return 0;
}
int orc_p3_set_bc(void* h, double* uh, double* bx, double* by) {
  static_cast<OracleP3*>(h)->set_bc(uh, bx, by);
  return 0;
}
int orc_p3_lh(void* h, double* uh, double* bx, double* by, double* du, double* dbx, double* dby) {
  static_cast<OracleP3*>(h)->Lh(uh, bx, by, du, dbx, dby);
  return 0;
}
int orc_p3_limit(void* h, double* uh, double* bx, double* by, int32_t* flags) {
  static_cast<OracleP3*>(h)->limit_all(uh, bx, by, flags);
  return 0;
}
int orc_p3_dt(void* h, const double* uh, double* dt) {
  *dt = static_cast<OracleP3*>(h)->calc_dt(uh);
  return 0;
}
int orc_p3_step(void* h, double* uh, double* bx, double* by, double* t, double tend, double* dt) {
  static_cast<OracleP3*>(h)->step(uh, bx, by, t, tend, dt);
  return 0;
}
int orc_p3_diagnostics(void* h, const double* uh, double* umax, double* totaldiv) {
  static_cast<OracleP3*>(h)->diagnostics(uh, umax, totaldiv);
  return 0;
}
// the basis tables, for the orthogonality and trace pins: phiG, phixG,
// phiyG [25*15 each, (a*5+b)*15+d], phiGR/GL/GU/GD [5*15 each], corner
// values RU/LU/RD/LD [15 each], mm [15]
void orc_p3_basis(void* h, double* out) {
  const OracleP3& o = *static_cast<OracleP3*>(h);
  double* q = out;
  for (auto* T : {&o.phiG, &o.phixG, &o.phiyG})
    for (int a = 0; a < NG; ++a)
      for (int b = 0; b < NG; ++b)
        for (int d = 0; d < NP3; ++d) *q++ = (*T)[a][b][d];
  for (auto* T : {&o.phiGR, &o.phiGL, &o.phiGU, &o.phiGD})
    for (int g = 0; g < NG; ++g)
      for (int d = 0; d < NP3; ++d) *q++ = (*T)[g][d];
  for (auto* T : {&o.phiRU, &o.phiLU, &o.phiRD, &o.phiLD, &o.mm})
    for (int d = 0; d < NP3; ++d) *q++ = (*T)[d];
}

// ------------------------------------------ the cylindrical variant (cy) --
void* orc_cy_create(const GdfCyConfig* cfg) {
  if (!cfg) return nullptr;
  OracleCy* o = new OracleCy();
  if (!o->setup(*cfg)) { delete o; return nullptr; }
  return o;
}
void orc_cy_destroy(void* h) { delete static_cast<OracleCy*>(h); }
int orc_cy_init_data(void* h, int problem, double* uh, double* br, double* bz) {
  static_cast<OracleCy*>(h)->init_data(problem, uh, br, bz);
  return 0;
}
int orc_cy_set_bc(void* h, double* uh) {
  static_cast<OracleCy*>(h)->set_bc(uh);
  return 0;
}
int orc_cy_lh(void* h, double* uh, double t_rk, double* du, double* dbr, double* dbz) {
  static_cast<OracleCy*>(h)->lh(uh, t_rk, du, dbr, dbz);
  return 0;
}
int orc_cy_limit(void* h, double* uh, double* br, double* bz, int32_t* flags) {
  static_cast<OracleCy*>(h)->limit(uh, br, bz, flags);
  return 0;
}
int orc_cy_dt(void* h, const double* uh, double* dt) {
  *dt = static_cast<OracleCy*>(h)->calc_dt(uh);
  return 0;
}
int orc_cy_step(void* h, double* uh, double* br, double* bz, double* t, double tend, double* dt) {
  static_cast<OracleCy*>(h)->step(uh, br, bz, t, tend, dt);
  return 0;
}
int orc_cy_diagnostics(void* h, const double* uh, double* umax, double* totaldiv, double* pmin) {
  static_cast<OracleCy*>(h)->diagnostics(uh, umax, totaldiv, pmin);
  return 0;
}
int orc_cy_l2_error(void* h, int problem, const double* uh, double t, double* l2) {
  static_cast<OracleCy*>(h)->l2_error(problem, uh, t, l2);
  return 0;
}
#endif

}  // extern "C"
