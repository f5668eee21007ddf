// gdf_p3_basis.h -- the k = 3 variant's basis tables (get_basis,
// MPI_BalsaraP3/main.f90:782-1119) as one plain struct, built on the host
// (gdf_host.cpp, no FMA contraction) and passed to every P3 kernel by value.
#pragma once

namespace gdf3 {

constexpr int NG = 5;     // NumGLP
constexpr int NP3 = 15;   // dimPk for kk = 3
constexpr int NQ3 = 10;   // dimPk1: the solution's modes (test functions of Lh)
constexpr int NB3 = 4;    // kk + 1 face modes
constexpr int NE = 8;     // NumEq

struct BasisP3 {
  double lambda[NG], weight[NG];
  // phiG(i,j,d) as phiG[i-1][j-1][d-1]; the derivative tables include 1/hx1, 1/hy1
  double phiG[NG][NG][NP3], phixG[NG][NG][NP3], phiyG[NG][NG][NP3];
  // x faces indexed by the y point, y faces by the x point
  double phiGR[NG][NP3], phiGL[NG][NP3], phiGU[NG][NP3], phiGD[NG][NP3];
  double phiRU[NP3], phiLU[NP3], phiRD[NP3], phiLD[NP3], mm[NP3];
  // edge basis, its derivatives along the edge, end values, mass
  double EzG[NG][NB3], EzxG[NG][NB3], EzyG[NG][NB3], EzR[NB3], EzL[NB3], mmE[NB3];
};

// get_basis for cells of half-widths hx1, hy1 (host)
void build_basis_p3(double hx1, double hy1, BasisP3* b);

}  // namespace gdf3
