// gdf_kernels.cuh -- device data layout and kernel declarations of the
// B200 GDF P2 step.
//
// Layout in HBM (all FP64):
//   U, U0, UI : the reference's uh(0:Nx+1, 0:Ny+1, 10, 8) in Fortran order,
//               i.e. one (Nx+2)x(Ny+2) plane per (mode, variable) slot with
//               i fastest. Only the 52 live slots are ever read or written;
//               the 28 dead slots stay zero. U is the limited stage state,
//               U0 the step's initial state (uh0), UI the pre-limit stage
//               state (uI / uII of RK3.f90).
//   BX*, BY*  : Bx(0:Nx,1:Ny,3) and By(1:Nx,0:Ny,3), Fortran order.
//   Fxh       : Fxhat as 40 planes (n*5 + g) of (Nx+1) x Ny, i fastest.
//   Fyh       : Fyhat as 40 planes of Nx x (Ny+1).
//   EzRL/EzUD : 5 planes each; EzV : (Nx+1) x (Ny+1).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

#include "../../include/gdf.h"

#include "gdf_physics.cuh"

namespace gdf {

constexpr int NLIVE = 52;

// Per-handle constants, passed to every kernel by value (__grid_constant__).
struct Consts {
  Phys P;
  int nx, ny, nx2, ny2;
  long long plane, fxplane, fyplane, vplane;
  double hx, hy, hx1, hy1;
  double cxs, cys;          // 0.5/hx, 0.5/hy (Lh.f90:275,291)
  double Mh2x, Mh2y;        // M*hx**2, M*hy**2 (minmod.f90:10)
  double Mh2x_b, Mh2y_b;    // minmodB bounds: M*hy**2 for Bx, M*hx**2 for By
  double rxy, ryx;          // hx/hy, hy/hx (div_free_Balsara.f90:36-37)
  double tvb_slope, cfl, ck, pow_hxhy;
  int bc_r, bc_l, bc_u, bc_d;
  int pp, faceb, ez_fhat, eig_y_zero_w, detector, sticky, dt_floor_stop, umax_all;
  int tvb_p1;               // TVB_Limiter_P1 in place of TVB_Limiter_P2
  double w[NG], lam[NG];
  double phiG[NG][NG][NP], phix[NG][NG][NP], phiy[NG][NG][NP];
  double phiGLL[2][NG][NG][NP];
  double ppM[NP];           // max over the 50 GLL-mixed points of |phiGLL(.,.,d,.)|
  double phiGR[NG][NP], phiGL[NG][NP], phiGU[NG][NP], phiGD[NG][NP];
  double phiRU[NP], phiLU[NP], phiRD[NP], phiLD[NP];
  double mm[NP];
  double EzxG[NG][3], EzyG[NG][3], mmE[3], EzR[3], EzL[3], EzU[3], EzD[3];
};

// The grid-independent basis tables (get_GLP.f90, get_basis.f90 on the
// reference element): the same for every configuration, so the device holds
// one copy (gdf_device.cuh c_basis) that every kernel reads from constant
// memory. Consts keeps its own copy for the host.
struct Basis {
  double w[NG], lam[NG];
  double phiG[NG][NG][NP];
  double phiGLL[2][NG][NG][NP];
  double ppM[NP];
  double phiGR[NG][NP], phiGL[NG][NP], phiGU[NG][NP], phiGD[NG][NP];
  double phiRU[NP], phiLU[NP], phiRD[NP], phiLD[NP];
  double mm[NP];
  double mmE[3], EzR[3], EzL[3], EzU[3], EzD[3];
};

// Device-resident time state of a handle (RK3.f90 t, dt).
struct Scal {
  double t, dt, tend;
  double umax, totaldiv, pmin;
  int active;         // 1 while the current step is running
  int status;         // bit 0: non-finite / non-positive state seen
  long long steps;    // steps taken since upload
  long long troubled; // cells flagged by the last step
};

// Host helpers shared by the single-problem handle and the ensemble
// (gdf_kernels.cu): the constants of a configuration, and the checks of a
// configuration and of an uploaded state (0 or a GDF_ERR_* code with msg).
void consts_for(const GdfConfig& c, Consts& K);
void basis_of(const Consts& K, Basis& B);
int config_error(const GdfConfig* c, std::string& msg);
int dead_slot_error(const GdfConfig& c, const double* uh, std::string& msg);

}  // namespace gdf
