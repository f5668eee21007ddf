// gdf_cy_host.cpp -- host side of the cylindrical variant's C ABI that needs
// no device: the problem presets (the init*.txt includes of
// MHD_GDF_cy3D_0421/init_data.f90:16) and the initial data
// (init_data.f90:18-139). Compiled without FMA contraction so the
// projections round as the reference's loops do.

#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/gdf_cy.h"

namespace {

constexpr int NG = 5, NPC = 10, NQC = 6, NE = 8;

const double kLam[NG] = {-0.9061798459386639927976269, -0.5384693101056830910363144, 0,
                         0.5384693101056830910363144, 0.9061798459386639927976269};
const double kW[NG] = {0.2369268850561890875142640, 0.4786286704993664680412915, 0.5688888888888888888888889,
                       0.4786286704993664680412915, 0.2369268850561890875142640};

inline double sq(double x) { return x * x; }

// The conserved U1..U8 of init0.txt .. init7.txt at (r, z, phi). The files
// write U6, U7 as r*B1, r*B2, except init0, init6 and init7, which write
// B1, B2 (kept as written).
void problem_U(int prob, double g, double r, double z, double phi, double* U) {
  const double pi = 4 * std::atan(1.0), g1 = g - 1;
  double p = 0, rho = 1, v1 = 0, v2 = 0, v3 = 0, B1 = 0, B2 = 0, B3 = 0;
  bool times_r = true;
  if (prob == GDF_CY_SMOOTH_VORTEX) {          // init0.txt: the file's (x, y) are (r, z)
    const double r2 = r * r + z * z;
    const double e = std::exp(0.5 * (1 - r2));
    p = 1 - r2 / (8.0 * sq(pi)) * std::exp(1 - r2);
    v1 = 1 - 1.0 / (2.0 * pi) * z * e;
    v2 = 1 + 1.0 / (2.0 * pi) * r * e;
    B1 = -(1.0 / (2.0 * pi) * z * e);
    B2 = 1.0 / (2.0 * pi) * r * e;
    times_r = false;
  } else if (prob == GDF_CY_SIN3D) {           // init1.txt
    p = 1; rho = 1 + 0.5 * std::sin(r + z); v1 = 1; v2 = 1;
    B1 = -(0.5 * std::sin(z) * std::cos(phi));
    B2 = 0.5 * std::sin(r) * std::cos(phi);
    B3 = 0.5 * std::sin(z) * std::sin(phi);
  } else if (prob == GDF_CY_DIV_TEST) {        // init2.txt
    p = 1; rho = 1 + 0.5 * std::sin(r + z); v1 = 1; v2 = 1;
    B1 = std::sin(r) * std::sin(z) * std::sin(phi);
    B2 = std::cos(r) * std::cos(z) * std::sin(phi);
    B3 = std::sin(r) * std::sin(z) * std::cos(phi);
  } else if (prob == GDF_CY_ORSZAG_TANG) {     // init3.txt
    p = g; rho = g * g; v1 = -std::sin(z); v2 = std::sin(r);
    B1 = -(6 * pi * std::sin(z) / r);
    B2 = 6 * pi * std::sin(2 * r) / r;
  } else if (prob == GDF_CY_ORSZAG_TANG2) {    // init4.txt
    p = g; rho = g * g; v1 = -std::sin(z); v2 = std::sin(r);
    B1 = -(std::sin(z) * std::cos(phi));
    B2 = std::sin(2 * r) * std::cos(phi);
    B3 = std::sin(z) * std::sin(phi);
  } else if (prob == GDF_CY_EXPLOSION) {       // init5.txt, vjet.f90 pS
    const double rr = std::sqrt(sq(r - 0.5) + sq(z));
    p = (rr > 0.1) ? 0.1 : 10;
    B2 = 1;
  } else if (prob == GDF_CY_ROTOR) {           // init6.txt, Rotor_functions.f90 (centre (1.5, 0.5))
    const double rr = std::sqrt(sq(r - 1.5) + sq(z - 0.5)), r0 = 0.1, r1 = 0.115;
    const double f = (r1 - rr) / (r1 - r0);
    if (rr < r0) {
      rho = 10.0; v1 = -(2 * (z - 0.5) / r0); v2 = 2 * (r - 1.5) / r0;
    } else if (rr >= r0 && rr < r1) {
      rho = 1.0 + 9.0 * f; v1 = -(2 * f * (z - 0.5) / rr); v2 = 2 * f * (r - 1.5) / rr;
    } else {
      rho = 1.0;
    }
    p = 0.5; B2 = 2.4 / std::sqrt(4 * pi);
    times_r = false;
  } else {                                     // init7.txt
    p = 1; B3 = 1.0 / r;
    times_r = false;
  }
  U[0] = rho;
  U[1] = rho * v1;
  U[2] = rho * v2;
  U[3] = rho * v3;
  U[4] = p / g1 + 0.5 * rho * (sq(v1) + sq(v2) + sq(v3)) + 0.5 * (sq(B1) + sq(B2) + sq(B3));
  U[5] = times_r ? r * B1 : B1;
  U[6] = times_r ? r * B2 : B2;
  U[7] = B3;
}

// phiG(i1, j1, d) for d = 1..6 and EzG(i1, d) (get_basis.f90:49-164)
double phiG(int a, int b, int d) {
  const double li = kLam[a], lj = kLam[b], c13 = 1.0 / 3.0;
  switch (d) {
    case 0: return 1;
    case 1: return li;
    case 2: return lj;
    case 3: return sq(li) - c13;
    case 4: return li * lj;
    default: return sq(lj) - c13;
  }
}
double EzG(int a, int d) { return d == 0 ? 1 : (d == 1 ? kLam[a] : sq(kLam[a]) - 1.0 / 3.0); }
const double kMM[NQC] = {1, 1.0 / 3.0, 1.0 / 3.0, 4.0 / 45.0, 1.0 / 9.0, 4.0 / 45.0};
const double kMME[3] = {1, 1.0 / 3.0, 4.0 / 45.0};

bool valid(const GdfCyConfig* c) {
  if (!c || c->nr < 2 || c->nz < 2) return false;
  if (c->lphi != 1 && c->lphi != 2 && c->lphi != 4 && c->lphi != 8) return false;
  if (!(c->rb > c->ra) || !(c->zb > c->za)) return false;
  return true;
}

}  // namespace

extern "C" {

// init0.txt .. init7.txt: domain, boundaries, end time, M, RHSCopen
int gdf_cy_config_problem(int32_t problem, int32_t nr, int32_t nz, int32_t lphi, GdfCyConfig* cfg, double* tend) {
  if (!cfg || nr < 2 || nz < 2 || (lphi != 1 && lphi != 2 && lphi != 4 && lphi != 8)) return GDF_ERR_ARG;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->nr = nr;
  cfg->nz = nz;
  cfg->lphi = lphi;
  cfg->flux_type = 2;          // com.txt:1 flux_type = 2 (HLL)
  cfg->gamma = 5.0 / 3.0;      // com.txt:26
  cfg->cfl = 0.2;              // calculate_dt.f90:11 (RKorder 3)
  cfg->change_tol = 1e-6;      // TVB_Limiter_P2.f90:75
  cfg->jet_r = 1.5;            // set_bc.f90:76
  const double pi = 4 * std::atan(1.0);
  double te = 0;
  int bc[4] = {1, 1, 1, 1};    // R, L, U, D
  switch (problem) {
    case GDF_CY_SMOOTH_VORTEX:
      cfg->ra = -5; cfg->rb = 5; cfg->za = -5; cfg->zb = 5; te = 1; cfg->tvb_m = 1000000;
      break;
    case GDF_CY_SIN3D:
    case GDF_CY_DIV_TEST:
      cfg->ra = 2 * pi; cfg->rb = 4 * pi; cfg->za = 0; cfg->zb = 2 * pi;
      te = problem == GDF_CY_SIN3D ? 1 : 0;
      cfg->tvb_m = 1000000; cfg->rhsc_open = 1;
      bc[0] = bc[1] = 4;
      break;
    case GDF_CY_ORSZAG_TANG:
      cfg->ra = 6 * pi; cfg->rb = 8 * pi; cfg->za = 0; cfg->zb = 2 * pi; te = 4; cfg->tvb_m = 10;
      break;
    case GDF_CY_ORSZAG_TANG2:
      cfg->ra = 10 * pi; cfg->rb = 12 * pi; cfg->za = 0; cfg->zb = 2 * pi; te = 0.5; cfg->tvb_m = 1;
      bc[0] = bc[1] = 4;
      break;
    case GDF_CY_EXPLOSION:
      cfg->ra = 0.1; cfg->rb = 1; cfg->za = -0.5; cfg->zb = 0.5; te = 0.001; cfg->tvb_m = 1;
      bc[0] = bc[1] = bc[2] = bc[3] = 2;
      break;
    case GDF_CY_ROTOR:
      cfg->ra = 1; cfg->rb = 2; cfg->za = 0; cfg->zb = 1; te = 0.015; cfg->tvb_m = 1;
      bc[0] = bc[1] = bc[2] = bc[3] = 2;
      break;
    case GDF_CY_JET:
      cfg->ra = 1; cfg->rb = 2; cfg->za = 0; cfg->zb = 1; te = 0.6; cfg->tvb_m = 1000000;
      bc[0] = bc[1] = 5; bc[2] = bc[3] = 2;
      break;
    default:
      return GDF_ERR_ARG;
  }
  cfg->bc_r = bc[0]; cfg->bc_l = bc[1]; cfg->bc_u = bc[2]; cfg->bc_d = bc[3];
  if (tend) *tend = te;
  return GDF_OK;
}

// init_data.f90:36-139: cells accumulate w(i1)*w(j1)*phiG*U over the 5x5
// Gauss points per mode, then 0.25*, then /mm; faces 0.5*w*U*EzG, /mmE;
// the shock problems (init5, init6) take the point values at the cell
// centres and face midpoints instead.
int gdf_cy_init_data(const GdfCyConfig* cfg, int32_t problem, double* uh, double* br, double* bz) {
  if (!valid(cfg) || !uh || !br || !bz || problem < 0 || problem > 7) return GDF_ERR_ARG;
  const int Nx = cfg->nr, Ny = cfg->nz, NPH = 2 * cfg->lphi;
  const double hr = (cfg->rb - cfg->ra) / Nx, hz = (cfg->zb - cfg->za) / Ny;
  const double pi = 4 * std::atan(1.0), hphi = 2 * pi / NPH;
  const double hr1 = 0.5 * hr, hz1 = 0.5 * hz;
  const size_t NX2 = (size_t)Nx + 2, NY2 = (size_t)Ny + 2, ncp = NX2 * NY2 * NPH;
  std::memset(uh, 0, ncp * NPC * NE * sizeof(double));
  const size_t nbr = (size_t)(Nx + 1) * Ny * NPH, nbz = (size_t)Nx * (Ny + 1) * NPH;
  std::memset(br, 0, nbr * 3 * sizeof(double));
  std::memset(bz, 0, nbz * 3 * sizeof(double));
  std::vector<double> Rc(Nx + 1), Zc(Ny + 1), Ph(NPH);
  for (int i = 1; i <= Nx; ++i) Rc[i] = cfg->ra + (i - 0.5) * hr;
  for (int j = 1; j <= Ny; ++j) Zc[j] = cfg->za + (j - 0.5) * hz;
  for (int k = 0; k < NPH; ++k) Ph[k] = k * hphi;
  const double g = cfg->gamma;
  auto U = [&](int i, int j, int kk, int d, int n) {
    return (size_t)i + NX2 * ((size_t)j + NY2 * ((size_t)kk + NPH * ((size_t)d + NPC * (size_t)n)));
  };
  auto BR = [&](int i, int j, int kk, int d) {
    return (size_t)i + (size_t)(Nx + 1) * ((size_t)(j - 1) + (size_t)Ny * ((size_t)kk + NPH * (size_t)d));
  };
  auto BZ = [&](int i, int j, int kk, int d) {
    return (size_t)(i - 1) + (size_t)Nx * ((size_t)j + (size_t)(Ny + 1) * ((size_t)kk + NPH * (size_t)d));
  };
  const bool shock = problem == GDF_CY_EXPLOSION || problem == GDF_CY_ROTOR;
  if (!shock) {
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= Ny; ++j)
      for (int i = 1; i <= Nx; ++i)
        for (int kk = 0; kk < NPH; ++kk) {
          double Uq[NG][NG][NE];
          for (int a = 0; a < NG; ++a)
            for (int b = 0; b < NG; ++b) problem_U(problem, g, Rc[i] + hr1 * kLam[a], Zc[j] + hz1 * kLam[b], Ph[kk], Uq[a][b]);
          for (int d = 0; d < NQC; ++d) {
            double acc[NE] = {0, 0, 0, 0, 0, 0, 0, 0};
            for (int a = 0; a < NG; ++a)
              for (int b = 0; b < NG; ++b) {
                const double wp = kW[a] * kW[b] * phiG(a, b, d);
                for (int n = 0; n < NE; ++n) acc[n] = acc[n] + wp * Uq[a][b][n];
              }
            for (int n = 0; n < NE; ++n) uh[U(i, j, kk, d, n)] = 0.25 * acc[n] / kMM[d];
          }
        }
    for (int kk = 0; kk < NPH; ++kk)
      for (int j = 1; j <= Ny; ++j)
        for (int i = 0; i <= Nx; ++i) {
          double Ub[NG][NE];
          for (int b = 0; b < NG; ++b) problem_U(problem, g, cfg->ra + i * hr, Zc[j] + hz1 * kLam[b], Ph[kk], Ub[b]);
          for (int d = 0; d < 3; ++d) {
            double acc = 0;
            for (int b = 0; b < NG; ++b) acc = acc + 0.5 * kW[b] * Ub[b][5] * EzG(b, d);
            br[BR(i, j, kk, d)] = acc / kMME[d];
          }
        }
    for (int kk = 0; kk < NPH; ++kk)
      for (int j = 0; j <= Ny; ++j)
        for (int i = 1; i <= Nx; ++i) {
          double Ua[NG][NE];
          for (int a = 0; a < NG; ++a) problem_U(problem, g, Rc[i] + hr1 * kLam[a], cfg->za + j * hz, Ph[kk], Ua[a]);
          for (int d = 0; d < 3; ++d) {
            double acc = 0;
            for (int a = 0; a < NG; ++a) acc = acc + 0.5 * kW[a] * Ua[a][6] * EzG(a, d);
            bz[BZ(i, j, kk, d)] = acc / kMME[d];
          }
        }
    return GDF_OK;
  }
  double Uv[NE];
  for (int kk = 0; kk < NPH; ++kk)
    for (int j = 1; j <= Ny; ++j)
      for (int i = 1; i <= Nx; ++i) {
        problem_U(problem, g, Rc[i], Zc[j], Ph[kk], Uv);
        for (int n = 0; n < NE; ++n) uh[U(i, j, kk, 0, n)] = Uv[n];
      }
  for (int kk = 0; kk < NPH; ++kk)
    for (int j = 1; j <= Ny; ++j)
      for (int i = 0; i <= Nx; ++i) {
        problem_U(problem, g, cfg->ra + i * hr, Zc[j], Ph[kk], Uv);
        br[BR(i, j, kk, 0)] = Uv[5];
      }
  for (int kk = 0; kk < NPH; ++kk)
    for (int j = 0; j <= Ny; ++j)
      for (int i = 1; i <= Nx; ++i) {
        problem_U(problem, g, Rc[i], cfg->za + j * hz, Ph[kk], Uv);
        bz[BZ(i, j, kk, 0)] = Uv[6];
      }
  return GDF_OK;
}

}  // extern "C"
