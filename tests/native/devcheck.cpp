// Host build of the library's pointwise physics (gdf_physics.cuh) for the
// CPU tests: the same source the sm_100a kernels compile, compiled here
// without FMA contraction and compared value-for-value with the oracle.
#include "../../freljord-cfd-arsenal_b200/csrc/gdf_physics.cuh"

using gdf::Phys;

static Phys mk(const double* prm, const int* iprm) {
  Phys P;
  P.gamma = prm[0];
  P.gamma1 = prm[0] - 1;
  P.gflux = prm[1];
  P.hlld_eps = prm[2];
  P.flux = iprm[0];
  P.kml_w = iprm[1];
  P.eig_p_typo = iprm[2];
  P.eig_identity = iprm[3];
  return P;
}

extern "C" {
// prm = {gamma, gamma_flux, hlld_eps}, iprm = {flux, kml_w, eig_p_typo, eig_identity}
void dev_face_flux(const double* prm, const int* iprm, const double* ul, const double* ur, int dir1, double* fh) {
  Phys P = mk(prm, iprm);
  double fl[8], fr[8];
  gdf::face_flux(P, ul, ur, dir1 - 1, fh, fl, fr);
}
double dev_vertex_ez(const double* prm, const int* iprm, const double* uru, const double* ulu, const double* urd,
                     const double* uld) {
  Phys P = mk(prm, iprm);
  return gdf::vertex_ez(P, uru, ulu, urd, uld);
}
void dev_eigenmatrix(const double* prm, const int* iprm, int dir1, const double* prim8, double* R, double* L) {
  Phys P = mk(prm, iprm);
  gdf::eigenmatrix(P, dir1 - 1, prim8[0], prim8[1], prim8[2], prim8[3], prim8[4], prim8[5], prim8[6], prim8[7], R, L);
}
void dev_eigenvalue(const double* prm, const int* iprm, const double* U, int dir1, double* amax, double* amin) {
  Phys P = mk(prm, iprm);
  gdf::fast_speeds(P, U, dir1 - 1, *amax, *amin);
}
}
