/*
 * gdf_cy.h - C ABI of the B200 (sm_100a) implementation of the cylindrical
 * variant of the globally divergence-free DG MHD method,
 * MHD_GDF_cy3D_0421/ of L1ssandra/Freljord-CFD-arsenal: ideal MHD in
 * (r, z, phi) with a modal P2 solution in the (r, z) plane (dimPk1 = 6 test
 * functions, the cubic modes carried by the divergence-free B), 2*Lphi
 * planes in phi coupled by a Fourier derivative (Lh.f90:96-126), the
 * geometric source terms of the conservative cylindrical form
 * (Lh.f90:73-77), the optional manufactured-solution source (Source.f90,
 * RHSCopen), HLL/LF fluxes with local Lax-Friedrichs edge electric fields
 * (LhEz.f90:5-34) and the 2-D LF vertex field (LF_Flux_2D.f90), SSP-RK3
 * (RK3.f90), the characteristic TVB limiter on B = rB/r (TVB_Limiter_P2.f90)
 * with face-B minmod, and Balsara's reconstruction of rB from the faces and
 * d(Bphi)/dphi (div_free_Balsara.f90).
 *
 * Arrays are the reference's COMMON arrays (com.txt:36-68) in Fortran order
 * with its extents, NPH = 2*Lphi:
 *
 *   uh : real(8) uh(0:Nr+1, 0:Nz+1, 0:NPH-1, 10, 8)
 *        index  i + (Nr+2)*(j + (Nz+2)*(kk + NPH*((d-1) + 10*(n-1))))
 *        n = 6, 7 hold r*B_r and r*B_z, n = 8 holds B_phi
 *   Br : real(8) Br(0:Nr, 1:Nz, 0:NPH-1, 3)
 *        index  i + (Nr+1)*((j-1) + Nz*(kk + NPH*(d-1)))   (r*B_r on r-faces)
 *   Bz : real(8) Bz(1:Nr, 0:Nz, 0:NPH-1, 3)
 *        index  (i-1) + Nr*(j + (Nz+1)*(kk + NPH*(d-1)))   (r*B_z on z-faces)
 *   du : as uh; dBr as Br; dBz as Bz.
 *
 * Slots the method keeps at zero (modes 7-10 of n = 1-5 and 8, mode 10 of
 * n = 6, mode 7 of n = 7) must be zero on upload (GDF_ERR_ARG otherwise)
 * and are zero on download. Ghost cells (i = 0, Nr+1 or j = 0, Nz+1) are
 * refreshed by set_bc before every use and carry no state. Status codes,
 * gdf_last_error(), threading and synchronisation are those of gdf.h.
 */
#ifndef GDF_CY_H
#define GDF_CY_H

#include <stdint.h>

#include "gdf.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Problems of init_data.f90:6-14 (init0.txt .. init7.txt). */
enum {
  GDF_CY_SMOOTH_VORTEX = 0,  /* init0.txt */
  GDF_CY_SIN3D = 1,          /* init1.txt: manufactured solution, RHSCopen */
  GDF_CY_DIV_TEST = 2,       /* init2.txt */
  GDF_CY_ORSZAG_TANG = 3,    /* init3.txt: the reference's main.f90 case   */
  GDF_CY_ORSZAG_TANG2 = 4,   /* init4.txt */
  GDF_CY_EXPLOSION = 5,      /* init5.txt */
  GDF_CY_ROTOR = 6,          /* init6.txt */
  GDF_CY_JET = 7             /* init7.txt: force-free B_phi = 1/r          */
};

/* Boundary codes of set_bc.f90: r sides 1 periodic, 2 mirror extension
 * (evenex), 3 axis (evenex/oddex, left side only), 4 periodic with r*B
 * rescaled by rb/ra, 5 periodic with B_phi = 1/r at the edge; z sides
 * 1 periodic, 2 copy, 4 copy with the jet inlet (bottom only). */
typedef struct GdfCyConfig {
  int32_t nr, nz, lphi;       /* com.txt:1 Nr, Nz, Lphi (1, 2, 4 or 8)       */
  int32_t bc_r, bc_l, bc_u, bc_d;
  int32_t flux_type;          /* Lh.f90:316-328: 0 central, 1 LF, 2 HLL       */
  int32_t rhsc_open;          /* Lh.f90:80, LhEz.f90:174: source S1..S7        */
  int32_t reserved_i;
  double ra, rb, za, zb;      /* init*.txt domain                              */
  double gamma;               /* com.txt:26                                    */
  double cfl;                 /* calculate_dt.f90:8 (0.2)                      */
  double tvb_m;               /* init*.txt M (minmod.f90, minmodB.f90)          */
  double change_tol;          /* TVB_Limiter_P2.f90:75 (1e-6)                   */
  double jet_r;               /* set_bc.f90:76 inlet radius (1.5)               */
  double reserved_d[3];
} GdfCyConfig;

/* Preset of a problem on an nr x nz x 2*lphi grid (the init*.txt include of
 * init_data.f90:16): domain, boundaries, M, RHSCopen; HLL, CFL 0.2,
 * gamma 5/3. *tend receives the problem's end time. */
int gdf_cy_config_problem(int32_t problem, int32_t nr, int32_t nz, int32_t lphi,
                          GdfCyConfig *cfg, double *tend);

/* Host initial data (init_data.f90:18-139): L2 projection of the cells
 * (5x5 Gauss, dimPk1 modes) and of the faces, or the point values of the
 * shock problems. Arrays in the layouts above; uh's ghost cells are zero. */
int gdf_cy_init_data(const GdfCyConfig *cfg, int32_t problem, double *uh,
                     double *br, double *bz);

typedef struct GdfCyHandle GdfCyHandle;

int gdf_cy_create(const GdfCyConfig *cfg, GdfCyHandle **out);
int gdf_cy_destroy(GdfCyHandle *h);
int gdf_cy_upload(GdfCyHandle *h, const double *uh, const double *br, const double *bz);
int gdf_cy_download(GdfCyHandle *h, double *uh, double *br, double *bz);
int gdf_cy_set_time(GdfCyHandle *h, double t);
int gdf_cy_get_time(GdfCyHandle *h, double *t);

/* The start of RK3 (RK3.f90:8-10): TVB_Limiter_P2 and div_free_Balsara on
 * the uploaded state. */
int gdf_cy_prepare(GdfCyHandle *h);

/* One time step (RK3.f90:42-138): dt from calculate_dt, clipped at tend,
 * three stages each followed by the limiter and the reconstruction. */
int gdf_cy_step(GdfCyHandle *h, double tend, double *t, double *dt);

/* Up to max_steps steps, graph-replayed, stopping once t reaches tend. */
int gdf_cy_advance(GdfCyHandle *h, double tend, int32_t max_steps, double *t,
                   int32_t *steps);

/* `steps` graph replays without a host synchronisation between them, timed
 * with CUDA events on the handle's stream: *ms the device time, *steps_taken
 * the steps that advanced t (replays after t reaches tend do nothing). */
int gdf_cy_advance_timed(GdfCyHandle *h, double tend, int32_t steps, double *t,
                         int32_t *steps_taken, double *ms);

/* Lh then LhEz on the given state at source time t_rk (set_bc applied to a
 * device copy): du, dBr, dBz in the layouts above. */
int gdf_cy_lh(GdfCyHandle *h, const double *uh, const double *br, const double *bz,
              double t_rk, double *du, double *dbr, double *dbz);

/* TVB_Limiter_P2 then div_free_Balsara on the given state, in place. */
int gdf_cy_limit(GdfCyHandle *h, double *uh, double *br, double *bz);

/* calculate_dt of the given state. */
int gdf_cy_dt(GdfCyHandle *h, const double *uh, double *dt);

/* calculate_umax, calculate_totaldiv and calculate_pmin of the handle's
 * state (any pointer may be NULL). */
int gdf_cy_diagnostics(GdfCyHandle *h, double *umax, double *totaldiv, double *pmin);

/* Kernels launched by the handle so far. */
int gdf_cy_kernel_launches(GdfCyHandle *h, int64_t *n);

#ifdef __cplusplus
}
#endif

#endif /* GDF_CY_H */
