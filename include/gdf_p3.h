/*
 * gdf_p3.h - C ABI of the B200 (sm_100a) implementation of the third-order
 * (k = 3) variant of the 2-D ideal-MHD globally divergence-free DG method,
 * MPI_BalsaraP3/main.f90 of L1ssandra/Freljord-CFD-arsenal: modal P3
 * solution (dimPk = 15 slots, the degree-4 ones carried by the
 * divergence-free B), four-mode face B, 5-point Gauss quadrature, the
 * ten-stage fourth-order SSP Runge-Kutta loop (RK4, main.f90:1315-1431), a
 * characteristic TVB limiter with the P3 reconstruction on every cell
 * (TVB_Limiter, main.f90:3283-3482) and Balsara's reconstruction of the
 * cell B (div_free_Balsara, main.f90:3108-3233).
 *
 * The reference runs one MPI rank per block of a 2-D decomposition with
 * Nphi = 0; on one device the whole grid is one block, and the arrays below
 * are the reference's per-rank arrays of a single-rank run, in Fortran
 * order with the reference's extents (main.f90:25-35, the phi index of
 * extent 1 dropped):
 *
 *   uh : real(8) uh(0:Nx+1, 0:Ny+1, 15, 8)
 *        index  i + (Nx+2)*(j + (Ny+2)*((d-1) + 15*(n-1)))
 *   Bx : real(8) Bx(0:Nx, 0:Ny+1, 4)  index i + (Nx+1)*(j + (Ny+2)*(d-1))
 *   By : real(8) By(0:Nx+1, 0:Ny, 4)  index i + (Nx+2)*(j + (Ny+1)*(d-1))
 *   du : as uh; dBx as Bx; dBy as By.
 *
 * Slots that the method keeps at zero (modes 11-15 of rho, rhou, rhov,
 * rhow, E, Bz; modes 12, 13, 15 of the cell Bx; 11, 13, 14 of the cell By)
 * must be zero on upload (GDF_ERR_ARG otherwise) and are zero on download.
 * Status codes, gdf_last_error(), threading and synchronisation are those of
 * gdf.h.
 */
#ifndef GDF_P3_H
#define GDF_P3_H

#include <stdint.h>

#include "gdf.h"

#ifdef __cplusplus
extern "C" {
#endif

/*
 * Run-time configuration. The reference fixes these at compile time
 * (main.f90:9 flux_type, :19 gamma, :1319 CFL) or per initial-data module
 * (mesh: domain, boundaries, tend, M and beta; :126-155, 197-226, 310-339,
 * 458-489); gdf_p3_config_problem() fills them for a problem.
 */
typedef struct GdfP3Config {
  int32_t nx, ny;            /* main.f90:9 Nx0, Ny0 (one block)               */
  double xa, xb, ya, yb;     /* mesh                                          */
  int32_t bc_r, bc_l, bc_u, bc_d; /* GDF_BC_* (bcR, bcL, bcU, bcD)           */
  int32_t flux_type;         /* GDF_FLUX_* (main.f90:9: HLL)                  */
  double gamma;              /* main.f90:19: 5/3                              */
  double cfl;                /* RK4: 0.75 (main.f90:1319)                     */
  double tvb_m;              /* M of the TVB minmod                           */
  double tvb_beta;           /* beta of minmod/minmodB (main.f90:3971,3995)   */
  double hlld_eps;           /* HLLD second-stage threshold (:2495): 1e-6     */
  double change_tol;         /* limiter change test (:3330): 1e-13            */
  /* a block of a decomposed grid: the cell width is that of the whole grid,
   * (xb - xa) / nx_global with xa, xb the whole domain (main.f90:565-566
   * use Nx0, Ny0); 0 for a grid that is one block */
  int32_t nx_global, ny_global;
  int32_t reserved[2];
} GdfP3Config;

typedef struct GdfP3Handle GdfP3Handle;

/* Fill cfg for problem GDF_PROB_VORTEX (module init1), GDF_PROB_ORSZAG_TANG
 * (init3), GDF_PROB_ROTOR (init4) or GDF_PROB_CLOUD_SHOCK (init6) on an
 * nx x ny grid; *tend (may be NULL) gets the module's end time. */
int gdf_p3_config_problem(int32_t problem, int32_t nx, int32_t ny, GdfP3Config* cfg, double* tend);

/* init_data (main.f90:534-661) on the host: L2 projection of the problem's
 * conserved variables on modes 1-10 (5 x 5 Gauss points) and of the face
 * fields on the four edge modes; ghost slots left zero. */
int gdf_p3_init_data(const GdfP3Config* cfg, int32_t problem, double* uh, double* bx, double* by);

int gdf_p3_create(const GdfP3Config* cfg, GdfP3Handle** out);
int gdf_p3_destroy(GdfP3Handle* h);

/* Copy the state in (t set to 0) or out. */
int gdf_p3_upload(GdfP3Handle* h, const double* uh, const double* bx, const double* by);
int gdf_p3_download(GdfP3Handle* h, double* uh, double* bx, double* by);
int gdf_p3_set_time(GdfP3Handle* h, double t);

/* RK4's start (main.f90:1322-1324): TVB_Limiter then div_free_Balsara on
 * the uploaded state. */
int gdf_p3_prepare(GdfP3Handle* h);

/* One pass of RK4's loop body (main.f90:1335-1423): calculate_dt, the
 * clamp to tend, ten Lh stages with their limiting. *t and *dt may be NULL. */
int gdf_p3_step(GdfP3Handle* h, double tend, double* t, double* dt);

/* Steps until t >= tend or max_steps, replaying one CUDA graph per step. */
int gdf_p3_advance(GdfP3Handle* h, double tend, int32_t max_steps, double* t, int32_t* steps);

/* gdf_p3_advance over exactly `steps` graph replays, timed with CUDA
 * events on the handle's stream around them (*ms, device milliseconds). */
int gdf_p3_advance_timed(GdfP3Handle* h, double tend, int32_t steps, double* t, int32_t* steps_taken, double* ms);

/* Kernel launches issued on this handle so far (graph replays count each
 * node). */
int64_t gdf_p3_kernel_launches(GdfP3Handle* h);

/*
 * Stage-level control, for a block of a grid decomposed over several
 * devices (the reference's MPI ranks, main.f90:8-11): the caller fills the
 * ghost layers between the calls (set_bc's exchange, main.f90:1574-1867)
 * and reduces the speeds over the blocks (calculate_dt's MPI maximum,
 * :1492-1538). One step: gdf_p3_step_speeds on every block, the maxima,
 * gdf_p3_step_begin, then for stage s = 1..10: fill the ghosts of U, then
 * gdf_p3_stage_lh(s); unless s == 5: fill the ghosts of T (cells) and of
 * BXT/BYT (Bx ghost rows, By ghost columns), then gdf_p3_stage_limit.
 * Device arrays (gdf_p3_block_arrays): U, T as 84 slot planes of
 * (Nx+2) x (Ny+2) (slot order: modes 1-10 of each variable, then Bx modes 11,
 * 14 after Bx's ten and By modes 12, 15 after By's ten), BX, BXT, BY, BYT in
 * the host layout of Bx, By. The calls are asynchronous on the handle's
 * stream (gdf_p3_stream) except step_speeds and step_begin, which return
 * values.
 */
int gdf_p3_block_arrays(GdfP3Handle* h, double** U, double** T, double** BX, double** BY, double** BXT,
                        double** BYT);
void* gdf_p3_stream(GdfP3Handle* h);
int gdf_p3_step_speeds(GdfP3Handle* h, double* ax, double* ay);
int gdf_p3_step_begin(GdfP3Handle* h, double ax, double ay, double tend, double* t, double* dt);
int gdf_p3_stage_lh(GdfP3Handle* h, int32_t stage);
int gdf_p3_stage_limit(GdfP3Handle* h);
/* T = U, BXT = BX, BYT = BY: with a ghost fill of T and gdf_p3_stage_limit,
 * the block's part of gdf_p3_prepare */
int gdf_p3_stage_load_t(GdfP3Handle* h);

/* The three calls below take a state from the caller, which replaces the
 * handle's resident state. */

/* Lh (main.f90:1871-2350) of the given state: set_bc, then du, dBx, dBy
 * (ghost cells, ghost face rows and modes 11-15 of du are 0). */
int gdf_p3_lh(GdfP3Handle* h, const double* uh, const double* bx, const double* by, double* du, double* dbx,
              double* dby);

/* TVB_Limiter then div_free_Balsara on the given state, in place (interior
 * cells and every face; the ghost cells come back as set_bc left them). */
int gdf_p3_limit(GdfP3Handle* h, double* uh, double* bx, double* by);

/* calculate_dt (main.f90:1469-1541) of the given state. */
int gdf_p3_dt(GdfP3Handle* h, const double* uh, double* dt);

/* calculate_umax (max |rho mean|) and calculate_totaldiv of the resident
 * state (main.f90:1433-1465, 3235-3279). */
int gdf_p3_diagnostics(GdfP3Handle* h, double* umax, double* totaldiv);

#ifdef __cplusplus
}
#endif

#endif /* GDF_P3_H */
