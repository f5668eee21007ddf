/*
 * gdf.h - C ABI of the B200 (sm_100a) implementation of the 2-D ideal-MHD
 * P2 discontinuous-Galerkin step with globally divergence-free (Balsara)
 * constrained transport, as in GDF_Balsara_P2_0316/ of
 * L1ssandra/Freljord-CFD-arsenal.
 *
 * The reference has no foreign-function interface: its "API" is a set of
 * argument-less Fortran subroutines sharing COMMON blocks (com.txt:19-54),
 * driven by main.f90:1-23 -> RK3.f90. Every entry point below replaces one
 * of those subroutines (cited per function) and takes the reference's
 * arrays in Fortran (column-major) order with the reference's extents, so
 * a Fortran host can pass its COMMON arrays through iso_c_binding unchanged:
 *
 *   uh : real(8) uh(0:Nx+1, 0:Ny+1, 10, 8)
 *        index  i + (Nx+2)*(j + (Ny+2)*((d-1) + 10*(n-1)))   (i,j from 0)
 *   Bx : real(8) Bx(0:Nx, 1:Ny, 3)      index i + (Nx+1)*((j-1) + Ny*(d-1))
 *   By : real(8) By(1:Nx, 0:Ny, 3)      index (i-1) + Nx*(j + (Ny+1)*(d-1))
 *   du : same extents as uh; dEz1 as Bx; dEz2 as By.
 *   flags : int32 flags(1:Nx, 1:Ny)     index (i-1) + Nx*(j-1)
 *
 * All arithmetic on the solver path is IEEE binary64. Every call returns an
 * int status: GDF_OK (0) or a GDF_ERR_* code; gdf_last_error() gives the
 * message of the last failure on the calling thread. Calls on one handle
 * are not thread-safe; each handle owns its device memory and one CUDA
 * stream, and every call is synchronous at return.
 */
#ifndef GDF_H
#define GDF_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GDF_ABI_VERSION 1

enum {
  GDF_OK = 0,
  GDF_ERR_ARG = 1,      /* bad argument or configuration                  */
  GDF_ERR_CUDA = 2,     /* CUDA runtime failure (message has the detail)  */
  GDF_ERR_NUMERIC = 3,  /* non-finite state or non-positive dt detected   */
  GDF_ERR_TIMEOUT = 4,  /* a bounded device wait gave up                  */
  GDF_ERR_NOMEM = 5,    /* device allocation failed                       */
  GDF_ERR_STATE = 6     /* call out of order (e.g. step before upload)    */
};

/* Numerical flux (com.txt:1 flux_type; Lh.f90:220-230, LhEz.f90:57-65). */
enum { GDF_FLUX_LF = 1, GDF_FLUX_HLL = 2, GDF_FLUX_HLLC = 3, GDF_FLUX_HLLD = 4 };

/* Boundary conditions (set_bc.f90:5-27). */
enum { GDF_BC_PERIODIC = 1, GDF_BC_OUTFLOW = 2 };

/* Troubled-cell detector feeding the characteristic limiter
 * (TVB_Limiter_P2.f90:12,22). */
enum {
  GDF_DETECT_ALL = 0,    /* reference as shipped: every cell is limited    */
  GDF_DETECT_KXRCF = 1,  /* KXRCF_Detector.f90 gates the limiter           */
  GDF_DETECT_LEARNED = 2 /* the learned indicator (gdf_set_indicator) gates
                            the limiter; KXRCF decides where it is unsure  */
};

/* Initial-data problems (init_data.f90:3-19 include list; sizes and
 * parameters of the benchmark problems are set by the caller). */
enum {
  GDF_PROB_VORTEX = 0,      /* init1.txt smooth MHD vortex                 */
  GDF_PROB_ORSZAG_TANG = 1, /* init3.txt                                   */
  GDF_PROB_ROTOR = 2,       /* rotor, init4.txt / Rotor_functions.f90 shape */
  GDF_PROB_BLAST = 3,       /* blast, init5.txt / p0.f90 shape             */
  GDF_PROB_CLOUD_SHOCK = 4  /* init6.txt / Cloud_Shock_functions.f90       */
};

/*
 * Run-time configuration. The reference fixes all of this at compile time
 * (com.txt:1,7, init*.txt, calculate_dt.f90:5-9) or by commenting lines in
 * and out; the knobs below name those lines. gdf_config_reference() fills
 * the values of GDF_Balsara_P2_0316 as shipped.
 */
typedef struct GdfConfig {
  int32_t nx, ny;            /* com.txt:1 Nx, Ny                               */
  double xa, xb, ya, yb;     /* init*.txt domain                               */
  int32_t bc_r, bc_l, bc_u, bc_d; /* init*.txt bcR/bcL/bcU/bcD                 */
  double gamma;              /* com.txt:7 (Lh, eigenvalueMm, pressure)         */
  double gamma_flux;         /* MHD_flux.f90:7 and eigenmatrix.f90:19 use 5/3
                                whatever com.txt says; set equal to gamma for
                                a consistent-gamma run                         */
  int32_t flux_type;         /* GDF_FLUX_*                                      */
  double cfl;                /* calculate_dt.f90:8 (0.15; DF 0.2)              */
  double tvb_m;              /* init*.txt M (minmod.f90:10)                    */
  double tvb_slope;          /* TVB_Limiter_P2.f90:111-112 factor (0.75; DF 2/3) */
  double hlld_eps;           /* HLLD_Flux.f90:126 threshold (1e-4; DF 1e-12)   */
  int32_t pp_limiter;        /* TVB_Limiter_P2.f90:123 call pp_Limiter         */
  int32_t faceb_limiter;     /* TVB_Limiter_P2.f90:186-187 apply Bxmod/Bymod   */
  int32_t ez_face_fhat;      /* LhEz.f90:6-31: 0 local LF Ez, 1 -Fxhat7/Fyhat6 */
  int32_t eig_p_typo;        /* eigenmatrix.f90:21 DF form -0.5|u|^2           */
  int32_t eig_identity;      /* eigenmatrix.f90:397-404 identity fallback      */
  int32_t eig_y_zero_w;      /* DF TVB_Limiter_P2.f90:71 passes u3=B3=0        */
  int32_t kml_w_term;        /* Lh.f90:126 KML includes w*B3 (DF drops it)     */
  int32_t dt_floor_stop;     /* RK3.f90:69-71 dt<1e-7 ends the run             */
  int32_t umax_all_vars;     /* DF calculate_umax over all 8 averages          */
  int32_t detector;          /* GDF_DETECT_*                                    */
  double kxrcf_ck;           /* KXRCF_Detector.f90:7 threshold Ck              */
  int32_t kxrcf_sticky;      /* KXRCF flags never reset (Is_Trouble_Cell)      */
  int32_t tvb_p1;            /* TVB_Limiter_P1.f90 in place of TVB_Limiter_P2:
                                the two slopes only, higher modes zeroed where
                                changed, face-B minmod always applied       */
  int32_t reserved_i[6];
  double reserved_d[4];
} GdfConfig;

/* Reference configuration of GDF_Balsara_P2_0316 as shipped (HLL, CFL 0.15,
 * gamma 5/3, M 10, no pp, no face-B limiting, every cell limited) on an
 * nx x ny grid of [0,1]^2 with periodic boundaries. */
int gdf_config_reference(int32_t nx, int32_t ny, GdfConfig *out);

/* Problem presets: domain, boundaries, gamma, M and flux of the named
 * problem on an nx x ny grid, over the reference configuration. Replaces
 * the init*.txt include (init_data.f90:19). *tend receives the end time. */
int gdf_problem_config(int32_t problem, int32_t nx, int32_t ny, GdfConfig *out,
                       double *tend);

/* Host-side initial data (init_data.f90:1-123: L2 projection of cells and
 * faces, or point values when the problem is a shock problem). params may
 * be NULL for the defaults; for GDF_PROB_BLAST it is
 * {cx, cy, r0, p_in, p_out, rho, Bx, By}. Writes uh (ghosts zero), Bx, By.
 * Pure host code; no device is touched. */
int gdf_init_data(const GdfConfig *cfg, int32_t problem, const double *params,
                  double *uh, double *bx, double *by);

typedef struct GdfHandle GdfHandle;

/* Allocate device state for cfg on the current CUDA device. */
int gdf_create(const GdfConfig *cfg, GdfHandle **out);
int gdf_destroy(GdfHandle *h);

/* Copy the full reference arrays to / from the device (synchronous). */
int gdf_upload(GdfHandle *h, const double *uh, const double *bx, const double *by);
int gdf_download(GdfHandle *h, double *uh, double *bx, double *by);
/* As gdf_download, but only the 52 live (mode, variable) planes of uh are
 * written; the 28 dead ones of the caller's array are left as they are (the
 * P2 scheme never populates them, so a host that keeps one uh array, as the
 * reference's COMMON block, already holds zeros there). 35% less
 * device-to-host traffic per call. No counterpart in the reference. */
int gdf_download_live(GdfHandle *h, double *uh, double *bx, double *by);
/* The state a step needs and produces, in its smallest form (synchronous).
 * Replaces the transfer of uh(0:Nx+1,0:Ny+1,10,8) plus Bx/By (com.txt:48)
 * for a host that round-trips the state every step; no counterpart in the
 * reference. cells holds modes 1-6 of the six variables that evolve in the
 * cell (reference variables 1-5: rho, rho u, rho v, rho w, E, and 8: Bz)
 * over the interior cells, cells[i + Nx*(j + Ny*(d + 6*v))] for cell
 * (i+1, j+1), mode d+1, v = 0..5 for variables 1, 2, 3, 4, 5, 8 (36 Nx Ny
 * doubles); bx, by are the reference's face arrays. The rest of uh is a
 * function of these: the cell Bx/By modes are div_free_Balsara of the face
 * fields (div_free_Balsara.f90:13-79, the last write to them in every
 * stage), the ghosts are set_bc of the interior with the ghost B modes
 * cleared (how every step leaves them, div_free_Balsara.f90:11).
 * gdf_upload_state rebuilds them on the device, so a step after it equals,
 * value for value, a step of the state gdf_download_state returned; 28%
 * fewer bytes cross the bus each way than with gdf_upload and
 * gdf_download_live. A host that needs the full uh rebuilds it with the
 * reference's own div_free_Balsara and set_bc, or calls gdf_download. */
int gdf_upload_state(GdfHandle *h, const double *cells, const double *bx, const double *by);
int gdf_download_state(GdfHandle *h, double *cells, double *bx, double *by);

/* RK3.f90:5-12: t = 0, set_bc, TVB_Limiter_P2, div_free_Balsara on the
 * resident state. flags (may be NULL) receives the troubled-cell word of
 * that limiter pass (bits 0-7 changed variables, bit 24 KXRCF flag). */
int gdf_prepare(GdfHandle *h, int32_t *flags);

/* One SSP-RK3 step of the resident state: RK3.f90:60-151 (calculate_dt,
 * t clamp, 3 x [set_bc, Lh, LhEz, combine, TVB_Limiter_P2,
 * div_free_Balsara]). *t is read as the current time and receives the new
 * time; *dt_out receives dt. flags (may be NULL) receives per cell the
 * changed-variable masks of stage 1/2/3 in bits 0-7/8-15/16-23 and the
 * KXRCF flags of the three stages in bits 24/25/26. */
int gdf_step(GdfHandle *h, double tend, double *t, double *dt_out, int32_t *flags);

/* Up to max_steps steps (device-resident loop, no host sync between
 * steps); stops once t reaches tend. *steps receives the number taken. */
int gdf_advance(GdfHandle *h, double tend, int32_t max_steps, double *t,
                int32_t *steps);

/* gdf_advance without intermediate host synchronisation, with the device
 * time of the `steps` graph replays (CUDA events on the handle's stream,
 * recorded before the first and after the last) in *device_ms. */
int gdf_advance_timed(GdfHandle *h, double tend, int32_t steps, double *t,
                      int32_t *steps_taken, double *device_ms);

/* Make `device` the current CUDA device of the calling thread for this
 * library (one process per GPU; call before gdf_create). */
int gdf_set_device(int32_t device);

/* init_data.f90:21-121 on the device, written straight into the handle's
 * resident state (replaces gdf_init_data + gdf_upload for a large grid or
 * an ensemble: nothing crosses the bus but a few coefficient tables).
 * problem and params as gdf_init_data; the values equal gdf_init_data's
 * bit for bit for every problem but GDF_PROB_VORTEX, whose exp runs on the
 * device (within a couple of units in the last place). Synchronous. */
int gdf_init_data_device(GdfHandle *h, int32_t problem, const double *params);

/* Fine-grained drop-ins on caller arrays (uploaded, computed, downloaded).
 * gdf_lh:   Lh.f90 (du for all cells; ghost entries 0). uh ghosts are used
 *           as given, as Lh does.
 * gdf_lhez: LhEz.f90 (dEz1, dEz2) for the same uh, Bx, By.
 * gdf_limit: TVB_Limiter_P2.f90 then div_free_Balsara.f90 on uh (ghosts as
 *           given, rewritten by its set_bc), Bx, By in place.
 * gdf_dt:   calculate_dt.f90 on the cell averages of uh.                 */
int gdf_lh(GdfHandle *h, const double *uh, double *du);
int gdf_lhez(GdfHandle *h, const double *uh, double *dez1, double *dez2);
int gdf_limit(GdfHandle *h, double *uh, double *bx, double *by, int32_t *flags);
int gdf_dt(GdfHandle *h, const double *uh, double *dt);

/* Inputs of the learned troubled-cell indicator for every interior cell of
 * uh (a state as gdf_limit takes it, ghosts set): X[(i-1) + Nx*(j-1)][90],
 * the 6 P2 modes of rho, pressure and |B|^2 of the cell and its four
 * neighbours, scaled per cell. No counterpart in the reference (whose only
 * detector is KXRCF_Detector.f90). */
int gdf_features(GdfHandle *h, const double *uh, float *X);

/* ---- learned troubled-cell indicator (no counterpart in the reference) ---
 * A 90-64-64-1 network (GELU, GELU, sigmoid) on the gdf_features inputs,
 * trained by the library's own kernels (BF16 tensor-core products, FP32
 * accumulation, Adam on FP32 master weights). Parameters are packed FP32:
 * W1[90][64], b1[64], W2[64][64], b2[64], w3[64], b3 (10049 values). */
#define GDF_MLP_NPARAM 10049
typedef struct GdfMlp GdfMlp;
int gdf_mlp_create(int32_t seed, GdfMlp **out);   /* Glorot init from seed */
int gdf_mlp_destroy(GdfMlp *m);
int gdf_mlp_set_params(GdfMlp *m, const float *params);   /* resets Adam */
int gdf_mlp_get_params(GdfMlp *m, float *params);
/* Gradient of the mean weighted binary cross-entropy (positives weighted
 * pos_weight) over all n samples X[n][90], y[n] in {0,1}. */
int gdf_mlp_grad(GdfMlp *m, const float *X, const float *y, int64_t n, float pos_weight,
                 float *grad, float *loss);
/* Adam (lr, betas 0.9/0.999) over shuffled minibatches; epoch_loss (may be
 * NULL) receives the mean loss of each epoch. */
int gdf_mlp_train(GdfMlp *m, const float *X, const float *y, int64_t n, int32_t epochs,
                  int32_t batch, float lr, float pos_weight, int32_t seed, float *epoch_loss);
int gdf_mlp_predict(GdfMlp *m, const float *X, int64_t n, float *p);
/* Products of the training step (no counterpart in the reference): 1 (the
 * default) runs the five matrix products of a 128-sample tile as tcgen05
 * UMMAs with BF16 operands in shared memory and FP32 accumulators in tensor
 * memory; 0 runs them as mma.sync m16n8k16 tiles (64 samples per block).
 * Same roundings either way; only the order of the FP32 sums inside a
 * product differs. A tcgen05 tile that waits more than 2 s for its products
 * gives up, and the training call returns GDF_ERR_TIMEOUT. */
int gdf_mlp_set_products(GdfMlp *m, int32_t tcgen05);
const char *gdf_mlp_last_error(void);
/* Use the network m (copied) as the troubled-cell detector of h when its
 * config has detector GDF_DETECT_LEARNED: the limiter runs where p >= t_hi,
 * and where t_lo <= p < t_hi if KXRCF flags the cell. */
int gdf_set_indicator(GdfHandle *h, GdfMlp *m, float t_lo, float t_hi);

/* ---- ensemble (no counterpart in the reference, which runs one problem
 * per process) -------------------------------------------------------------
 * n independent problems, each with its own GdfConfig (grid size, domain,
 * flux, limiter settings), advanced together: one persistent cooperative
 * kernel per RK3 stage over all instances, a step captured as one CUDA
 * graph. Each instance takes its own dt (its own calculate_dt maximum) and
 * stops at its own tend; its trajectory is value for value the one a
 * GdfHandle with the same config computes. Instance i's arrays have the
 * reference extents of its config. */
typedef struct GdfEnsemble GdfEnsemble;
int gdf_ens_create(const GdfConfig *cfgs, int32_t n, GdfEnsemble **out);
int gdf_ens_destroy(GdfEnsemble *e);
int gdf_ens_upload(GdfEnsemble *e, int32_t i, const double *uh, const double *bx, const double *by);
int gdf_ens_download(GdfEnsemble *e, int32_t i, double *uh, double *bx, double *by);
/* every instance must have detector GDF_DETECT_LEARNED; one network for all */
int gdf_ens_set_indicator(GdfEnsemble *e, GdfMlp *m, float t_lo, float t_hi);
/* t and tend of instance i (i = -1: all); resets its status */
int gdf_ens_set_time(GdfEnsemble *e, int32_t i, double t, double tend);
int gdf_ens_get_time(GdfEnsemble *e, int32_t i, double *t, double *dt, int64_t *steps);
/* RK3.f90:8-12 for every instance (t = 0, tend unbounded until set) */
int gdf_ens_prepare(GdfEnsemble *e);
/* `steps` ensemble steps: every instance with t < tend takes one step per
 * ensemble step. cell_updates = sum over instances of nx*ny*(steps taken),
 * n_active = instances still short of their tend, device_ms = CUDA-event
 * time of the replays (any may be NULL). GDF_ERR_NUMERIC names the first
 * failing instance; GDF_ERR_TIMEOUT if a grid barrier gave up. */
int gdf_ens_advance(GdfEnsemble *e, int32_t steps, int64_t *cell_updates, int32_t *n_active,
                    double *device_ms);
/* Tile shape: resident blocks per SM (0 = the occupancy limit), items per
 * thread of the face / vertex / set_bc / mode tiles (a warp takes 32x that
 * many faces), cells per thread of the residual tiles (a block 64x). */
int gdf_ens_set_tiles(GdfEnsemble *e, int32_t ctas_per_sm, int32_t face_per_thread,
                      int32_t cell_per_thread);
/* Execution mode: 0 = one persistent cooperative kernel per RK stage (grid
 * barriers between phases); 1 = one batched launch per phase over all
 * instances (the default: it measured faster on the 64-instance workload,
 * each phase keeping its own register allocation). Both are graph-captured
 * and give identical results; gdf_ens_tune picks by measurement. */
int gdf_ens_set_mode(GdfEnsemble *e, int32_t mode);
int gdf_ens_get_tiles(GdfEnsemble *e, int32_t *ctas_per_sm, int32_t *face_per_thread,
                      int32_t *cell_per_thread, int32_t *grid, int32_t *graph, int32_t *mode);
/* Autotuner: times `steps` steps of each candidate from the current state,
 * restoring the state after every trial, and keeps the fastest: the
 * persistent mode with blocks per SM 1..4 x face items 1,2,4 x cells
 * 1,2,4 (36), then the per-phase mode with face items x cells (9). ms_out
 * (GDF_ENS_TUNE_CANDIDATES floats, or NULL) receives ms per step, -1 where
 * not resident. */
enum { GDF_ENS_TUNE_CANDIDATES = 45 };
int gdf_ens_tune(GdfEnsemble *e, int32_t steps, float *ms_out);
int64_t gdf_ens_kernel_launches(GdfEnsemble *e);
/* Self-test of the persistent mode's bounded grid barrier (no counterpart in
 * the reference): `blocks` cooperative blocks meet at one barrier whose wait
 * is limited to limit_ns; skip_block (or -1) names a block that never
 * arrives. *timed_out = 1 when the others gave up and reported it, 0 when
 * all met. No state is touched; the device stays usable either way. */
int gdf_ens_barrier_selftest(int32_t blocks, int32_t skip_block, uint64_t limit_ns, int32_t *timed_out);
const char *gdf_ens_last_error(void);

/* Lh (as gdf_lh) on caller-owned DEVICE buffers, allocating no device
 * memory: d_uh and d_du are device pointers with the uh extents of the
 * config (d_du receives du, ghost and unused entries 0). No counterpart in
 * the reference. It is for callers that cannot call cudaMalloc: a host
 * whose device memory is fully planned at start-up (the reference's
 * static-COMMON model carried to the GPU), or code running inside a
 * framework whose memory pool forbids allocations outside it. Its scratch
 * (the face fluxes) is a fixed array compiled into this library, so every
 * GPU that loads the library holds ~12 MB until the process exits, and the
 * grid is limited to (nx+1)*ny <= 16640 and nx*(ny+1) <= 16640 faces
 * (128 x 128 fits); larger grids get GDF_ERR_ARG. Each call looks up the
 * scratch's device address for the current device and enqueues a ~10 KB
 * copy of the basis tables on `stream` ahead of its kernels, so calls stay
 * correct across a cudaDeviceReset. The first call on a device can also
 * load the library's device code there; make it before any stream capture.
 * Work is enqueued on `stream` (a cudaStream_t, NULL for the default
 * stream) and the call returns without synchronising. All calls share the
 * one scratch array, which keeps what the last call left (a call writes
 * every scratch entry it reads): calls that overlap on the GPU (other
 * streams, other threads) race, so serialise them on one stream per GPU. */
int gdf_lh_noalloc(const GdfConfig *cfg, const double *d_uh, double *d_du, void *stream);

/* calculate_umax.f90, calculate_totaldiv.f90, calculate_pmin.f90 on the
 * resident state, plus the number of cells flagged by the last step. */
int gdf_diagnostics(GdfHandle *h, double *umax, double *totaldiv, double *pmin,
                    int64_t *n_troubled);

/* Time and dt of the resident state (RK3.f90 t, dt). */
int gdf_get_time(GdfHandle *h, double *t, double *dt);
int gdf_set_time(GdfHandle *h, double t);

/* Number of kernels this handle has launched since creation. */
int64_t gdf_kernel_launches(GdfHandle *h);

/* The handle's CUDA stream (a cudaStream_t), for callers that time or
 * order work against it. No counterpart in the reference. */
void *gdf_stream(GdfHandle *h);

/* Measured FP64 ceiling for the roofline of this FP64-bound step (no
 * counterpart in the reference): runs an FMA-only kernel (independent
 * fused multiply-add chains, no memory traffic in its loop) with
 * blocks_per_sm blocks of 256 threads on every SM of the current device,
 * `iters` x 128 FMAs per thread, and returns its rate in TFLOP/s (2 flops
 * per FMA) and its CUDA-event time. Allocates and frees a small buffer. */
int gdf_fp64_fma_peak(int32_t blocks_per_sm, int32_t iters, double *tflops, double *ms);

/* Kernel kinds reported by gdf_profile. */
enum {
  GDF_K_SET_BC = 0, GDF_K_FACE_X = 1, GDF_K_FACE_Y = 2, GDF_K_VERTEX = 3,
  GDF_K_CELL = 4, GDF_K_BFACE = 5, GDF_K_LIMIT = 6, GDF_K_DT = 7, GDF_K_DIAG = 8,
  GDF_K_FACEB_LIMIT = 9, /* face-B minmod (faceb_limiter) */
  GDF_K_DIVFREE = 10,    /* div-free reconstruction when not fused into the limiter */
  GDF_K_LIMIT_TVB = 11,  /* the limiter's second pass over the gated cells */
  GDF_KERNEL_KINDS = 12
};

/* Run `steps` time steps of the resident state with CUDA events around
 * every launch (serialised, not graph-captured) and return, per kernel
 * kind, the mean device time of one launch in ms and the launches of that
 * kind per step. The reference times nothing (its SYSTEM_CLOCK calls in
 * TVB_Limiter_P2.f90:10,14,189 are commented out); this is the
 * per-kernel tracing of the port. */
int gdf_profile(GdfHandle *h, int32_t steps, double *ms_per_launch,
                int64_t *launches_per_kind, int32_t nkinds);

/* ---- output files, error norm and checkpoint (main.f90's flow) -------- */
/* save_solution.f90: Q1.txt..Q8.txt in dir (NULL or "" = current
 * directory), uh(i,j,d,n) of the interior cells, one value per line in the
 * reference's order (d, then j, then i), 17 significant digits. */
int gdf_save_solution(const GdfConfig *cfg, const double *uh, const char *dir);
/* RK3.f90:29-53,154-172: one frame appended to Q1flash.txt..Q8flash.txt and
 * its time to T.txt (reset = 1 starts the files afresh, as RK3's first
 * frame does). The caller decides when a frame is due: the reference writes
 * the state after prepare and then whenever t > (tend/frameMAX)*countf or
 * t == tend. */
int gdf_save_frame(const GdfConfig *cfg, const double *uh, double t, const char *dir, int32_t reset);
/* save_XY.f90: Xc.txt, Yc.txt (Gauss point coordinates of every column /
 * row of cells), lambda.txt, weight.txt. */
int gdf_save_xy(const GdfConfig *cfg, const char *dir);
/* calculate_L2error.f90: L2[8] = the L2 norms per variable of uh minus the
 * smooth vortex of init1.txt moved by (t20, t20) (main.f90 passes t20 =
 * tend when tend <= 5, else 0). Host only. */
int gdf_l2_error(const GdfConfig *cfg, const double *uh, double t20, double *L2);
/* The handle's configuration. */
int gdf_config_of(GdfHandle *h, GdfConfig *out);
/* Is_Trouble_Cell of KXRCF_Detector.f90: the sticky flags, int32
 * trouble(1:Nx,1:Ny) in Fortran order. */
int gdf_get_trouble(GdfHandle *h, int32_t *trouble);
int gdf_set_trouble(GdfHandle *h, const int32_t *trouble);
/* Binary checkpoint of a handle (no counterpart in the reference, which
 * cannot restart): configuration, t, dt, uh, Bx, By and the sticky flags.
 * Loading into a handle of the same configuration restores a run that then
 * continues value for value as if uninterrupted; another configuration or
 * a damaged file gives GDF_ERR_ARG. */
int gdf_checkpoint_save(GdfHandle *h, const char *path);
int gdf_checkpoint_load(GdfHandle *h, const char *path);

/* Message of the last failure on this thread ("" if none). */
const char *gdf_last_error(void);

/* 1 when the library was built without FMA contraction (bit-faithful to
 * an FMA-free CPU build of the reference), 0 for the fast build. */
int gdf_build_exact(void);

#ifdef __cplusplus
}
#endif

#endif /* GDF_H */
