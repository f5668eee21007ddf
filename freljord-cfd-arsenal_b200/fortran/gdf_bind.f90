! gdf_bind.f90 -- iso_c_binding interface to the B200 GDF P2 library
! (include/gdf.h), for the reference's Fortran host (main.f90, init_data.f90,
! save_solution.f90). Not compiled in this repository's build: the image has
! no Fortran compiler. Build it beside the reference's sources with
!   gfortran -O3 -fdefault-real-8 -fdefault-double-8 -c gdf_bind.f90
! and link the executable against lib/libgdf_b200.so.
module gdf_bind
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: GDF_OK = 0
  integer(c_int), parameter :: GDF_FLUX_LF = 1, GDF_FLUX_HLL = 2, GDF_FLUX_HLLC = 3, GDF_FLUX_HLLD = 4
  integer(c_int), parameter :: GDF_BC_PERIODIC = 1, GDF_BC_OUTFLOW = 2
  integer(c_int), parameter :: GDF_DETECT_ALL = 0, GDF_DETECT_KXRCF = 1

  type, bind(c) :: gdf_config
    integer(c_int32_t) :: nx, ny
    real(c_double)     :: xa, xb, ya, yb
    integer(c_int32_t) :: bc_r, bc_l, bc_u, bc_d
    real(c_double)     :: gamma, gamma_flux
    integer(c_int32_t) :: flux_type
    real(c_double)     :: cfl, tvb_m, tvb_slope, hlld_eps
    integer(c_int32_t) :: pp_limiter, faceb_limiter, ez_face_fhat, eig_p_typo, eig_identity
    integer(c_int32_t) :: eig_y_zero_w, kml_w_term, dt_floor_stop, umax_all_vars, detector
    real(c_double)     :: kxrcf_ck
    integer(c_int32_t) :: kxrcf_sticky
    integer(c_int32_t) :: tvb_p1
    integer(c_int32_t) :: reserved_i(6)
    real(c_double)     :: reserved_d(4)
  end type gdf_config

  interface
    integer(c_int) function gdf_config_reference(nx, ny, cfg) bind(c, name="gdf_config_reference")
      import :: c_int, c_int32_t, gdf_config
      integer(c_int32_t), value :: nx, ny
      type(gdf_config), intent(out) :: cfg
    end function
    integer(c_int) function gdf_create(cfg, h) bind(c, name="gdf_create")
      import :: c_int, c_ptr, gdf_config
      type(gdf_config), intent(in) :: cfg
      type(c_ptr), intent(out) :: h
    end function
    integer(c_int) function gdf_destroy(h) bind(c, name="gdf_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    ! uh(0:Nx1,0:Ny1,10,8), Bx(0:Nx,Ny,3), By(Nx,0:Ny,3) of com.txt, passed as they are
    integer(c_int) function gdf_upload(h, uh, bx, by) bind(c, name="gdf_upload")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in) :: uh(*), bx(*), by(*)
    end function
    integer(c_int) function gdf_download(h, uh, bx, by) bind(c, name="gdf_download")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: uh(*), bx(*), by(*)
    end function
    ! the step state in its smallest form: cells(Nx, Ny, 6, 6) holds modes
    ! 1-6 of variables 1-5 and 8 over the interior cells; the device rebuilds
    ! the cell B modes (div_free_Balsara) and the ghosts (set_bc)
    integer(c_int) function gdf_upload_state(h, cells, bx, by) bind(c, name="gdf_upload_state")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in) :: cells(*), bx(*), by(*)
    end function
    integer(c_int) function gdf_download_state(h, cells, bx, by) bind(c, name="gdf_download_state")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: cells(*), bx(*), by(*)
    end function
    ! init_data.f90 on the device, into the handle's state (params may be
    ! c_null_ptr for the problem's defaults)
    integer(c_int) function gdf_init_data_device(h, problem, params) bind(c, name="gdf_init_data_device")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
      integer(c_int), value :: problem
      type(c_ptr), value :: params
    end function
    integer(c_int) function gdf_prepare(h, flags) bind(c, name="gdf_prepare")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
      type(c_ptr), value :: flags
    end function
    integer(c_int) function gdf_step(h, tend, t, dt, flags) bind(c, name="gdf_step")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), value :: tend
      real(c_double), intent(inout) :: t
      real(c_double), intent(out) :: dt
      type(c_ptr), value :: flags
    end function
    integer(c_int) function gdf_advance(h, tend, max_steps, t, steps) bind(c, name="gdf_advance")
      import :: c_int, c_ptr, c_double, c_int32_t
      type(c_ptr), value :: h
      real(c_double), value :: tend
      integer(c_int32_t), value :: max_steps
      real(c_double), intent(inout) :: t
      integer(c_int32_t), intent(out) :: steps
    end function
    integer(c_int) function gdf_diagnostics(h, umax, totaldiv, pmin, ntrouble) bind(c, name="gdf_diagnostics")
      import :: c_int, c_ptr, c_double, c_int64_t
      type(c_ptr), value :: h
      real(c_double), intent(out) :: umax, totaldiv, pmin
      integer(c_int64_t), intent(out) :: ntrouble
    end function
    type(c_ptr) function gdf_last_error() bind(c, name="gdf_last_error")
      import :: c_ptr
    end function
    ! output files of save_solution.f90 / RK3.f90 frames / save_XY.f90,
    ! calculate_L2error.f90, and the binary checkpoint (dir, path: C strings,
    ! e.g. "out"//c_null_char)
    integer(c_int) function gdf_save_solution(cfg, uh, dir) bind(c, name="gdf_save_solution")
      import :: c_int, c_double, c_char, gdf_config
      type(gdf_config), intent(in) :: cfg
      real(c_double), intent(in) :: uh(*)
      character(kind=c_char), intent(in) :: dir(*)
    end function
    integer(c_int) function gdf_save_frame(cfg, uh, t, dir, reset) bind(c, name="gdf_save_frame")
      import :: c_int, c_double, c_char, gdf_config
      type(gdf_config), intent(in) :: cfg
      real(c_double), intent(in) :: uh(*)
      real(c_double), value :: t
      character(kind=c_char), intent(in) :: dir(*)
      integer(c_int), value :: reset
    end function
    integer(c_int) function gdf_save_xy(cfg, dir) bind(c, name="gdf_save_xy")
      import :: c_int, c_char, gdf_config
      type(gdf_config), intent(in) :: cfg
      character(kind=c_char), intent(in) :: dir(*)
    end function
    integer(c_int) function gdf_l2_error(cfg, uh, t20, l2) bind(c, name="gdf_l2_error")
      import :: c_int, c_double, gdf_config
      type(gdf_config), intent(in) :: cfg
      real(c_double), intent(in) :: uh(*)
      real(c_double), value :: t20
      real(c_double), intent(out) :: l2(8)
    end function
    integer(c_int) function gdf_checkpoint_save(h, path) bind(c, name="gdf_checkpoint_save")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: h
      character(kind=c_char), intent(in) :: path(*)
    end function
    integer(c_int) function gdf_checkpoint_load(h, path) bind(c, name="gdf_checkpoint_load")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: h
      character(kind=c_char), intent(in) :: path(*)
    end function
  end interface
end module gdf_bind
