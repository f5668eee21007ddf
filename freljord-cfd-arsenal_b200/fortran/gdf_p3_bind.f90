! gdf_p3_bind.f90 -- iso_c_binding interface to the k = 3 part of the B200
! library (include/gdf_p3.h), for the host of MPI_BalsaraP3/main.f90 run as
! one rank (Nphi = 0: the phi index of extent 1 is passed through, the
! arrays' memory order is unchanged). Not compiled in this repository's
! build: the image has no Fortran compiler. Build beside the reference with
!   gfortran -O3 -fdefault-real-8 -fdefault-double-8 -c gdf_p3_bind.f90
! and link against lib/libgdf_b200.so.
module gdf_p3_bind
  use iso_c_binding
  implicit none

  type, bind(c) :: gdf_p3_config
    integer(c_int32_t) :: nx, ny
    real(c_double)     :: xa, xb, ya, yb
    integer(c_int32_t) :: bc_r, bc_l, bc_u, bc_d
    integer(c_int32_t) :: flux_type
    real(c_double)     :: gamma, cfl, tvb_m, tvb_beta, hlld_eps, change_tol
    integer(c_int32_t) :: nx_global, ny_global
    integer(c_int32_t) :: reserved(2)
  end type gdf_p3_config

  interface
    integer(c_int) function gdf_p3_config_problem(problem, nx, ny, cfg, tend) &
        bind(c, name="gdf_p3_config_problem")
      import :: c_int, c_int32_t, c_double, gdf_p3_config
      integer(c_int32_t), value :: problem, nx, ny
      type(gdf_p3_config), intent(out) :: cfg
      real(c_double), intent(out) :: tend
    end function
    integer(c_int) function gdf_p3_create(cfg, h) bind(c, name="gdf_p3_create")
      import :: c_int, c_ptr, gdf_p3_config
      type(gdf_p3_config), intent(in) :: cfg
      type(c_ptr), intent(out) :: h
    end function
    integer(c_int) function gdf_p3_destroy(h) bind(c, name="gdf_p3_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    ! uh(0:Nx1,0:Ny1,0:Nphi,dimPk,NumEq), Bx(0:Nx,0:Ny1,0:Nphi,kk+1),
    ! By(0:Nx1,0:Ny,0:Nphi,kk+1) of module com, passed as they are
    integer(c_int) function gdf_p3_upload(h, uh, bx, by) bind(c, name="gdf_p3_upload")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in) :: uh(*), bx(*), by(*)
    end function
    integer(c_int) function gdf_p3_download(h, uh, bx, by) bind(c, name="gdf_p3_download")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: uh(*), bx(*), by(*)
    end function
    integer(c_int) function gdf_p3_prepare(h) bind(c, name="gdf_p3_prepare")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function gdf_p3_step(h, tend, t, dt) bind(c, name="gdf_p3_step")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), value :: tend
      real(c_double), intent(out) :: t, dt
    end function
    integer(c_int) function gdf_p3_diagnostics(h, umax, totaldiv) bind(c, name="gdf_p3_diagnostics")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: umax, totaldiv
    end function
  end interface
end module gdf_p3_bind
