! gdf_cy_bind.f90 -- iso_c_binding interface to the cylindrical part of the
! B200 library (include/gdf_cy.h), for the host of MHD_GDF_cy3D_0421/main.f90.
! The COMMON arrays uh(0:Nx1,0:Ny1,0:Nphi,dimPk,NumEq), Br(0:Nx,Ny,0:Nphi,k+1)
! and Bz(Nx,0:Ny,0:Nphi,k+1) are passed as they are. Not compiled in this
! repository's build: the image has no Fortran compiler. Build beside the
! reference with
!   gfortran -O3 -fdefault-real-8 -fdefault-double-8 -c gdf_cy_bind.f90
! and link against lib/libgdf_b200.so.
module gdf_cy_bind
  use iso_c_binding
  implicit none

  type, bind(c) :: gdf_cy_config
    integer(c_int32_t) :: nr, nz, lphi
    integer(c_int32_t) :: bc_r, bc_l, bc_u, bc_d
    integer(c_int32_t) :: flux_type, rhsc_open, reserved_i
    real(c_double)     :: ra, rb, za, zb
    real(c_double)     :: gamma, cfl, tvb_m, change_tol, jet_r
    real(c_double)     :: reserved_d(3)
  end type gdf_cy_config

  interface
    integer(c_int) function gdf_cy_config_problem(problem, nr, nz, lphi, cfg, tend) &
        bind(c, name="gdf_cy_config_problem")
      import :: c_int, c_int32_t, c_double, gdf_cy_config
      integer(c_int32_t), value :: problem, nr, nz, lphi
      type(gdf_cy_config), intent(out) :: cfg
      real(c_double), intent(out) :: tend
    end function
    integer(c_int) function gdf_cy_create(cfg, h) bind(c, name="gdf_cy_create")
      import :: c_int, c_ptr, gdf_cy_config
      type(gdf_cy_config), intent(in) :: cfg
      type(c_ptr), intent(out) :: h
    end function
    integer(c_int) function gdf_cy_destroy(h) bind(c, name="gdf_cy_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function gdf_cy_upload(h, uh, br, bz) bind(c, name="gdf_cy_upload")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in) :: uh(*), br(*), bz(*)
    end function
    integer(c_int) function gdf_cy_download(h, uh, br, bz) bind(c, name="gdf_cy_download")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: uh(*), br(*), bz(*)
    end function
    integer(c_int) function gdf_cy_prepare(h) bind(c, name="gdf_cy_prepare")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function gdf_cy_step(h, tend, t, dt) bind(c, name="gdf_cy_step")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), value :: tend
      real(c_double), intent(out) :: t, dt
    end function
    integer(c_int) function gdf_cy_diagnostics(h, umax, totaldiv, pmin) bind(c, name="gdf_cy_diagnostics")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: umax, totaldiv, pmin
    end function
  end interface
end module gdf_cy_bind
