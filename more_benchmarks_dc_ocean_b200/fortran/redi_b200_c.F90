!! redi_b200_c — iso_c_binding interface of libredi_b200.so (include/redi_b200.h).
!!
!! Not compile-tested: no Fortran compiler on this image. The field order, kinds
!! and count of every bind(C) type below are checked against the C header and the
!! Python ctypes mirror by tests/test_fortran_binding.py (a text check), which is
!! what keeps this file and the library in step.
!!
!! The derived types mirror the reference's stub types field by field
!! (redi/grid.F90 hgrid_t, redi/ocean_metrics.F90 ocean_metrics_t,
!! redi/ocean_eos.F90 ocean_eos_t, redi/multilayer_cgrid_state.F90
!! multilayer_cgrid_state_t, redi/ocean_boundary_types.F90 ocean_bc_state_t),
!! with every array replaced by the DEVICE address of that array (what
!! `!$acc host_data use_device` followed by c_loc yields). The procedures are the
!! handle API that stands for ocean_redi_t and its two entry points
!! (redi/ocean_redi.F90:466-529, 572-607, 927-1002).
module redi_b200_c
   use, intrinsic :: iso_c_binding
   implicit none
   private

   integer(c_int), parameter, public :: REDI_B200_OK = 0, REDI_B200_SKIPPED = 1
   integer(c_int), parameter, public :: REDI_B200_FP64 = 0, REDI_B200_MIXED = 1

   !> hgrid_t (redi/grid.F90:17-25)
   type, bind(C), public :: redi_b200_grid
      integer(c_int) :: nx_total, ny_total
      integer(c_int) :: nx_phys, ny_phys
      integer(c_int) :: nghost
      real(c_double) :: dx, dy
   end type redi_b200_grid

   !> ocean_metrics_t (redi/ocean_metrics.F90:14-22): device addresses
   type, bind(C), public :: redi_b200_metrics
      type(c_ptr) :: dy_cu, dx_cv, idxCu, idyCv, areaT, wet_u, wet_v
   end type redi_b200_metrics

   !> ocean_eos_t (redi/ocean_eos.F90:239-278): eos%variant is passed unchanged
   !> (1 LINEAR, 2 WRIGHT_97, 4 ROQUET_SPV; 3 TEOS-10 is rejected)
   type, bind(C), public :: redi_b200_eos
      integer(c_int) :: variant
      real(c_double) :: rho0, T_ref, S_ref, alpha_T, beta_S
   end type redi_b200_eos

   !> multilayer_cgrid_state_t (redi/multilayer_cgrid_state.F90:18-28):
   !> h_layer is a device address, hTr the HOST address of an array of ntracers
   !> device addresses (one per ms%tracers(it)%hTr)
   type, bind(C), public :: redi_b200_state
      integer(c_int) :: nz_ml
      integer(c_int) :: idx_temperature, idx_salinity
      integer(c_int) :: ntracers
      type(c_ptr) :: h_layer
      type(c_ptr) :: hTr
   end type redi_b200_state

   !> ocean_bc_state_t (redi/ocean_boundary_types.F90:20-24): bc_type per edge
   type, bind(C), public :: redi_b200_bc
      integer(c_int) :: west, east, south, north
   end type redi_b200_bc

   !> device addresses of a handle's Phase-A slots (ocean_redi_t%uPoL ... %vhEff)
   type, bind(C), public :: redi_b200_coeffs
      type(c_ptr) :: uPoL, uPoR, uhEff
      type(c_ptr) :: uKoL, uKoR
      type(c_ptr) :: vPoL, vPoR, vhEff
      type(c_ptr) :: vKoL, vKoR
      type(c_ptr) :: khtr_u, khtr_v
      integer(c_int) :: nsurf
   end type redi_b200_coeffs

   public :: redi_b200_init, redi_b200_destroy, redi_b200_set_enable, redi_b200_set_khtr
   public :: redi_b200_calc_coeffs, redi_b200_apply_flux, redi_b200_step, redi_b200_get_coeffs
   public :: redi_b200_error_count, redi_b200_last_error

   interface
      !> ocean_redi_init: h receives the handle
      integer(c_int) function redi_b200_init(grid, nz_ml, precision, h) bind(C, name="redi_b200_init")
         import :: c_int, c_ptr, redi_b200_grid
         type(redi_b200_grid), intent(in) :: grid
         integer(c_int), value :: nz_ml, precision
         type(c_ptr), intent(out) :: h
      end function redi_b200_init

      !> ocean_redi_destroy
      integer(c_int) function redi_b200_destroy(h) bind(C, name="redi_b200_destroy")
         import :: c_int, c_ptr
         type(c_ptr), value :: h
      end function redi_b200_destroy

      !> ocean_redi_t%enable
      integer(c_int) function redi_b200_set_enable(h, enable) bind(C, name="redi_b200_set_enable")
         import :: c_int, c_ptr
         type(c_ptr), value :: h
         integer(c_int), value :: enable
      end function redi_b200_set_enable

      !> ocean_redi_t%khtr
      integer(c_int) function redi_b200_set_khtr(h, khtr) bind(C, name="redi_b200_set_khtr")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: h
         real(c_double), value :: khtr
      end function redi_b200_set_khtr

      !> redi_calc_coeffs(grid, metrics, eos, this, ms)
      integer(c_int) function redi_b200_calc_coeffs(grid, metrics, eos, h, ms, stream) &
         bind(C, name="redi_b200_calc_coeffs")
         import :: c_int, c_ptr, redi_b200_grid, redi_b200_metrics, redi_b200_eos, redi_b200_state
         type(redi_b200_grid), intent(in) :: grid
         type(redi_b200_metrics), intent(in) :: metrics
         type(redi_b200_eos), intent(in) :: eos
         type(c_ptr), value :: h
         type(redi_b200_state), intent(in) :: ms
         type(c_ptr), value :: stream          ! c_null_ptr: the legacy default stream
      end function redi_b200_calc_coeffs

      !> redi_apply_flux(grid, metrics, this, ms, dt, khtr_u_ext, khtr_v_ext, bc)
      integer(c_int) function redi_b200_apply_flux(grid, metrics, h, ms, dt, khtr_u_ext, khtr_v_ext, bc, stream) &
         bind(C, name="redi_b200_apply_flux")
         import :: c_int, c_ptr, c_double, redi_b200_grid, redi_b200_metrics, redi_b200_state, redi_b200_bc
         type(redi_b200_grid), intent(in) :: grid
         type(redi_b200_metrics), intent(in) :: metrics
         type(c_ptr), value :: h
         type(redi_b200_state), intent(in) :: ms
         real(c_double), value :: dt
         type(c_ptr), value :: khtr_u_ext, khtr_v_ext   ! both non-null: the per-face path
         type(redi_b200_bc), intent(in), optional :: bc ! absent (NULL): every edge a wall
         type(c_ptr), value :: stream
      end function redi_b200_apply_flux

      !> redi_calc_coeffs then redi_apply_flux on the same state, in one call
      !> (same gates, statuses and results; one column pass fewer)
      integer(c_int) function redi_b200_step(grid, metrics, eos, h, ms, dt, khtr_u_ext, khtr_v_ext, bc, stream) &
         bind(C, name="redi_b200_step")
         import :: c_int, c_ptr, c_double, redi_b200_grid, redi_b200_metrics, redi_b200_eos, redi_b200_state, &
                   redi_b200_bc
         type(redi_b200_grid), intent(in) :: grid
         type(redi_b200_metrics), intent(in) :: metrics
         type(redi_b200_eos), intent(in) :: eos
         type(c_ptr), value :: h
         type(redi_b200_state), intent(in) :: ms
         real(c_double), value :: dt
         type(c_ptr), value :: khtr_u_ext, khtr_v_ext
         type(redi_b200_bc), intent(in), optional :: bc
         type(c_ptr), value :: stream
      end function redi_b200_step

      !> device addresses of the handle's coefficient slots
      integer(c_int) function redi_b200_get_coeffs(h, out) bind(C, name="redi_b200_get_coeffs")
         import :: c_int, c_ptr, redi_b200_coeffs
         type(c_ptr), value :: h
         type(redi_b200_coeffs), intent(out) :: out
      end function redi_b200_get_coeffs

      !> out-of-order coefficient sublayers seen since the last reset (synchronises)
      integer(c_int) function redi_b200_error_count(h, reset) bind(C, name="redi_b200_error_count")
         import :: c_int, c_ptr
         type(c_ptr), value :: h
         integer(c_int), value :: reset
      end function redi_b200_error_count

      !> message of the calling thread's last error (a NUL-terminated C string)
      type(c_ptr) function redi_b200_last_error() bind(C, name="redi_b200_last_error")
         import :: c_ptr
      end function redi_b200_last_error
   end interface
end module redi_b200_c
