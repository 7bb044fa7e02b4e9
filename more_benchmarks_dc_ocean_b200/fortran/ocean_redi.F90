!! ocean_redi — drop-in replacement of the reference's module of the same name
!! (redi/ocean_redi.F90), backed by libredi_b200.so through redi_b200_c.
!!
!! Not compile-tested: no Fortran compiler on this image.
!!
!! Public names and argument lists are the reference's (ocean_redi.F90:46-65,
!! 71-128, 466-564, 572-582, 927-946): ocean_redi_t with %init, %destroy,
!! %enter_data, %exit_data and the switches enable / continuous / khtr /
!! ref_pres, redi_calc_coeffs(grid, metrics, eos, this, ms) and
!! redi_apply_flux(grid, metrics, this, ms, dt, khtr_u_ext, khtr_v_ext, bc).
!! The model's own modules (constants, grid, ocean_metrics,
!! multilayer_cgrid_state, ocean_eos, ocean_boundary_types) are used unchanged.
!!
!! What differs inside: the Phase-A coefficient slots and the tracer snapshot
!! live in the library (device memory owned by the handle, reachable through
!! redi_b200_get_coeffs), so %enter_data / %exit_data have nothing to move;
!! every tracer of ms%tracers(:) is updated by one fused pass instead of a
!! snapshot and a kernel per tracer. Every array is handed over as the device
!! address OpenACC holds for it (`!$acc host_data use_device`, as
!! redi/drivers/redi_bridge.F90:70-87 does for the reference's own launcher).
!! The module's numerical helpers (redi_interface_scalar, redi_ppm_ave, ...) are
!! not re-exported: they are internal to the library's kernels.
#include "directives.h"
module ocean_redi
   use, intrinsic :: iso_c_binding
   use constants, only: wp
   use grid, only: hgrid_t
   use ocean_metrics, only: ocean_metrics_t
   use multilayer_cgrid_state, only: multilayer_cgrid_state_t
   use ocean_eos, only: ocean_eos_t
   use ocean_boundary_types, only: ocean_bc_state_t
   use redi_b200_c
   implicit none
   private

   public :: ocean_redi_t
   public :: redi_calc_coeffs
   public :: redi_apply_flux

   type :: ocean_redi_t
      logical :: is_init = .false.
      logical :: enable = .false.
      logical :: continuous = .true.
      real(wp) :: khtr = 0.0_wp
      real(wp) :: ref_pres = -1.0_wp
      integer :: nx_total = 0
      integer :: ny_total = 0
      integer :: nz_ml = 0
      integer :: nsurf = 0
      type(c_ptr) :: h = c_null_ptr      !! the library handle (coefficient slots, scratch)
      integer(c_int) :: precision = REDI_B200_FP64
   contains
      procedure, non_overridable :: init => ocean_redi_init
      procedure, non_overridable :: destroy => ocean_redi_destroy
      procedure, non_overridable :: enter_data => ocean_redi_enter_data
      procedure, non_overridable :: exit_data => ocean_redi_exit_data
   end type ocean_redi_t

contains

   subroutine check(rc, where)
      integer(c_int), intent(in) :: rc
      character(*), intent(in) :: where
      character(kind=c_char), pointer :: msg(:)
      integer :: n
      if (rc >= 0) return
      call c_f_pointer(redi_b200_last_error(), msg, [512])
      n = 0
      do while (n < 512)
         if (msg(n + 1) == c_null_char) exit
         n = n + 1
      end do
      write (*, '(a, ": ", 512a)') where, msg(1:n)
      error stop "ocean_redi: libredi_b200 call failed"
   end subroutine check

   function grid_c(grid) result(g)
      type(hgrid_t), intent(in) :: grid
      type(redi_b200_grid) :: g
      g%nx_total = grid%nx_total
      g%ny_total = grid%ny_total
      g%nx_phys = grid%nx_phys
      g%ny_phys = grid%ny_phys
      g%nghost = grid%nghost
      g%dx = grid%dx
      g%dy = grid%dy
   end function grid_c

   !> ocean_redi_init (ocean_redi.F90:466-507): the library stops where the
   !> reference's init does (2*nz+2 beyond what the kernels hold) with an error.
   subroutine ocean_redi_init(this, grid, nz_ml)
      class(ocean_redi_t), intent(inout) :: this
      type(hgrid_t), intent(in) :: grid
      integer, intent(in), optional :: nz_ml
      integer :: nz
      nz = 1
      if (present(nz_ml)) nz = nz_ml
      if (nz < 1) nz = 1
      call check(redi_b200_init(grid_c(grid), int(nz, c_int), this%precision, this%h), "ocean_redi_init")
      this%nx_total = grid%nx_total
      this%ny_total = grid%ny_total
      this%nz_ml = nz
      this%nsurf = 2*nz + 2
      this%is_init = .true.
   end subroutine ocean_redi_init

   subroutine ocean_redi_destroy(this)
      class(ocean_redi_t), intent(inout) :: this
      integer(c_int) :: rc
      this%is_init = .false.
      if (c_associated(this%h)) rc = redi_b200_destroy(this%h)
      this%h = c_null_ptr
      this%nx_total = 0
      this%ny_total = 0
      this%nz_ml = 0
      this%nsurf = 0
   end subroutine ocean_redi_destroy

   !> The slots are device memory of the library from init on: nothing to copy.
   subroutine ocean_redi_enter_data(this)
      class(ocean_redi_t), intent(inout) :: this
   end subroutine ocean_redi_enter_data

   subroutine ocean_redi_exit_data(this)
      class(ocean_redi_t), intent(inout) :: this
   end subroutine ocean_redi_exit_data

   !> Pushes the Fortran switches into the handle; the library applies the
   !> reference's gates (ocean_redi.F90:585-593, 951-978) itself.
   subroutine sync_switches(this)
      type(ocean_redi_t), intent(inout) :: this
      call check(redi_b200_set_enable(this%h, merge(1_c_int, 0_c_int, this%enable)), "ocean_redi enable")
      call check(redi_b200_set_khtr(this%h, real(this%khtr, c_double)), "ocean_redi khtr")
   end subroutine sync_switches

   !> redi_calc_coeffs (ocean_redi.F90:572-607)
   subroutine redi_calc_coeffs(grid, metrics, eos, this, ms)
      type(hgrid_t), intent(in) :: grid
      type(ocean_metrics_t), intent(in) :: metrics
      type(ocean_eos_t), intent(in) :: eos
      type(ocean_redi_t), intent(inout) :: this
      type(multilayer_cgrid_state_t), intent(in), target :: ms
      type(redi_b200_metrics) :: m
      type(redi_b200_eos) :: e
      type(redi_b200_state) :: s
      type(c_ptr), allocatable, target :: trp(:)
      integer :: it, ntr

      if (.not. this%is_init) return
      if (.not. this%enable) return
      if (ms%idx_temperature <= 0 .or. ms%idx_salinity <= 0) return
      if (.not. allocated(ms%h_layer)) return
      call sync_switches(this)
      ntr = size(ms%tracers)
      allocate (trp(ntr))
      do it = 1, ntr
         !$acc host_data use_device(ms%tracers(it)%hTr)
         trp(it) = c_loc(ms%tracers(it)%hTr)
         !$acc end host_data
      end do
      !$acc host_data use_device(metrics%dy_cu, metrics%dx_cv, metrics%idxCu, metrics%idyCv, &
      !$acc                      metrics%areaT, metrics%wet_u, metrics%wet_v, ms%h_layer)
      m%dy_cu = c_loc(metrics%dy_cu)
      m%dx_cv = c_loc(metrics%dx_cv)
      m%idxCu = c_loc(metrics%idxCu)
      m%idyCv = c_loc(metrics%idyCv)
      m%areaT = c_loc(metrics%areaT)
      m%wet_u = c_loc(metrics%wet_u)
      m%wet_v = c_loc(metrics%wet_v)
      s%h_layer = c_loc(ms%h_layer)
      !$acc end host_data
      e%variant = eos%variant
      e%rho0 = eos%rho0
      e%T_ref = eos%T_ref
      e%S_ref = eos%S_ref
      e%alpha_T = eos%alpha_T
      e%beta_S = eos%beta_S
      s%nz_ml = ms%nz_ml
      s%idx_temperature = ms%idx_temperature
      s%idx_salinity = ms%idx_salinity
      s%ntracers = ntr
      s%hTr = c_loc(trp)
      call check(redi_b200_calc_coeffs(grid_c(grid), m, e, this%h, s, c_null_ptr), "redi_calc_coeffs")
   end subroutine redi_calc_coeffs

   !> redi_apply_flux (ocean_redi.F90:927-1002): khtr_u_ext / khtr_v_ext and bc
   !> optional as in the reference; every tracer of ms is updated.
   subroutine redi_apply_flux(grid, metrics, this, ms, dt, khtr_u_ext, khtr_v_ext, bc)
      type(hgrid_t), intent(in) :: grid
      type(ocean_metrics_t), intent(in) :: metrics
      type(ocean_redi_t), intent(inout) :: this
      type(multilayer_cgrid_state_t), intent(inout), target :: ms
      real(wp), intent(in) :: dt
      real(wp), intent(in), optional, target :: khtr_u_ext(:, :)
      real(wp), intent(in), optional, target :: khtr_v_ext(:, :)
      type(ocean_bc_state_t), intent(in), optional :: bc
      type(redi_b200_metrics) :: m
      type(redi_b200_state) :: s
      type(redi_b200_bc) :: b
      type(c_ptr) :: ku, kv
      type(c_ptr), allocatable, target :: trp(:)
      integer :: it, ntr

      if (.not. this%is_init) return
      if (.not. this%enable) return
      if (.not. allocated(ms%h_layer)) return
      if (.not. allocated(ms%tracers)) return
      call sync_switches(this)
      ntr = size(ms%tracers)
      allocate (trp(ntr))
      do it = 1, ntr
         !$acc host_data use_device(ms%tracers(it)%hTr)
         trp(it) = c_loc(ms%tracers(it)%hTr)
         !$acc end host_data
      end do
      ku = c_null_ptr
      kv = c_null_ptr
      if (present(khtr_u_ext) .and. present(khtr_v_ext)) then
         !$acc host_data use_device(khtr_u_ext, khtr_v_ext)
         ku = c_loc(khtr_u_ext)
         kv = c_loc(khtr_v_ext)
         !$acc end host_data
      end if
      !$acc host_data use_device(metrics%dy_cu, metrics%dx_cv, metrics%idxCu, metrics%idyCv, &
      !$acc                      metrics%areaT, metrics%wet_u, metrics%wet_v, ms%h_layer)
      m%dy_cu = c_loc(metrics%dy_cu)
      m%dx_cv = c_loc(metrics%dx_cv)
      m%idxCu = c_loc(metrics%idxCu)
      m%idyCv = c_loc(metrics%idyCv)
      m%areaT = c_loc(metrics%areaT)
      m%wet_u = c_loc(metrics%wet_u)
      m%wet_v = c_loc(metrics%wet_v)
      s%h_layer = c_loc(ms%h_layer)
      !$acc end host_data
      s%nz_ml = ms%nz_ml
      s%idx_temperature = ms%idx_temperature
      s%idx_salinity = ms%idx_salinity
      s%ntracers = ntr
      s%hTr = c_loc(trp)
      if (present(bc)) then
         b%west = bc%west%bc_type
         b%east = bc%east%bc_type
         b%south = bc%south%bc_type
         b%north = bc%north%bc_type
         call check(redi_b200_apply_flux(grid_c(grid), m, this%h, s, real(dt, c_double), ku, kv, b, c_null_ptr), &
                    "redi_apply_flux")
      else
         call check(redi_b200_apply_flux(grid_c(grid), m, this%h, s, real(dt, c_double), ku, kv, &
                                         stream=c_null_ptr), "redi_apply_flux")
      end if
   end subroutine redi_apply_flux

end module ocean_redi
