!-------------------------------------------------------------------------------
!> ISO_C_BINDING shim: the NICAM tracer-advection kernels of IcoAtmosBenchmark_v1
!! (module mod_src_tracer of kernels/NICAM/{dyn_horiz_adv_flux,dyn_horiz_adv_limiter,
!! dyn_vert_adv_limiter}/src) on a B200 through libicoadv's C ABI (include/icoadv.h).
!!
!! A driver switches `use mod_src_tracer` to `use ica_shim` and calls ica_shim_setup once its
!! module globals and metrics are set (after CONST_setup and the snapshot read in main.f90);
!! every kernel call then keeps its argument list:
!!
!!   call horizontal_flux( flx_h, flx_h_pl, GRD_xc, GRD_xc_pl, rhog_mean, rhog_mean_pl,   &
!!                         rhogvx, rhogvx_pl, rhogvy, rhogvy_pl, rhogvz, rhogvz_pl,       &
!!                         SET_dt_large )          ! dyn_horiz_adv_flux/src/main.f90:229-235
!!
!! Sizes come from the driver's module globals (mod_misc / problem_size.inc:28-50: ADM_gall_1d,
!! ADM_kall, ADM_kmin, ADM_kmax, ADM_lall, ADM_have_pl, ADM_have_sgp) through
!! ica_init_regions, and the metrics (GRD_xr, GMTR_p/t/a and their pole arrays, with the K0
!! axis of length 1) through ica_set_geometry, copied to the GPU once.  The arrays themselves
!! are passed as they are: Fortran column-major var(ij,k,l,m) is the C layout the library
!! reads.  RP = DP calls the FP64 entry points; a build with -DSINGLE (RP = SP, as
!! mod_precision.f90) calls the *_f32 ones.  A nonzero status of the library prints
!! ica_last_error() and stops, as the reference stops on errors.
!!
!! Qout_post of horizontal_limiter_thuburn is OPTIONAL here: present, the limiter reads it
!! as the extracted kernel reads its snapshot (mod_src_tracer.f90:369-373); absent, the
!! library runs the Qout halo fill itself (NICAM's COMM_data_transfer at :371), which needs
!! a context over a whole grid (ica_shim_setup_grid); a one-region driver context refuses it.
!!
!! This file is compiled with the driver (gfortran -cpp ... icoadv_f.f90, linked with
!! -licoadv); no Fortran compiler was available where this library was built and tested, so
!! the same calls are exercised from C by tests/c_driver/ica_driver.c.
!-------------------------------------------------------------------------------
module ica_shim
  use iso_c_binding
  use mod_precision, only: RP, DP, SP
  use mod_misc, only: &
       ADM_gall_1d, ADM_gall, ADM_gall_pl, ADM_kall, ADM_kmin, ADM_kmax, &
       ADM_lall, ADM_lall_pl, ADM_have_pl, ADM_have_sgp,                &
       GRD_xr, GRD_xr_pl, GMTR_p, GMTR_p_pl, GMTR_t, GMTR_t_pl, GMTR_a, GMTR_a_pl
  implicit none
  private

  public :: ica_shim_setup
  public :: ica_shim_setup_grid
  public :: ica_shim_finalize
  public :: horizontal_flux
  public :: horizontal_limiter_thuburn
  public :: vertical_limiter_thuburn

  type(c_ptr), save :: ctx = c_null_ptr

  !--- the C ABI (include/icoadv.h)
  type, bind(C) :: ica_dims
     integer(c_int) :: glevel, rlevel, vlayer, device
  end type ica_dims

  interface
     integer(c_int) function ica_init(dims, out) bind(C, name="ica_init")
       import :: c_int, c_ptr, ica_dims
       type(ica_dims), intent(in) :: dims
       type(c_ptr), intent(out) :: out
     end function ica_init
     integer(c_int) function ica_init_regions(gall_1d, kall, kmin, kmax, lall, have_pl, have_sgp, device, out) &
          bind(C, name="ica_init_regions")
       import :: c_int, c_ptr
       integer(c_int), value :: gall_1d, kall, kmin, kmax, lall, have_pl, device
       integer(c_int), intent(in) :: have_sgp(*)
       type(c_ptr), intent(out) :: out
     end function ica_init_regions
     integer(c_int) function ica_finalize(c) bind(C, name="ica_finalize")
       import :: c_int, c_ptr
       type(c_ptr), value :: c
     end function ica_finalize
     type(c_ptr) function ica_last_error() bind(C, name="ica_last_error")
       import :: c_ptr
     end function ica_last_error
     integer(c_int) function ica_set_geometry(c, xr, xr_pl, p, p_pl, t, t_pl, a, a_pl) &
          bind(C, name="ica_set_geometry")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: c
       real(c_double), intent(in) :: xr(*), xr_pl(*), p(*), p_pl(*), t(*), t_pl(*), a(*), a_pl(*)
     end function ica_set_geometry

     integer(c_int) function ica_horizontal_flux(c, flx_h, flx_h_pl, GRD_xc, GRD_xc_pl, rho, rho_pl, &
          rhovx, rhovx_pl, rhovy, rhovy_pl, rhovz, rhovz_pl, dt) bind(C, name="ica_horizontal_flux")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: c
       real(c_double), intent(inout) :: flx_h(*), flx_h_pl(*), GRD_xc(*), GRD_xc_pl(*)
       real(c_double), intent(in) :: rho(*), rho_pl(*), rhovx(*), rhovx_pl(*), rhovy(*), rhovy_pl(*), &
            rhovz(*), rhovz_pl(*)
       real(c_double), value :: dt
     end function ica_horizontal_flux
     integer(c_int) function ica_horizontal_flux_f32(c, flx_h, flx_h_pl, GRD_xc, GRD_xc_pl, rho, rho_pl, &
          rhovx, rhovx_pl, rhovy, rhovy_pl, rhovz, rhovz_pl, dt) bind(C, name="ica_horizontal_flux_f32")
       import :: c_int, c_ptr, c_float
       type(c_ptr), value :: c
       real(c_float), intent(inout) :: flx_h(*), flx_h_pl(*), GRD_xc(*), GRD_xc_pl(*)
       real(c_float), intent(in) :: rho(*), rho_pl(*), rhovx(*), rhovx_pl(*), rhovy(*), rhovy_pl(*), &
            rhovz(*), rhovz_pl(*)
       real(c_float), value :: dt
     end function ica_horizontal_flux_f32

     integer(c_int) function ica_horizontal_limiter_thuburn(c, q_a, q_a_pl, q, q_pl, d, d_pl, ch, ch_pl, &
          cmask, cmask_pl, Qout_prev, Qout_prev_pl, Qout_post, Qout_post_pl) &
          bind(C, name="ica_horizontal_limiter_thuburn")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: c
       real(c_double), intent(inout) :: q_a(*), q_a_pl(*)
       real(c_double), intent(in) :: q(*), q_pl(*), d(*), d_pl(*), ch(*), ch_pl(*), cmask(*), cmask_pl(*)
       real(c_double), intent(inout) :: Qout_prev(*), Qout_prev_pl(*)
       type(c_ptr), value :: Qout_post, Qout_post_pl
     end function ica_horizontal_limiter_thuburn
     integer(c_int) function ica_horizontal_limiter_thuburn_f32(c, q_a, q_a_pl, q, q_pl, d, d_pl, ch, ch_pl, &
          cmask, cmask_pl, Qout_prev, Qout_prev_pl, Qout_post, Qout_post_pl) &
          bind(C, name="ica_horizontal_limiter_thuburn_f32")
       import :: c_int, c_ptr, c_float
       type(c_ptr), value :: c
       real(c_float), intent(inout) :: q_a(*), q_a_pl(*)
       real(c_float), intent(in) :: q(*), q_pl(*), d(*), d_pl(*), ch(*), ch_pl(*), cmask(*), cmask_pl(*)
       real(c_float), intent(inout) :: Qout_prev(*), Qout_prev_pl(*)
       type(c_ptr), value :: Qout_post, Qout_post_pl
     end function ica_horizontal_limiter_thuburn_f32

     integer(c_int) function ica_vertical_limiter_thuburn(c, q_h, q_h_pl, q, q_pl, d, d_pl, ck, ck_pl) &
          bind(C, name="ica_vertical_limiter_thuburn")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: c
       real(c_double), intent(inout) :: q_h(*), q_h_pl(*)
       real(c_double), intent(in) :: q(*), q_pl(*), d(*), d_pl(*), ck(*), ck_pl(*)
     end function ica_vertical_limiter_thuburn
     integer(c_int) function ica_vertical_limiter_thuburn_f32(c, q_h, q_h_pl, q, q_pl, d, d_pl, ck, ck_pl) &
          bind(C, name="ica_vertical_limiter_thuburn_f32")
       import :: c_int, c_ptr, c_float
       type(c_ptr), value :: c
       real(c_float), intent(inout) :: q_h(*), q_h_pl(*)
       real(c_float), intent(in) :: q(*), q_pl(*), d(*), d_pl(*), ck(*), ck_pl(*)
     end function ica_vertical_limiter_thuburn_f32
  end interface

contains

  !> Nonzero library status: print ica_last_error() and stop (the reference's error path).
  subroutine ica_shim_check(rc, what)
    integer(c_int), intent(in) :: rc
    character(len=*), intent(in) :: what
    character(kind=c_char), pointer :: msg(:)
    integer :: n
    if (rc == 0) return
    call c_f_pointer(ica_last_error(), msg, [4096])
    n = 0
    do while (n < 4096)
       if (msg(n + 1) == c_null_char) exit
       n = n + 1
    end do
    write(*, '(A,A,I0,A,4096A)') what, ': libicoadv status ', rc, ': ', msg(1:n)
    stop
  end subroutine ica_shim_check

  !> Context over the driver's own arrays: ADM_* sizes of mod_misc, then the metrics.
  subroutine ica_shim_setup(device)
    integer, intent(in) :: device
    integer(c_int) :: sgp(ADM_lall), hp
    integer :: l
    do l = 1, ADM_lall
       sgp(l) = merge(1_c_int, 0_c_int, ADM_have_sgp(l))
    end do
    hp = merge(1_c_int, 0_c_int, ADM_have_pl)
    call ica_shim_check(ica_init_regions(int(ADM_gall_1d, c_int), int(ADM_kall, c_int), int(ADM_kmin, c_int), &
         int(ADM_kmax, c_int), int(ADM_lall, c_int), hp, sgp, int(device, c_int), ctx), 'ica_init_regions')
    call ica_shim_geometry()
  end subroutine ica_shim_setup

  !> Context over a whole grid (all 10*4^rlevel regions on this GPU): also runs the halo fills.
  subroutine ica_shim_setup_grid(glevel, rlevel, vlayer, device)
    integer, intent(in) :: glevel, rlevel, vlayer, device
    type(ica_dims) :: d
    d = ica_dims(int(glevel, c_int), int(rlevel, c_int), int(vlayer, c_int), int(device, c_int))
    call ica_shim_check(ica_init(d, ctx), 'ica_init')
    call ica_shim_geometry()
  end subroutine ica_shim_setup_grid

  !> The metrics are FP64 in the library (an FP32 copy is derived for the *_f32 entries).
  subroutine ica_shim_geometry()
    real(c_double), allocatable :: xr(:), xr_pl(:), p(:), p_pl(:), t(:), t_pl(:), a(:), a_pl(:)
    xr = real(reshape(GRD_xr, [size(GRD_xr)]), c_double)
    xr_pl = real(reshape(GRD_xr_pl, [size(GRD_xr_pl)]), c_double)
    p = real(reshape(GMTR_p, [size(GMTR_p)]), c_double)
    p_pl = real(reshape(GMTR_p_pl, [size(GMTR_p_pl)]), c_double)
    t = real(reshape(GMTR_t, [size(GMTR_t)]), c_double)
    t_pl = real(reshape(GMTR_t_pl, [size(GMTR_t_pl)]), c_double)
    a = real(reshape(GMTR_a, [size(GMTR_a)]), c_double)
    a_pl = real(reshape(GMTR_a_pl, [size(GMTR_a_pl)]), c_double)
    call ica_shim_check(ica_set_geometry(ctx, xr, xr_pl, p, p_pl, t, t_pl, a, a_pl), 'ica_set_geometry')
  end subroutine ica_shim_geometry

  subroutine ica_shim_finalize()
    if (c_associated(ctx)) call ica_shim_check(ica_finalize(ctx), 'ica_finalize')
    ctx = c_null_ptr
  end subroutine ica_shim_finalize

  !> horizontal_flux, dyn_horiz_adv_flux/src/mod_src_tracer.f90:42-90
  subroutine horizontal_flux(flx_h, flx_h_pl, GRD_xc, GRD_xc_pl, rho, rho_pl, rhovx, rhovx_pl, &
       rhovy, rhovy_pl, rhovz, rhovz_pl, dt)
    real(RP), intent(out) :: flx_h    (ADM_gall   ,ADM_kall,ADM_lall   ,6)
    real(RP), intent(out) :: flx_h_pl (ADM_gall_pl,ADM_kall,ADM_lall_pl  )
    real(RP), intent(out) :: GRD_xc   (ADM_gall   ,ADM_kall,ADM_lall   ,3,3)
    real(RP), intent(out) :: GRD_xc_pl(ADM_gall_pl,ADM_kall,ADM_lall_pl,  3)
    real(RP), intent(in)  :: rho      (ADM_gall   ,ADM_kall,ADM_lall   )
    real(RP), intent(in)  :: rho_pl   (ADM_gall_pl,ADM_kall,ADM_lall_pl)
    real(RP), intent(in)  :: rhovx    (ADM_gall   ,ADM_kall,ADM_lall   )
    real(RP), intent(in)  :: rhovx_pl (ADM_gall_pl,ADM_kall,ADM_lall_pl)
    real(RP), intent(in)  :: rhovy    (ADM_gall   ,ADM_kall,ADM_lall   )
    real(RP), intent(in)  :: rhovy_pl (ADM_gall_pl,ADM_kall,ADM_lall_pl)
    real(RP), intent(in)  :: rhovz    (ADM_gall   ,ADM_kall,ADM_lall   )
    real(RP), intent(in)  :: rhovz_pl (ADM_gall_pl,ADM_kall,ADM_lall_pl)
    real(RP), intent(in)  :: dt
#ifdef SINGLE
    call ica_shim_check(ica_horizontal_flux_f32(ctx, flx_h, flx_h_pl, GRD_xc, GRD_xc_pl, rho, rho_pl, &
         rhovx, rhovx_pl, rhovy, rhovy_pl, rhovz, rhovz_pl, real(dt, c_float)), 'horizontal_flux')
#else
    call ica_shim_check(ica_horizontal_flux(ctx, flx_h, flx_h_pl, GRD_xc, GRD_xc_pl, rho, rho_pl, &
         rhovx, rhovx_pl, rhovy, rhovy_pl, rhovz, rhovz_pl, real(dt, c_double)), 'horizontal_flux')
#endif
  end subroutine horizontal_flux

  !> horizontal_limiter_thuburn, dyn_horiz_adv_limiter/src/mod_src_tracer.f90:42-84
  subroutine horizontal_limiter_thuburn(q_a, q_a_pl, q, q_pl, d, d_pl, ch, ch_pl, cmask, cmask_pl, &
       Qout_prev, Qout_prev_pl, Qout_post, Qout_post_pl)
    real(RP), intent(inout) :: q_a     (ADM_gall   ,ADM_kall,ADM_lall   ,6)
    real(RP), intent(inout) :: q_a_pl  (ADM_gall_pl,ADM_kall,ADM_lall_pl  )
    real(RP), intent(in)    :: q       (ADM_gall   ,ADM_kall,ADM_lall     )
    real(RP), intent(in)    :: q_pl    (ADM_gall_pl,ADM_kall,ADM_lall_pl  )
    real(RP), intent(in)    :: d       (ADM_gall   ,ADM_kall,ADM_lall     )
    real(RP), intent(in)    :: d_pl    (ADM_gall_pl,ADM_kall,ADM_lall_pl  )
    real(RP), intent(in)    :: ch      (ADM_gall   ,ADM_kall,ADM_lall   ,6)
    real(RP), intent(in)    :: ch_pl   (ADM_gall_pl,ADM_kall,ADM_lall_pl  )
    real(RP), intent(in)    :: cmask   (ADM_gall   ,ADM_kall,ADM_lall   ,6)
    real(RP), intent(in)    :: cmask_pl(ADM_gall_pl,ADM_kall,ADM_lall_pl  )
    real(RP), intent(out)   :: Qout_prev   (ADM_gall   ,ADM_kall,ADM_lall   ,2)
    real(RP), intent(out)   :: Qout_prev_pl(ADM_gall_pl,ADM_kall,ADM_lall_pl,2)
    real(RP), intent(in), optional, target :: Qout_post   (ADM_gall   ,ADM_kall,ADM_lall   ,2)
    real(RP), intent(in), optional, target :: Qout_post_pl(ADM_gall_pl,ADM_kall,ADM_lall_pl,2)
    type(c_ptr) :: post, post_pl
    post = c_null_ptr
    post_pl = c_null_ptr
    if (present(Qout_post) .neqv. present(Qout_post_pl)) then
       write(*, *) 'horizontal_limiter_thuburn: give both Qout_post and Qout_post_pl, or neither'
       stop
    end if
    if (present(Qout_post)) then
       post = c_loc(Qout_post)
       post_pl = c_loc(Qout_post_pl)
    end if
#ifdef SINGLE
    call ica_shim_check(ica_horizontal_limiter_thuburn_f32(ctx, q_a, q_a_pl, q, q_pl, d, d_pl, ch, ch_pl, &
         cmask, cmask_pl, Qout_prev, Qout_prev_pl, post, post_pl), 'horizontal_limiter_thuburn')
#else
    call ica_shim_check(ica_horizontal_limiter_thuburn(ctx, q_a, q_a_pl, q, q_pl, d, d_pl, ch, ch_pl, &
         cmask, cmask_pl, Qout_prev, Qout_prev_pl, post, post_pl), 'horizontal_limiter_thuburn')
#endif
  end subroutine horizontal_limiter_thuburn

  !> vertical_limiter_thuburn, dyn_vert_adv_limiter/src/mod_src_tracer.f90:41-67
  subroutine vertical_limiter_thuburn(q_h, q_h_pl, q, q_pl, d, d_pl, ck, ck_pl)
    real(RP), intent(inout) :: q_h  (ADM_gall   ,ADM_kall,ADM_lall   )
    real(RP), intent(inout) :: q_h_pl(ADM_gall_pl,ADM_kall,ADM_lall_pl)
    real(RP), intent(in)    :: q    (ADM_gall   ,ADM_kall,ADM_lall   )
    real(RP), intent(in)    :: q_pl (ADM_gall_pl,ADM_kall,ADM_lall_pl)
    real(RP), intent(in)    :: d    (ADM_gall   ,ADM_kall,ADM_lall   )
    real(RP), intent(in)    :: d_pl (ADM_gall_pl,ADM_kall,ADM_lall_pl)
    real(RP), intent(in)    :: ck   (ADM_gall   ,ADM_kall,ADM_lall   ,2)
    real(RP), intent(in)    :: ck_pl(ADM_gall_pl,ADM_kall,ADM_lall_pl,2)
#ifdef SINGLE
    call ica_shim_check(ica_vertical_limiter_thuburn_f32(ctx, q_h, q_h_pl, q, q_pl, d, d_pl, ck, ck_pl), &
         'vertical_limiter_thuburn')
#else
    call ica_shim_check(ica_vertical_limiter_thuburn(ctx, q_h, q_h_pl, q, q_pl, d, d_pl, ck, ck_pl), &
         'vertical_limiter_thuburn')
#endif
  end subroutine vertical_limiter_thuburn

end module ica_shim
