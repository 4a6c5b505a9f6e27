!-------------------------------------------------------------------------------!
! adcgpu_iface.F90 -- ISO_C_BINDING interface to libadcgpu (include/adcgpu.h).
!
! A Fortran host (ADCIRC's TIMESTEP / GWCE_New) uses this module to call the
! B200 implementation of the 2DDI hot path.  The types mirror adc_params_t,
! adc_arrays_t, adc_step_t and adc_stepout_t field for field; array members
! are C_LOC of the host's module arrays (column-major, 1-based contents).
! Not compiled in this repository (no Fortran compiler is installed); built by
! the host's own CMake with -lstdc++ and the library on the link line.
!-------------------------------------------------------------------------------!
module adcgpu_iface
   use, intrinsic :: iso_c_binding
   implicit none
   private

   integer(c_int), parameter, public :: ADC_OK = 0, ADC_ERR_DIAG = 1
   integer(c_int), parameter, public :: ADC_PREC_FP64 = 0, ADC_PREC_MIXED = 1

   type, bind(C), public :: adc_params_t
      real(c_double) :: dt, g, a00, b00, c00, h0, velmin, slim, hbreak, ftheta, &
                        fgamma, convcr, prbckgrnd_mh2o
      integer(c_int) :: ifnlfa, ifnlct, ifnlcat, nolifa, iflinbf, ifnlbf, ifhybf, &
                        itmax, nws, ifwind, isldia, pad_
   end type

   type, bind(C), public :: adc_arrays_t
      integer(c_int) :: np, ne, mnei, neta, nbfr, nvel, nvelme, nbou
      type(c_ptr) :: x, y, dp, nm, nneigh, neitab, fdxe, fdye, areas, csr_position
      type(c_ptr) :: tau0var, evm, fric, corif
      type(c_ptr) :: nbd, amig, per, face, ff, emo, efa, nbv, lbcodei, csii, siii, me2gw
      type(c_ptr) :: bndlen2o3
      type(c_ptr) :: eta1, eta2, etas, uu1, vv1, uu2, vv2, qx1, qy1, qx2, qy2, h1, h2
      type(c_ptr) :: tk, tkm, nodecode, nnodecode, noff, mju, totalarea, alphal
      type(c_ptr) :: wsx1, wsy1, wsx2, wsy2, pr1, pr2, coef, obccoef
      type(c_ptr) :: gwce_lv, mom_lv_x, mom_lv_y
      type(c_ptr) :: nelezng, zngif1, zngif2, zngif3, neitabele
      type(c_ptr) :: barlanht, barlancfsp
      type(c_ptr) :: ibconn, barinht, barincfsb, barincfsp, nvell
      type(c_ptr) :: pipeht, pipecoef, pipediam
   end type

   type, bind(C), public :: adc_step_t
      integer(c_int) :: it, pad_
      real(c_double) :: timeloc, timeh, rampelev, rampmete, rampextflux, rampintflux
   end type

   type, bind(C), public :: adc_flux_t
      integer(c_int) :: nffr, flux_settling_it
      type(c_ptr) :: famig, fper, fff, fface, qnam, qnph, enam, enph
   end type

   ! non-periodic boundary series (fort.19 elevations, fort.20 fluxes)
   type, bind(C), public :: adc_series_t
      integer(c_int) :: nrec, flux_settling_it
      real(c_double) :: interval, start_time
      type(c_ptr) :: values, values2
   end type

   type, bind(C), public :: adc_stepout_t
      integer(c_int) :: numitr, ier, ncchange, status
      real(c_double) :: ep, zeta, cme
      integer(c_int) :: n_w1_events, pad_
   end type

   ! step-to-step module scalars (NCChange, EP, RPARM(1:2), q1, vortex track)
   type, bind(C), public :: adc_scalars_t
      integer(c_int) :: ncchange, q1, vortex_counter, pad_
      real(c_double) :: ep, rparm1, rparm2, vortex_wtratio
   end type

   integer(c_int), parameter, public :: ADC_WARM_START = 2, ADC_F32_ASSEMBLY = 4, &
                                        ADC_F32_SPMV = 8, ADC_F32_MOMENTUM = 16

   type, bind(C), public :: adc_vortex_fix_t
      real(c_double) :: time, x, y, cpress, vmax, rmw, tvx, tvy
   end type

   type, bind(C), public :: adc_vortex_t
      integer(c_int) :: nfix, avg_minute, hemisphere, pad_
      real(c_double) :: start_time, bladj, rho_air, wind_mult, drag_limit
      type(c_ptr) :: fix
   end type

   public :: adc_jcg, adc_dfault, adc_gpu_bind, adc_gpu_free, adc_shift_friction, &
             adc_gwce_new, adc_wetdry, adc_momentum, adc_timestep, adc_sync_to_host, &
             adc_sync_from_host, adc_set_met, adc_set_vortex, adc_hotstart_write, &
             adc_hotstart_read, adc_set_flux, adc_set_elev_series, adc_set_flux_series

   interface
      ! drop-in for ITPACK jcg (itpackv.F:63): identical argument list
      subroutine adc_jcg(n, ndim, maxnz, jcoef, coef, rhs, u, iwksp, nw, wksp, &
                         iparm, rparm, ier) bind(C, name="adc_jcg")
         import :: c_int, c_double
         integer(c_int), intent(in) :: n, ndim, maxnz, nw
         integer(c_int), intent(inout) :: jcoef(ndim, maxnz), iwksp(*), iparm(12), ier
         real(c_double), intent(inout) :: coef(ndim, maxnz), rhs(n), u(n), wksp(nw), rparm(12)
      end subroutine

      subroutine adc_dfault(iparm, rparm) bind(C, name="adc_dfault")
         import :: c_int, c_double
         integer(c_int), intent(out) :: iparm(12)
         real(c_double), intent(out) :: rparm(12)
      end subroutine

      integer(c_int) function adc_gpu_bind(p, a, prec, ctx) bind(C, name="adc_gpu_bind")
         import :: c_int, c_ptr, adc_params_t, adc_arrays_t
         type(adc_params_t), intent(in) :: p
         type(adc_arrays_t), intent(in) :: a
         integer(c_int), value :: prec
         type(c_ptr), intent(out) :: ctx
      end function

      integer(c_int) function adc_gpu_free(ctx) bind(C, name="adc_gpu_free")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function

      integer(c_int) function adc_shift_friction(ctx, s) bind(C, name="adc_shift_friction")
         import :: c_int, c_ptr, adc_step_t
         type(c_ptr), value :: ctx
         type(adc_step_t), intent(in) :: s
      end function

      integer(c_int) function adc_gwce_new(ctx, s, o) bind(C, name="adc_gwce_new")
         import :: c_int, c_ptr, adc_step_t, adc_stepout_t
         type(c_ptr), value :: ctx
         type(adc_step_t), intent(in) :: s
         type(adc_stepout_t), intent(out) :: o
      end function

      integer(c_int) function adc_wetdry(ctx, s, o) bind(C, name="adc_wetdry")
         import :: c_int, c_ptr, adc_step_t, adc_stepout_t
         type(c_ptr), value :: ctx
         type(adc_step_t), intent(in) :: s
         type(adc_stepout_t), intent(out) :: o
      end function

      integer(c_int) function adc_momentum(ctx, s) bind(C, name="adc_momentum")
         import :: c_int, c_ptr, adc_step_t
         type(c_ptr), value :: ctx
         type(adc_step_t), intent(in) :: s
      end function

      integer(c_int) function adc_timestep(ctx, s, o) bind(C, name="adc_timestep")
         import :: c_int, c_ptr, adc_step_t, adc_stepout_t
         type(c_ptr), value :: ctx
         type(adc_step_t), intent(in) :: s
         type(adc_stepout_t), intent(out) :: o
      end function

      integer(c_int) function adc_sync_to_host(ctx) bind(C, name="adc_sync_to_host")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function

      integer(c_int) function adc_sync_from_host(ctx) bind(C, name="adc_sync_from_host")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function

      integer(c_int) function adc_set_met(ctx, wsx2, wsy2, pr2) bind(C, name="adc_set_met")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(in) :: wsx2(*), wsy2(*), pr2(*)
      end function

      ! NWS = 8 vortex track (fix points in mesh coordinates; see adcgpu.h)
      integer(c_int) function adc_set_vortex(ctx, v) bind(C, name="adc_set_vortex")
         import :: c_int, c_ptr, adc_vortex_t
         type(c_ptr), value :: ctx
         type(adc_vortex_t), intent(in) :: v
      end function

      ! periodic specified normal flux (timestep.F:861-880)
      integer(c_int) function adc_set_flux(ctx, f) bind(C, name="adc_set_flux")
         import :: c_int, c_ptr, adc_flux_t
         type(c_ptr), value :: ctx
         type(adc_flux_t), intent(in) :: f
      end function

      ! fort.19 (NPEBC, gwce.F:1659-1674) and fort.20 (NFFR <= 0,
      ! timestep.F:882-903) records, uploaded once after bind
      integer(c_int) function adc_set_elev_series(ctx, s) bind(C, name="adc_set_elev_series")
         import :: c_int, c_ptr, adc_series_t
         type(c_ptr), value :: ctx
         type(adc_series_t), intent(in) :: s
      end function

      integer(c_int) function adc_set_flux_series(ctx, s) bind(C, name="adc_set_flux_series")
         import :: c_int, c_ptr, adc_series_t
         type(c_ptr), value :: ctx
         type(adc_series_t), intent(in) :: s
      end function

      ! hotstart dump/load (write_output.F:4429-5582, hstart.F:47-2048);
      ! path is a NUL-terminated character array (trim(name)//c_null_char)
      integer(c_int) function adc_hotstart_write(ctx, path) bind(C, name="adc_hotstart_write")
         import :: c_int, c_ptr, c_char
         type(c_ptr), value :: ctx
         character(kind=c_char), intent(in) :: path(*)
      end function

      integer(c_int) function adc_hotstart_read(ctx, path) bind(C, name="adc_hotstart_read")
         import :: c_int, c_ptr, c_char
         type(c_ptr), value :: ctx
         character(kind=c_char), intent(in) :: path(*)
      end function

      integer(c_int) function adc_get_scalars(ctx, sc) bind(C, name="adc_get_scalars")
         import :: c_int, c_ptr, adc_scalars_t
         type(c_ptr), value :: ctx
         type(adc_scalars_t), intent(out) :: sc
      end function
   end interface
end module adcgpu_iface
