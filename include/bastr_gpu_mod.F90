!-------------------------------------------------------------------------------------------------
! bastr_gpu_mod -- iso_c_binding interface of libbastr_gpu (include/bastr_gpu.h) for the Bastr
! Fortran driver.
!
! It replaces, on the driver side, the hot-path modules that the B200 library takes over:
!   mainloop / mainloop2D / mainloop3D and everything under them  (solution.F90:20-170)
!   quantity_prepare                                               (solution.F90:1288-1329)
!   allocation / deallocation                                      (fftwlink.F90:370-490)
!   mpisizedis_fftw, prepareplan_fftw_plan                         (fftwlink.F90:34-153, 284-303)
!   fft2d / fft3d / ifft2d / ifft3d                                (fftwlink.F90:324-368)
! The driver keeps Bastr.F90's readinput, read_initial_field / read_continue_field, listinit,
! listwrite and writeflfed (readwrite.F90, utility.F90, hdf5io.F90) and the file formats.
!
! Build (a Fortran compiler and the reference's h5pfc wrapper are needed; none exists in this
! repository's build environment, so this file is compiled only on the driver's side):
!   h5pfc -O3 -c bastr_gpu_mod.F90
!   h5pfc -O3 ... bastr_gpu_mod.o Bastr.F90 ... -L<repo>/bastr_b200 -lbastr_gpu -Wl,-rpath,<repo>/bastr_b200
! Every function returns 0 on success and a negative status otherwise (BASTR_E_* below); the
! message of the last failed call on a handle comes from bastr_error_message.
!-------------------------------------------------------------------------------------------------
module bastr_gpu_mod
  use, intrinsic :: iso_c_binding
  implicit none
  private

  integer(c_int), parameter, public :: BASTR_OK = 0
  integer(c_int), parameter, public :: BASTR_E_INVALID = -1
  integer(c_int), parameter, public :: BASTR_E_UNSUPPORTED = -2
  integer(c_int), parameter, public :: BASTR_E_CUDA = -3
  integer(c_int), parameter, public :: BASTR_E_NAN = -4       ! "E" is a NaN (solution.F90:81)
  integer(c_int), parameter, public :: BASTR_E_STATE = -5
  integer(c_int), parameter, public :: BASTR_E_TOO_LARGE = -6
  integer(c_int32_t), parameter, public :: BASTR_FP64 = 0, BASTR_FP32 = 1

  ! the datin/input.dat values the time step reads (readwrite.F90:35-44), plus GPU knobs
  type, bind(c), public :: bastr_params
    integer(c_int32_t) :: ia, ja, ka
    real(c_double)     :: ref_tem, reynolds, deltat
    integer(c_int32_t) :: kmax, timemethod, forcemethod, forcek
    real(c_double)     :: target_energy
    integer(c_int32_t) :: lprojectd, precision, device, velgrad_every
  end type

  ! one main-loop iteration: the values listwrite logs (solution.F90:54-97)
  type, bind(c), public :: bastr_step_out
    integer(c_int64_t) :: nstep
    real(c_double)     :: time, Esspe, Edspe, k2Edspe, kMEdspe
    real(c_double)     :: velgrad(8)
    real(c_double)     :: factor, E
    real(c_double)     :: energy, Fen
  end type

  public :: bastr_create, bastr_destroy, bastr_set_state, bastr_get_state, bastr_set_counters, &
            bastr_get_counters, bastr_step, bastr_spectra, bastr_fft, bastr_transfer, bastr_hitgen, &
            bastr_h5_write_field, bastr_h5_read_field, bastr_last_error, bastr_error_message

  interface
    integer(c_int) function bastr_create(p, h) bind(c, name='bastr_create')
      import :: c_int, c_ptr, bastr_params
      type(bastr_params), intent(in) :: p
      type(c_ptr), intent(out) :: h
    end function

    integer(c_int) function bastr_destroy(h) bind(c, name='bastr_destroy')
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function

    ! u1, u2[, u3]: real(8) (1:ia,1:ja[,1:ka]), x fastest; u3 is ignored in 2D (pass u1)
    integer(c_int) function bastr_set_state(h, u1, u2, u3) bind(c, name='bastr_set_state')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in) :: u1(*), u2(*), u3(*)
    end function

    integer(c_int) function bastr_get_state(h, u1, u2, u3) bind(c, name='bastr_get_state')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: u1(*), u2(*), u3(*)
    end function

    integer(c_int) function bastr_set_counters(h, nstep, time) bind(c, name='bastr_set_counters')
      import :: c_int, c_ptr, c_int64_t, c_double
      type(c_ptr), value :: h
      integer(c_int64_t), value :: nstep
      real(c_double), value :: time
    end function

    integer(c_int) function bastr_get_counters(h, nstep, time) bind(c, name='bastr_get_counters')
      import :: c_int, c_ptr, c_int64_t, c_double
      type(c_ptr), value :: h
      integer(c_int64_t), intent(out) :: nstep
      real(c_double), intent(out) :: time
    end function

    ! n iterations of the main loop; shells(0:allkmax, 2, n) = Es then Ed per step.  Returns
    ! BASTR_E_NAN at the first step whose Es+Ed is NaN, with that step's state and counters.
    integer(c_int) function bastr_step(h, n, out, shells) bind(c, name='bastr_step')
      import :: c_int, c_ptr, c_int32_t, c_double, bastr_step_out
      type(c_ptr), value :: h
      integer(c_int32_t), value :: n
      type(bastr_step_out), intent(out) :: out(*)
      real(c_double), intent(out) :: shells(*)
    end function

    integer(c_int) function bastr_spectra(h, kn, Es, Ed, Ecount) bind(c, name='bastr_spectra')
      import :: c_int, c_ptr, c_double, c_int64_t
      type(c_ptr), value :: h
      real(c_double), intent(out) :: kn(*), Es(*), Ed(*)
      integer(c_int64_t), intent(out) :: Ecount(*)
    end function

    ! in place on a full complex(8) grid: dir = -1 forward scaled 1/N (fft2d/fft3d),
    ! dir = +1 backward unscaled (ifft2d/ifft3d)
    integer(c_int) function bastr_fft(h, array, dir) bind(c, name='bastr_fft')
      import :: c_int, c_ptr, c_double_complex, c_int32_t
      type(c_ptr), value :: h
      complex(c_double_complex), intent(inout) :: array(*)
      integer(c_int32_t), value :: dir
    end function

    ! Bastrpp transfer2d/transfer3d (Bastrpp.F90:174-305, 418-599) on the current state
    integer(c_int) function bastr_transfer(h, T, T1, T2) bind(c, name='bastr_transfer')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: T(*), T1(*), T2(*)
    end function

    ! Bastrpp hitgen2d/hitgen3d (variant 0) and hitgen2dbis (variant 1), Bastrpp.F90:601-1005
    integer(c_int) function bastr_hitgen(h, variant, seed, u1, u2, u3, angle, stats) bind(c, name='bastr_hitgen')
      import :: c_int, c_ptr, c_int32_t, c_int64_t, c_double
      type(c_ptr), value :: h
      integer(c_int32_t), value :: variant
      integer(c_int64_t), value :: seed
      real(c_double), intent(out) :: u1(*), u2(*), u3(*), angle(*), stats(8)
    end function

    ! field files without libhdf5 (the HDF5 subset of hdf5io.F90's files): writeflfed's
    ! u1,u2[,u3] + nstep/time (nstep < 0: no counters, as in flowini files), and the reads of
    ! read_initial_field / read_continue_field (pass c_null_ptr-backed optionals as needed)
    integer(c_int) function bastr_h5_write_field(path, ia, ja, ka, u1, u2, u3, nstep, time) &
        bind(c, name='bastr_h5_write_field')
      import :: c_int, c_char, c_int32_t, c_int64_t, c_double
      character(kind=c_char), intent(in) :: path(*)
      integer(c_int32_t), value :: ia, ja, ka
      real(c_double), intent(in) :: u1(*), u2(*), u3(*)
      integer(c_int64_t), value :: nstep
      real(c_double), value :: time
    end function

    integer(c_int) function bastr_h5_read_field(path, ia, ja, ka, u1, u2, u3, nstep, time) &
        bind(c, name='bastr_h5_read_field')
      import :: c_int, c_char, c_int32_t, c_int64_t, c_double
      character(kind=c_char), intent(in) :: path(*)
      integer(c_int32_t), value :: ia, ja, ka
      real(c_double), intent(out) :: u1(*), u2(*), u3(*)
      integer(c_int64_t), intent(out) :: nstep
      real(c_double), intent(out) :: time
    end function

    integer(c_int) function bastr_last_error(h, buf, n) bind(c, name='bastr_last_error')
      import :: c_int, c_ptr, c_char, c_int32_t
      type(c_ptr), value :: h
      character(kind=c_char), intent(out) :: buf(*)
      integer(c_int32_t), value :: n
    end function
  end interface

contains

  ! The message of the last failed call on h, as a Fortran string (the reference's `stop` text).
  function bastr_error_message(h) result(msg)
    type(c_ptr), intent(in) :: h
    character(len=512) :: msg
    character(kind=c_char) :: buf(512)
    integer(c_int) :: n, i
    n = bastr_last_error(h, buf, int(size(buf), c_int32_t))
    msg = ' '
    do i = 1, min(int(n), size(buf) - 1)
      msg(i:i) = buf(i)
    end do
  end function

end module bastr_gpu_mod
