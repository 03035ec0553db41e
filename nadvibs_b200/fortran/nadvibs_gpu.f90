! ISO_C_BINDING interface to libnadvibs_gpu.so (include/nadvibs.h) for the NadVibS Fortran
! driver.  The reference is built with -i8, so every integer here is integer(c_int64_t);
! reals are real(c_double); strings must end with c_null_char.  Status codes: 0 ok, < 0 error
! (nvb_last_error gives the message).
module nadvibs_gpu
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: NVB_FP64 = 0, NVB_MIXED = 1

  type, bind(C) :: nvb_options
    integer(c_int64_t) :: precision, device, quirk_cubic, quirk_lower, archive_max, hv_kernel, seed
  end type

  interface
    integer(c_int) function nvb_options_default(o) bind(C, name="nvb_options_default")
      import :: c_int, nvb_options
      type(nvb_options), intent(out) :: o
    end function
    integer(c_int) function nvb_create_from_files(basis, nadvibs, opt, h) bind(C, name="nvb_create_from_files")
      import :: c_int, c_char, c_ptr, nvb_options
      character(kind=c_char), dimension(*), intent(in) :: basis, nadvibs
      type(nvb_options), intent(in) :: opt
      type(c_ptr), intent(out) :: h
    end function
    integer(c_int) function nvb_destroy(h) bind(C, name="nvb_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    type(c_ptr) function nvb_last_error() bind(C, name="nvb_last_error")
      import :: c_ptr
    end function
    integer(c_int) function nvb_set_reorthog(h, reorthog, chkorthog) bind(C, name="nvb_set_reorthog")
      import :: c_int, c_int64_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int64_t), value :: reorthog, chkorthog
    end function
    integer(c_int) function nvb_set_archive(h, kind, max_vectors, path) bind(C, name="nvb_set_archive")
      import :: c_int, c_int64_t, c_char, c_ptr
      type(c_ptr), value :: h
      integer(c_int64_t), value :: kind, max_vectors
      character(kind=c_char), dimension(*), intent(in) :: path
    end function
    integer(c_int) function nvb_reorth_log(h, max_entries, iteration, lo, hi, count) bind(C, name="nvb_reorth_log")
      import :: c_int, c_int64_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int64_t), value :: max_entries
      integer(c_int64_t), intent(out) :: iteration(*), lo(*), hi(*), count
    end function
    integer(c_int) function nvb_reorth_omega(h, n, omega1, omega2, omega2_step) bind(C, name="nvb_reorth_omega")
      import :: c_int, c_int64_t, c_double, c_ptr
      type(c_ptr), value :: h
      integer(c_int64_t), value :: n
      real(c_double), intent(out) :: omega1(*), omega2(*), omega2_step(*)
    end function
    integer(c_int) function nvb_measure_fma(dtype, seconds, flops_per_s) bind(C, name="nvb_measure_fma")
      import :: c_int, c_int64_t, c_double
      integer(c_int64_t), value :: dtype
      real(c_double), value :: seconds
      real(c_double), intent(out) :: flops_per_s
    end function
    integer(c_int) function nvb_measure_tile_stream(tile_bytes, slots, ctas_per_sm, seconds, bytes_per_s) &
        bind(C, name="nvb_measure_tile_stream")
      import :: c_int, c_int64_t, c_double
      integer(c_int64_t), value :: tile_bytes, slots, ctas_per_sm
      real(c_double), value :: seconds
      real(c_double), intent(out) :: bytes_per_s
    end function
    integer(c_int) function nvb_hv_tile_stream(h, dtype, bytes_per_hv, tile_bytes, slots, ctas_per_sm) &
        bind(C, name="nvb_hv_tile_stream")
      import :: c_int, c_int64_t, c_double, c_ptr
      type(c_ptr), value :: h
      integer(c_int64_t), value :: dtype
      real(c_double), intent(out) :: bytes_per_hv
      integer(c_int64_t), intent(out) :: tile_bytes, slots, ctas_per_sm
    end function
    integer(c_int) function nvb_write_seed_report(h, path) bind(C, name="nvb_write_seed_report")
      import :: c_int, c_char, c_ptr
      type(c_ptr), value :: h
      character(kind=c_char), dimension(*), intent(in) :: path
    end function
    integer(c_int) function nvb_write_header(h, path) bind(C, name="nvb_write_header")
      import :: c_int, c_char, c_ptr
      type(c_ptr), value :: h
      character(kind=c_char), dimension(*), intent(in) :: path
    end function
    integer(c_int) function nvb_seed(h, weights) bind(C, name="nvb_seed")
      import :: c_int, c_ptr
      type(c_ptr), value :: h, weights
    end function
    integer(c_int) function nvb_lanczos(h, niter, alpha, beta) bind(C, name="nvb_lanczos")
      import :: c_int, c_int64_t, c_double, c_ptr
      type(c_ptr), value :: h
      integer(c_int64_t), value :: niter
      real(c_double), dimension(*), intent(out) :: alpha, beta
    end function
    integer(c_int) function nvb_save_restart(h, dir, vecdir) bind(C, name="nvb_save_restart")
      import :: c_int, c_char, c_ptr
      type(c_ptr), value :: h
      character(kind=c_char), dimension(*), intent(in) :: dir, vecdir
    end function
    integer(c_int) function nvb_load_restart(h, dir, vecdir) bind(C, name="nvb_load_restart")
      import :: c_int, c_char, c_ptr
      type(c_ptr), value :: h
      character(kind=c_char), dimension(*), intent(in) :: dir, vecdir
    end function
    integer(c_int) function nvb_write_eigenvalues(h, path) bind(C, name="nvb_write_eigenvalues")
      import :: c_int, c_char, c_ptr
      type(c_ptr), value :: h
      character(kind=c_char), dimension(*), intent(in) :: path
    end function
    integer(c_int) function nvb_ritz(h, n, e, bji, inten, sign, vect) bind(C, name="nvb_ritz")
      import :: c_int, c_int64_t, c_double, c_ptr
      type(c_ptr), value :: h
      integer(c_int64_t), value :: n
      real(c_double), dimension(*), intent(out) :: e, bji, inten
      integer(c_int64_t), dimension(*), intent(out) :: sign
      type(c_ptr), value :: vect
    end function
    integer(c_int) function nvb_lead_contributors(h, nroots, k, state, index, c2, phase, pct, rootinfo) &
        bind(C, name="nvb_lead_contributors")
      import :: c_int, c_int64_t, c_double, c_char, c_ptr
      type(c_ptr), value :: h
      integer(c_int64_t), value :: nroots, k
      integer(c_int64_t), dimension(*), intent(out) :: state, index, phase
      real(c_double), dimension(*), intent(out) :: c2, pct
      character(kind=c_char), dimension(*), intent(in) :: rootinfo
    end function
    integer(c_int) function nvb_spin_orbit(h, soroots, nroots, energy_ev, amp, overlap, sodata) &
        bind(C, name="nvb_spin_orbit")
      import :: c_int, c_int64_t, c_double, c_char, c_ptr
      type(c_ptr), value :: h
      integer(c_int64_t), value :: soroots, nroots
      real(c_double), dimension(*), intent(out) :: energy_ev, amp, overlap
      character(kind=c_char), dimension(*), intent(in) :: sodata
    end function
    ! gradient path (no reference counterpart): checkpoints of the forward, the reverse
    ! sweep through the recurrence (k = 0: automatic plan within the memory budget), its
    ! budget and the plan it used
    integer(c_int) function nvb_set_checkpoints(h, k) bind(C, name="nvb_set_checkpoints")
      import :: c_int, c_int64_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int64_t), value :: k
    end function
    integer(c_int) function nvb_lanczos_backward(h, n, alpha_bar, beta_bar, k, grad) &
        bind(C, name="nvb_lanczos_backward")
      import :: c_int, c_int64_t, c_double, c_ptr
      type(c_ptr), value :: h
      integer(c_int64_t), value :: n, k
      real(c_double), dimension(*), intent(in) :: alpha_bar, beta_bar
      real(c_double), dimension(*), intent(out) :: grad
    end function
    integer(c_int) function nvb_set_backward_memory(h, nbytes) bind(C, name="nvb_set_backward_memory")
      import :: c_int, c_int64_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int64_t), value :: nbytes
    end function
    integer(c_int) function nvb_backward_plan(h, plan) bind(C, name="nvb_backward_plan")
      import :: c_int, c_int64_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int64_t), dimension(4), intent(out) :: plan
    end function
  end interface
end module nadvibs_gpu
