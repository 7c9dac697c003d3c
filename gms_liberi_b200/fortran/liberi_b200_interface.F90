!! liberi_b200_interface.F90 -- Fortran front end of the B200 Fock-build engine.
!!
!! Drop-in for libERI's modules `liberi_interface` (src/interface/liberi_interface.F90)
!! and `gamess_liberi_wrapper` (src/interface/gms_liberi_wrapper.F90): same module
!! names, procedure names and argument lists, so GAMESS and the reference's test
!! programs link against libliberi_b200.so unchanged.  Every procedure calls the C
!! ABI of include/liberi_b200.h through iso_c_binding; a non-zero status is printed
!! with the engine's message and stops the program with `error stop 1`, as the
!! reference does (liberi_interface.F90:219-222, gms_liberi_wrapper.F90:117-127).
!!
!! Integer arguments are default `integer` in the reference; they are passed to the
!! C ABI as c_int (int32_t), as the reference's own notes require.  Build (where a
!! Fortran compiler exists):
!!   gfortran -c liberi_b200_interface.F90 && gfortran prog.F90 liberi_b200_interface.o \
!!            -L<path>/gms_liberi_b200/_build -lliberi_b200
module liberi_b200_c
  use, intrinsic :: iso_c_binding
  implicit none
  interface
    integer(c_int) function liberi_c_create(h) bind(C, name="liberi_c_create")
      import :: c_int, c_ptr
      type(c_ptr), intent(out) :: h
    end function
    integer(c_int) function liberi_c_destroy(h) bind(C, name="liberi_c_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function liberi_c_cleanup(h) bind(C, name="liberi_c_cleanup")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function liberi_c_setup(h, nsh, natoms, num_bas, mxgtot, ang_mom, contr_num, sh_loc, &
                                           atom_num, atom_loc, start_bas, end_bas, exponents, cs, cp, cd, cf, &
                                           coords, schwrz, my_rank, num_procs) bind(C, name="liberi_c_setup")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: nsh, natoms, num_bas, mxgtot, my_rank, num_procs
      integer(c_int), intent(in) :: ang_mom(*), contr_num(*), sh_loc(*), atom_num(*), atom_loc(*), &
                                    start_bas(*), end_bas(*)
      real(c_double), intent(in) :: exponents(*), cs(*), cp(*), cd(*), cf(*), coords(*), schwrz(*)
    end function
    integer(c_int) function liberi_c_fock_build(h, density, fock, n) bind(C, name="liberi_c_fock_build")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in) :: density(*)
      real(c_double), intent(inout) :: fock(*)
      integer(c_int), value :: n
    end function
    integer(c_int) function liberi_c_last_error(buf, n) bind(C, name="liberi_c_last_error")
      import :: c_int, c_char
      character(kind=c_char), intent(out) :: buf(*)
      integer(c_int), value :: n
    end function
  end interface
contains
  subroutine liberi_b200_check(rc, where)
    integer(c_int), intent(in) :: rc
    character(len=*), intent(in) :: where
    character(kind=c_char) :: buf(512)
    integer(c_int) :: ignored
    integer :: i
    character(len=512) :: msg
    if (rc == 0) return
    ignored = liberi_c_last_error(buf, 512_c_int)
    msg = ' '
    do i = 1, 512
      if (buf(i) == c_null_char) exit
      msg(i:i) = buf(i)
    end do
    write (*, *) "ERROR in ", where, ": ", trim(msg)
    error stop 1
  end subroutine
end module liberi_b200_c

module liberi_interface
  use, intrinsic :: iso_c_binding
  use liberi_b200_c
  implicit none
  private
  public :: liberi_handle_t, liberi_create, liberi_destroy, liberi_setup, liberi_fock_build, liberi_cleanup

  type :: liberi_handle_t
    private
    type(c_ptr) :: h = c_null_ptr
  end type liberi_handle_t

contains

  subroutine liberi_create(handle)
    type(liberi_handle_t), intent(out) :: handle
    call liberi_b200_check(liberi_c_create(handle%h), "liberi_create")
  end subroutine

  subroutine liberi_destroy(handle)
    type(liberi_handle_t), intent(inout) :: handle
    if (c_associated(handle%h)) call liberi_b200_check(liberi_c_destroy(handle%h), "liberi_destroy")
    handle%h = c_null_ptr
  end subroutine

  subroutine liberi_setup(handle, nsh_in, natoms_in, num_bas_in, mxgtot_in, ang_mom_in, contr_num_in, &
                          sh_loc_in, atom_num_in, atom_loc_in, start_bas_in, end_bas_in, exponents_in, &
                          contr_coef_s_in, contr_coef_p_in, contr_coef_d_in, contr_coef_f_in, coords_in, &
                          schwrz_int_in, my_rank_in, num_procs_in)
    type(liberi_handle_t), intent(inout) :: handle
    integer, intent(in) :: nsh_in, natoms_in, num_bas_in, mxgtot_in, my_rank_in, num_procs_in
    integer, intent(in) :: ang_mom_in(nsh_in), contr_num_in(nsh_in), sh_loc_in(nsh_in), atom_num_in(nsh_in), &
                           atom_loc_in(nsh_in), start_bas_in(nsh_in), end_bas_in(nsh_in)
    real(c_double), intent(in) :: exponents_in(mxgtot_in*nsh_in), contr_coef_s_in(mxgtot_in*nsh_in), &
                                  contr_coef_p_in(mxgtot_in*nsh_in), contr_coef_d_in(mxgtot_in*nsh_in), &
                                  contr_coef_f_in(mxgtot_in*nsh_in), coords_in(3*natoms_in), &
                                  schwrz_int_in((nsh_in*(nsh_in + 1))/2)
    if (.not. c_associated(handle%h)) call liberi_create(handle)
    call liberi_b200_check(liberi_c_setup(handle%h, int(nsh_in, c_int), int(natoms_in, c_int), &
                           int(num_bas_in, c_int), int(mxgtot_in, c_int), int(ang_mom_in, c_int), &
                           int(contr_num_in, c_int), int(sh_loc_in, c_int), int(atom_num_in, c_int), &
                           int(atom_loc_in, c_int), int(start_bas_in, c_int), int(end_bas_in, c_int), &
                           exponents_in, contr_coef_s_in, contr_coef_p_in, contr_coef_d_in, contr_coef_f_in, &
                           coords_in, schwrz_int_in, int(my_rank_in, c_int), int(num_procs_in, c_int)), &
                           "liberi_setup")
  end subroutine

  subroutine liberi_fock_build(handle, density_in, fock_out, matrix_size)
    type(liberi_handle_t), intent(inout) :: handle
    integer, intent(in) :: matrix_size
    real(c_double), intent(in) :: density_in(matrix_size)
    real(c_double), intent(inout) :: fock_out(matrix_size)
    if (.not. c_associated(handle%h)) then
      write (*, *) "ERROR: liberi_fock_build called before liberi_setup"
      error stop 1
    end if
    call liberi_b200_check(liberi_c_fock_build(handle%h, density_in, fock_out, int(matrix_size, c_int)), &
                           "liberi_fock_build")
  end subroutine

  subroutine liberi_cleanup(handle)
    type(liberi_handle_t), intent(inout) :: handle
    if (c_associated(handle%h)) call liberi_b200_check(liberi_c_cleanup(handle%h), "liberi_cleanup")
  end subroutine

end module liberi_interface

module gamess_liberi_wrapper
  use, intrinsic :: iso_c_binding
  use liberi_interface
  implicit none
  private
  public :: liberi_init, liberi_fock, liberi_finalize

  type(liberi_handle_t), save :: handle
  logical, save :: is_initialized = .false.
  integer, save :: matrix_size = 0

contains

  subroutine liberi_init(natoms, num_bas, nsh, mxgtot, ang_mom, contr_num, sh_loc, atom_num, atom_loc, &
                         start_bas, end_bas, exponents, contr_coef_s, contr_coef_p, contr_coef_d, contr_coef_f, &
                         coords, schwrz_int, my_rank, num_procs)
    integer, intent(in) :: natoms, num_bas, nsh, mxgtot, my_rank, num_procs
    integer, intent(in) :: ang_mom(nsh), contr_num(nsh), sh_loc(nsh), atom_num(nsh), atom_loc(nsh), &
                           start_bas(nsh), end_bas(nsh)
    real(c_double), intent(in) :: exponents(mxgtot*nsh), contr_coef_s(mxgtot*nsh), contr_coef_p(mxgtot*nsh), &
                                  contr_coef_d(mxgtot*nsh), contr_coef_f(mxgtot*nsh), coords(3*natoms), &
                                  schwrz_int((nsh*(nsh + 1))/2)
    if (is_initialized) then
      call liberi_cleanup(handle)
      call liberi_destroy(handle)
    end if
    call liberi_create(handle)
    call liberi_setup(handle, nsh, natoms, num_bas, mxgtot, ang_mom, contr_num, sh_loc, atom_num, atom_loc, &
                      start_bas, end_bas, exponents, contr_coef_s, contr_coef_p, contr_coef_d, contr_coef_f, &
                      coords, schwrz_int, my_rank, num_procs)
    matrix_size = (num_bas*(num_bas + 1))/2
    is_initialized = .true.
  end subroutine

  subroutine liberi_fock(density, fock, n)
    integer, intent(in) :: n
    real(c_double), intent(in) :: density(n)
    real(c_double), intent(inout) :: fock(n)
    if (.not. is_initialized) then
      write (*, *) "ERROR: liberi_fock called before liberi_init"
      error stop 1
    end if
    if (n /= matrix_size) then
      write (*, *) "ERROR: matrix size mismatch in liberi_fock"
      write (*, *) "  Expected:", matrix_size
      write (*, *) "  Got:", n
      error stop 1
    end if
    call liberi_fock_build(handle, density, fock, n)
  end subroutine

  subroutine liberi_finalize()
    if (is_initialized) then
      call liberi_cleanup(handle)
      call liberi_destroy(handle)
      is_initialized = .false.
    end if
  end subroutine

end module gamess_liberi_wrapper
