! Fortran 2003 shim over the C ABI of include/ommgpu.h.
!
! It provides the names an existing libOMM / MatrixSwitch / pspBLAS caller
! uses -- type(matrix), m_allocate, m_deallocate, m_register_sden,
! m_register_pcsc, mm_multiply, m_add, m_trace, mm_trace, m_scale, m_set,
! m_set_element, m_get_element, psp_gemspm, psp_gespmm, omm and omm_callback -- so that
! such a caller relinks against libommgpu.so instead of the reference
! libraries.  Non-zero status codes of the C ABI are turned back into the
! reference's die() behaviour (message to MatrixSwitch.err, stop 1,
! MatrixSwitch_ops.F90:232-254).
!
! This file is not compiled by the repository's build (no Fortran compiler is
! available to it).  Compile it next to the application, e.g.
!   gfortran -c -ffree-line-length-none MatrixSwitch_gpu.F90
! and link the objects with -L<lib dir> -lommgpu.
module MatrixSwitch
  use iso_c_binding
  implicit none
  private

  integer, parameter :: dp = selected_real_kind(15, 300)

  type, public :: matrix
    type(c_ptr) :: h = c_null_ptr
    logical :: is_initialized = .false.
    logical :: is_real = .true.
    integer :: dim1 = 0, dim2 = 0
  end type matrix

  public :: m_allocate, m_deallocate, m_register_sden, m_register_pcsc, mm_multiply, m_add, m_trace, mm_trace
  public :: m_scale, m_set, m_set_element, m_get_element, psp_gemspm, psp_gespmm, omm, omm_callback, ms_check

  ! omm_callback's H(C, HC) (omm_callback.F90:45-55)
  abstract interface
    subroutine h_routine(C, HC)
      import :: matrix
      type(matrix), intent(in) :: C
      type(matrix), intent(inout) :: HC
    end subroutine h_routine
  end interface
  procedure(h_routine), pointer, save :: user_H => null()
  integer, save :: cb_m = 0, cb_n = 0
  logical, save :: cb_real = .true.

  interface
    integer(c_int) function msw_allocate(A, d1, d2, label) bind(c, name="msw_allocate")
      import :: c_ptr, c_int, c_char
      type(c_ptr), intent(inout) :: A
      integer(c_int), value :: d1, d2
      character(kind=c_char), dimension(5), intent(in) :: label
    end function
    integer(c_int) function msw_deallocate(A) bind(c, name="msw_deallocate")
      import :: c_ptr, c_int
      type(c_ptr), intent(inout) :: A
    end function
    integer(c_int) function msw_register_sden(A, d1, d2, host, is_complex) bind(c, name="msw_register_sden")
      import :: c_ptr, c_int
      type(c_ptr), intent(inout) :: A
      integer(c_int), value :: d1, d2, is_complex
      type(c_ptr), value :: host
    end function
    integer(c_int) function msw_register_csc(A, label, d1, d2, nnz, colptr, rowind, val, base) &
        bind(c, name="msw_register_csc")
      import :: c_ptr, c_int, c_char
      type(c_ptr), intent(inout) :: A
      character(kind=c_char), dimension(5), intent(in) :: label
      integer(c_int), value :: d1, d2, nnz, base
      type(c_ptr), value :: colptr, rowind, val
    end function
    integer(c_int) function msw_mm_dmultiply(A, opA, B, opB, C, alpha, beta, label) bind(c, name="msw_mm_dmultiply")
      import :: c_ptr, c_int, c_char, c_double
      type(c_ptr), value :: A, B, C
      character(kind=c_char), value :: opA, opB
      real(c_double), value :: alpha, beta
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function msw_m_dadd(A, opA, C, alpha, beta, label) bind(c, name="msw_m_dadd")
      import :: c_ptr, c_int, c_char, c_double
      type(c_ptr), value :: A, C
      character(kind=c_char), value :: opA
      real(c_double), value :: alpha, beta
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function msw_m_dtrace(A, alpha, label) bind(c, name="msw_m_dtrace")
      import :: c_ptr, c_int, c_char, c_double
      type(c_ptr), value :: A
      real(c_double), intent(out) :: alpha
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function msw_mm_dtrace(A, B, alpha, label) bind(c, name="msw_mm_dtrace")
      import :: c_ptr, c_int, c_char, c_double
      type(c_ptr), value :: A, B
      real(c_double), intent(out) :: alpha
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function msw_m_dscale(C, beta, label) bind(c, name="msw_m_dscale")
      import :: c_ptr, c_int, c_char, c_double
      type(c_ptr), value :: C
      real(c_double), value :: beta
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function msw_m_dset(C, seC, alpha, beta, label) bind(c, name="msw_m_dset")
      import :: c_ptr, c_int, c_char, c_double
      type(c_ptr), value :: C
      character(kind=c_char), value :: seC
      real(c_double), value :: alpha, beta
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function msw_m_dset_element(C, i, j, alpha, beta, label) bind(c, name="msw_m_dset_element")
      import :: c_ptr, c_int, c_char, c_double
      type(c_ptr), value :: C
      integer(c_int), value :: i, j
      real(c_double), value :: alpha, beta
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function msw_m_dget_element(C, i, j, alpha, label) bind(c, name="msw_m_dget_element")
      import :: c_ptr, c_int, c_char, c_double
      type(c_ptr), value :: C
      integer(c_int), value :: i, j
      real(c_double), intent(out) :: alpha
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function psp_gpu_dgemspm(M, N, K, A, opA, B, opB, C, alpha, beta) bind(c, name="psp_gpu_dgemspm")
      import :: c_ptr, c_int, c_char, c_double
      integer(c_int), value :: M, N, K
      type(c_ptr), value :: A, B, C
      character(kind=c_char), value :: opA, opB
      real(c_double), value :: alpha, beta
    end function
    integer(c_int) function psp_gpu_dgespmm(M, N, K, A, opA, B, opB, C, alpha, beta) bind(c, name="psp_gpu_dgespmm")
      import :: c_ptr, c_int, c_char, c_double
      integer(c_int), value :: M, N, K
      type(c_ptr), value :: A, B, C
      character(kind=c_char), value :: opA, opB
      real(c_double), value :: alpha, beta
    end function
    integer(c_int) function omm_gpu(m, n, H, S, new_S, e_min, D_min, calc_ED, eta, C_min, init_C, T, scale_T, &
        flavour, np, ip, cg_tol, long_out, dealloc, m_storage, m_operation) bind(c, name="omm_gpu")
      import :: c_ptr, c_int, c_char, c_double, c_bool
      integer(c_int), value :: m, n, flavour, np, ip
      type(c_ptr), value :: H, S, D_min, C_min, T
      logical(c_bool), value :: new_S, calc_ED, init_C, long_out, dealloc
      real(c_double), intent(out) :: e_min
      real(c_double), value :: eta, scale_T, cg_tol
      character(kind=c_char), dimension(5), intent(in) :: m_storage
      character(kind=c_char), dimension(3), intent(in) :: m_operation
    end function
    integer(c_int) function omm_gpu_callback(m, n, H, user, S, new_S, e_min, D_min, calc_ED, eta, C_min, init_C, &
        T, scale_T, flavour, np, ip, cg_tol, long_out, dealloc, m_storage, m_operation) bind(c, name="omm_gpu_callback")
      import :: c_ptr, c_funptr, c_int, c_char, c_double, c_bool
      integer(c_int), value :: m, n, flavour, np, ip
      type(c_funptr), value :: H
      type(c_ptr), value :: user, S, D_min, C_min, T
      logical(c_bool), value :: new_S, calc_ED, init_C, long_out, dealloc
      real(c_double), intent(out) :: e_min
      real(c_double), value :: eta, scale_T, cg_tol
      character(kind=c_char), dimension(5), intent(in) :: m_storage
      character(kind=c_char), dimension(3), intent(in) :: m_operation
    end function
    type(c_ptr) function omm_gpu_last_error() bind(c, name="omm_gpu_last_error")
      import :: c_ptr
    end function
  end interface

contains

  ! status -> the reference's die(): message to MatrixSwitch.err, stop 1
  subroutine ms_check(rc, where)
    integer(c_int), intent(in) :: rc
    character(*), intent(in) :: where
    character(kind=c_char), pointer :: msg(:)
    integer :: u, k
    if (rc >= 0) return
    call c_f_pointer(omm_gpu_last_error(), msg, [1024])
    open(newunit=u, file='MatrixSwitch.err', status='replace')
    write(u, '(a)') 'FATAL ERROR in matrix_switch!'
    write(u, '(a)', advance='no') where//': '
    do k = 1, 1024
      if (msg(k) == c_null_char) exit
      write(u, '(a)', advance='no') msg(k)
    end do
    write(u, '(a)') ''
    close(u)
    stop 1
  end subroutine ms_check

  function c5(s) result(c)
    character(*), intent(in) :: s
    character(kind=c_char), dimension(5) :: c
    integer :: k
    do k = 1, 5
      c(k) = s(k:k)
    end do
  end function c5

  function c3(s) result(c)
    character(*), intent(in), optional :: s
    character(kind=c_char), dimension(3) :: c
    integer :: k
    if (present(s)) then
      do k = 1, 3
        c(k) = s(k:k)
      end do
    else
      c = ['g', 'p', 'u']
    end if
  end function c3

  subroutine m_allocate(m_name, i, j, label)
    type(matrix), intent(inout) :: m_name
    integer, intent(in) :: i, j
    character(5), intent(in), optional :: label
    character(5) :: lab
    lab = 'gdden'
    if (present(label)) lab = label
    call ms_check(msw_allocate(m_name%h, int(i, c_int), int(j, c_int), c5(lab)), 'm_allocate')
    m_name%is_initialized = .true.
    m_name%is_real = (lab(2:2) == 'd')
    m_name%dim1 = i
    m_name%dim2 = j
  end subroutine m_allocate

  subroutine m_deallocate(m_name)
    type(matrix), intent(inout) :: m_name
    call ms_check(msw_deallocate(m_name%h), 'm_deallocate')
    m_name%is_initialized = .false.
  end subroutine m_deallocate

  subroutine m_register_sden(m_name, A)
    type(matrix), intent(inout) :: m_name
    real(dp), intent(inout), target :: A(:, :)
    call ms_check(msw_register_sden(m_name%h, int(size(A, 1), c_int), int(size(A, 2), c_int), c_loc(A), 0_c_int), &
                  'm_register_sden')
    m_name%is_initialized = .true.
    m_name%dim1 = size(A, 1)
    m_name%dim2 = size(A, 2)
  end subroutine m_register_sden

  ! CSC with Fortran 1-based col_ptr / row_ind (pspBLAS convention); desc(3:4) are the global sizes
  subroutine m_register_pcsc(m_name, idx1, idx2, val, desc)
    type(matrix), intent(inout) :: m_name
    integer, intent(in), target :: idx1(:), idx2(:)
    real(dp), intent(in), target :: val(:)
    integer, intent(in) :: desc(9)
    call ms_check(msw_register_csc(m_name%h, c5('gdcsc'), int(desc(3), c_int), int(desc(4), c_int), &
                                   int(size(val), c_int), c_loc(idx2), c_loc(idx1), c_loc(val), 1_c_int), &
                  'm_register_pcsc')
    m_name%is_initialized = .true.
    m_name%dim1 = desc(3)
    m_name%dim2 = desc(4)
  end subroutine m_register_pcsc

  subroutine mm_multiply(A, opA, B, opB, C, alpha, beta, label)
    type(matrix), intent(in) :: A, B
    type(matrix), intent(inout) :: C
    character(1), intent(in) :: opA, opB
    real(dp), intent(in) :: alpha, beta
    character(3), intent(in), optional :: label
    call ms_check(msw_mm_dmultiply(A%h, opA, B%h, opB, C%h, alpha, beta, c3(label)), 'mm_multiply')
  end subroutine mm_multiply

  subroutine m_add(A, opA, C, alpha, beta, label)
    type(matrix), intent(in) :: A
    type(matrix), intent(inout) :: C
    character(1), intent(in) :: opA
    real(dp), intent(in) :: alpha, beta
    character(3), intent(in), optional :: label
    call ms_check(msw_m_dadd(A%h, opA, C%h, alpha, beta, c3(label)), 'm_add')
  end subroutine m_add

  subroutine m_trace(A, alpha, label)
    type(matrix), intent(in) :: A
    real(dp), intent(out) :: alpha
    character(3), intent(in), optional :: label
    call ms_check(msw_m_dtrace(A%h, alpha, c3(label)), 'm_trace')
  end subroutine m_trace

  subroutine mm_trace(A, B, alpha, label)
    type(matrix), intent(in) :: A, B
    real(dp), intent(out) :: alpha
    character(3), intent(in), optional :: label
    call ms_check(msw_mm_dtrace(A%h, B%h, alpha, c3(label)), 'mm_trace')
  end subroutine mm_trace

  subroutine m_scale(C, beta, label)
    type(matrix), intent(inout) :: C
    real(dp), intent(in) :: beta
    character(3), intent(in), optional :: label
    call ms_check(msw_m_dscale(C%h, beta, c3(label)), 'm_scale')
  end subroutine m_scale

  subroutine m_set(C, seC, alpha, beta, label)
    type(matrix), intent(inout) :: C
    character(1), intent(in) :: seC
    real(dp), intent(in) :: alpha, beta
    character(3), intent(in), optional :: label
    call ms_check(msw_m_dset(C%h, seC, alpha, beta, c3(label)), 'm_set')
  end subroutine m_set

  subroutine m_set_element(C, i, j, alpha, beta, label)
    type(matrix), intent(inout) :: C
    integer, intent(in) :: i, j
    real(dp), intent(in) :: alpha, beta
    character(3), intent(in), optional :: label
    call ms_check(msw_m_dset_element(C%h, int(i, c_int), int(j, c_int), alpha, beta, c3(label)), 'm_set_element')
  end subroutine m_set_element

  subroutine m_get_element(C, i, j, alpha, label)
    type(matrix), intent(in) :: C
    integer, intent(in) :: i, j
    real(dp), intent(out) :: alpha
    character(3), intent(in), optional :: label
    call ms_check(msw_m_dget_element(C%h, int(i, c_int), int(j, c_int), alpha, c3(label)), 'm_get_element')
  end subroutine m_get_element

  subroutine psp_gemspm(M, N, K, A, opA, B, opB, C, alpha, beta)
    integer, intent(in) :: M, N, K
    type(matrix), intent(in) :: A, B
    type(matrix), intent(inout) :: C
    character(1), intent(in) :: opA, opB
    real(dp), intent(in) :: alpha, beta
    call ms_check(psp_gpu_dgemspm(int(M, c_int), int(N, c_int), int(K, c_int), A%h, opA, B%h, opB, C%h, alpha, &
                                  beta), 'psp_gemspm')
  end subroutine psp_gemspm

  subroutine psp_gespmm(M, N, K, A, opA, B, opB, C, alpha, beta)
    integer, intent(in) :: M, N, K
    type(matrix), intent(in) :: A, B
    type(matrix), intent(inout) :: C
    character(1), intent(in) :: opA, opB
    real(dp), intent(in) :: alpha, beta
    call ms_check(psp_gpu_dgespmm(int(M, c_int), int(N, c_int), int(K, c_int), A%h, opA, B%h, opB, C%h, alpha, &
                                  beta), 'psp_gespmm')
  end subroutine psp_gespmm

  ! omm (libOMM/src/omm.F90:5-51), same arguments; an unallocated S or T is passed as NULL
  subroutine omm(m, n, H, S, new_S, e_min, D_min, calc_ED, eta, C_min, init_C, T, scale_T, flavour, np, ip, &
                 cg_tol, long_out, dealloc, m_storage, m_operation)
    integer, intent(in) :: m, n, flavour, np, ip
    type(matrix), intent(inout) :: H, S, D_min, C_min, T
    logical, intent(in) :: new_S, calc_ED, init_C, long_out, dealloc
    real(dp), intent(out) :: e_min
    real(dp), intent(in) :: eta, scale_T, cg_tol
    character(5), intent(in) :: m_storage
    character(3), intent(in) :: m_operation
    type(c_ptr) :: Sp, Tp
    integer(c_int) :: rc
    Sp = c_null_ptr
    Tp = c_null_ptr
    if (S%is_initialized) Sp = S%h
    if (T%is_initialized) Tp = T%h
    rc = omm_gpu(int(m, c_int), int(n, c_int), H%h, Sp, logical(new_S, c_bool), e_min, D_min%h, &
                 logical(calc_ED, c_bool), eta, C_min%h, logical(init_C, c_bool), Tp, scale_T, int(flavour, c_int), &
                 int(np, c_int), int(ip, c_int), cg_tol, logical(long_out, c_bool), logical(dealloc, c_bool), &
                 c5(m_storage), c3(m_operation))
    call ms_check(rc, 'omm')
  end subroutine omm

  ! the C routine omm_gpu_callback calls: wraps the lent handles into type(matrix) for the
  ! caller's H (they alias library buffers and are not deallocated here)
  integer(c_int) function h_trampoline(C, HC, user) bind(c)
    type(c_ptr), value :: C, HC, user
    type(matrix) :: Cm, HCm
    Cm%h = C
    Cm%is_initialized = .true.
    Cm%is_real = cb_real
    Cm%dim1 = cb_n
    Cm%dim2 = cb_m
    HCm = Cm
    HCm%h = HC
    call user_H(Cm, HCm)
    h_trampoline = 0
  end function h_trampoline

  subroutine omm_callback(m, n, H, S, new_S, e_min, D_min, calc_ED, eta, C_min, init_C, T, scale_T, flavour, np, &
                          ip, cg_tol, long_out, dealloc, m_storage, m_operation)
    integer, intent(in) :: m, n, flavour, np, ip
    procedure(h_routine) :: H
    type(matrix), intent(inout) :: S, D_min, C_min, T
    logical, intent(in) :: new_S, calc_ED, init_C, long_out, dealloc
    real(dp), intent(out) :: e_min
    real(dp), intent(in) :: eta, scale_T, cg_tol
    character(5), intent(in) :: m_storage
    character(3), intent(in) :: m_operation
    type(c_ptr) :: Sp, Tp
    integer(c_int) :: rc
    Sp = c_null_ptr
    Tp = c_null_ptr
    if (S%is_initialized) Sp = S%h
    if (T%is_initialized) Tp = T%h
    user_H => H
    cb_m = m
    cb_n = n
    cb_real = C_min%is_real
    rc = omm_gpu_callback(int(m, c_int), int(n, c_int), c_funloc(h_trampoline), c_null_ptr, Sp, &
                          logical(new_S, c_bool), e_min, D_min%h, logical(calc_ED, c_bool), eta, C_min%h, &
                          logical(init_C, c_bool), Tp, scale_T, int(flavour, c_int), int(np, c_int), int(ip, c_int), &
                          cg_tol, logical(long_out, c_bool), logical(dealloc, c_bool), c5(m_storage), c3(m_operation))
    user_H => null()
    call ms_check(rc, 'omm_callback')
  end subroutine omm_callback

end module MatrixSwitch
