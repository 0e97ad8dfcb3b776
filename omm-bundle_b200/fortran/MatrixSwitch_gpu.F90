! Fortran 2003 shim over the C ABI of include/ommgpu.h.
!
! It provides the names an existing libOMM / MatrixSwitch / pspBLAS caller
! uses -- type(matrix), m_allocate, m_deallocate, m_register_sden,
! m_register_pcsc, mm_multiply, m_add, m_trace, mm_trace, m_scale, m_set,
! m_set_element, m_get_element (each generic over real and complex, like
! MatrixSwitch.F90:69-70,105-106,124-125,148-149,167-168,197-198,225-226,247-248),
! psp_gemspm, psp_gespmm (pspMspm.F90:58-183, pspSpmm.F90:58-190), omm and
! omm_callback -- and, in module MatrixSwitch_wrapper, the string-key layer
! (ms_wrapper_open, ms_lookup-based routines, omm_wrapper) -- so that such a
! caller relinks against libommgpu.so instead of the reference libraries.
! Defaults are the reference's: m_allocate without a label makes 'sdden'
! (MatrixSwitch.F90:344-347) and an operation without a label is 'ref'.
! Non-zero status codes of the C ABI are turned back into the
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
  public :: c3, ckey

  interface mm_multiply
    module procedure mm_dmultiply, mm_zmultiply
  end interface mm_multiply
  interface m_add
    module procedure m_dadd, m_zadd
  end interface m_add
  interface m_trace
    module procedure m_dtrace, m_ztrace
  end interface m_trace
  interface mm_trace
    module procedure mm_dtrace, mm_ztrace
  end interface mm_trace
  interface m_scale
    module procedure m_dscale, m_zscale
  end interface m_scale
  interface m_set
    module procedure m_dset, m_zset
  end interface m_set
  interface m_set_element
    module procedure m_dset_element, m_zset_element
  end interface m_set_element
  interface m_get_element
    module procedure m_dget_element, m_zget_element
  end interface m_get_element
  interface m_register_sden
    module procedure m_register_sdden, m_register_szden
  end interface m_register_sden
  interface m_register_pcsc
    module procedure m_register_pdcsc, m_register_pzcsc
  end interface m_register_pcsc
  interface psp_gemspm
    module procedure psp_dgemspm, psp_zgemspm
  end interface psp_gemspm
  interface psp_gespmm
    module procedure psp_dgespmm, psp_zgespmm
  end interface psp_gespmm

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
    integer(c_int) function msw_mm_zmultiply(A, opA, B, opB, C, alpha, beta, label) bind(c, name="msw_mm_zmultiply")
      import :: c_ptr, c_int, c_char, c_double_complex
      type(c_ptr), value :: A, B, C
      character(kind=c_char), value :: opA, opB
      complex(c_double_complex), intent(in) :: alpha, beta
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function msw_m_zadd(A, opA, C, alpha, beta, label) bind(c, name="msw_m_zadd")
      import :: c_ptr, c_int, c_char, c_double_complex
      type(c_ptr), value :: A, C
      character(kind=c_char), value :: opA
      complex(c_double_complex), intent(in) :: alpha, beta
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function msw_m_ztrace(A, alpha, label) bind(c, name="msw_m_ztrace")
      import :: c_ptr, c_int, c_char, c_double_complex
      type(c_ptr), value :: A
      complex(c_double_complex), intent(out) :: alpha
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function msw_mm_ztrace(A, B, alpha, label) bind(c, name="msw_mm_ztrace")
      import :: c_ptr, c_int, c_char, c_double_complex
      type(c_ptr), value :: A, B
      complex(c_double_complex), intent(out) :: alpha
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function msw_m_zscale(C, beta, label) bind(c, name="msw_m_zscale")
      import :: c_ptr, c_int, c_char, c_double_complex
      type(c_ptr), value :: C
      complex(c_double_complex), intent(in) :: beta
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function msw_m_zset(C, seC, alpha, beta, label) bind(c, name="msw_m_zset")
      import :: c_ptr, c_int, c_char, c_double_complex
      type(c_ptr), value :: C
      character(kind=c_char), value :: seC
      complex(c_double_complex), intent(in) :: alpha, beta
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function msw_m_zset_element(C, i, j, alpha, beta, label) bind(c, name="msw_m_zset_element")
      import :: c_ptr, c_int, c_char, c_double_complex
      type(c_ptr), value :: C
      integer(c_int), value :: i, j
      complex(c_double_complex), intent(in) :: alpha, beta
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function msw_m_zget_element(C, i, j, alpha, label) bind(c, name="msw_m_zget_element")
      import :: c_ptr, c_int, c_char, c_double_complex
      type(c_ptr), value :: C
      integer(c_int), value :: i, j
      complex(c_double_complex), intent(out) :: alpha
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function psp_gpu_zgemspm(M, N, K, A, opA, B, opB, C, alpha, beta) bind(c, name="psp_gpu_zgemspm")
      import :: c_ptr, c_int, c_char, c_double_complex
      integer(c_int), value :: M, N, K
      type(c_ptr), value :: A, B, C
      character(kind=c_char), value :: opA, opB
      complex(c_double_complex), intent(in) :: alpha, beta
    end function
    integer(c_int) function psp_gpu_zgespmm(M, N, K, A, opA, B, opB, C, alpha, beta) bind(c, name="psp_gpu_zgespmm")
      import :: c_ptr, c_int, c_char, c_double_complex
      integer(c_int), value :: M, N, K
      type(c_ptr), value :: A, B, C
      character(kind=c_char), value :: opA, opB
      complex(c_double_complex), intent(in) :: alpha, beta
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
      c = ['r', 'e', 'f']  ! the reference's implementation when no label is given
    end if
  end function c3

  ! a NUL-terminated copy of a key (trailing blanks dropped) for the C string-key layer
  function ckey(s) result(c)
    character(*), intent(in) :: s
    character(kind=c_char, len=len_trim(s) + 1) :: c
    c = trim(s)//c_null_char
  end function ckey

  subroutine m_allocate(m_name, i, j, label)
    type(matrix), intent(inout) :: m_name
    integer, intent(in) :: i, j
    character(5), intent(in), optional :: label
    character(5) :: lab
    lab = 'sdden'  ! MatrixSwitch.F90:344-347
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

  subroutine m_register_sdden(m_name, A)
    type(matrix), intent(inout) :: m_name
    real(dp), intent(inout), target :: A(:, :)
    call ms_check(msw_register_sden(m_name%h, int(size(A, 1), c_int), int(size(A, 2), c_int), c_loc(A), 0_c_int), &
                  'm_register_sden')
    m_name%is_initialized = .true.
    m_name%dim1 = size(A, 1)
    m_name%dim2 = size(A, 2)
  end subroutine m_register_sdden

  ! CSC with Fortran 1-based col_ptr / row_ind (pspBLAS convention); desc(3:4) are the global sizes
  subroutine m_register_pdcsc(m_name, idx1, idx2, val, desc)
    type(matrix), intent(inout) :: m_name
    integer, intent(in), target :: idx1(:), idx2(:)
    real(dp), intent(in), target :: val(:)
    integer, intent(in) :: desc(9)
    call ms_check(msw_register_csc(m_name%h, c5('pdcsc'), int(desc(3), c_int), int(desc(4), c_int), &
                                   int(size(val), c_int), c_loc(idx2), c_loc(idx1), c_loc(val), 1_c_int), &
                  'm_register_pcsc')
    m_name%is_initialized = .true.
    m_name%dim1 = desc(3)
    m_name%dim2 = desc(4)
  end subroutine m_register_pdcsc

  subroutine mm_dmultiply(A, opA, B, opB, C, alpha, beta, label)
    type(matrix), intent(in) :: A, B
    type(matrix), intent(inout) :: C
    character(1), intent(in) :: opA, opB
    real(dp), intent(in) :: alpha, beta
    character(3), intent(in), optional :: label
    call ms_check(msw_mm_dmultiply(A%h, opA, B%h, opB, C%h, alpha, beta, c3(label)), 'mm_multiply')
  end subroutine mm_dmultiply

  subroutine m_dadd(A, opA, C, alpha, beta, label)
    type(matrix), intent(in) :: A
    type(matrix), intent(inout) :: C
    character(1), intent(in) :: opA
    real(dp), intent(in) :: alpha, beta
    character(3), intent(in), optional :: label
    call ms_check(msw_m_dadd(A%h, opA, C%h, alpha, beta, c3(label)), 'm_add')
  end subroutine m_dadd

  subroutine m_dtrace(A, alpha, label)
    type(matrix), intent(in) :: A
    real(dp), intent(out) :: alpha
    character(3), intent(in), optional :: label
    call ms_check(msw_m_dtrace(A%h, alpha, c3(label)), 'm_trace')
  end subroutine m_dtrace

  subroutine mm_dtrace(A, B, alpha, label)
    type(matrix), intent(in) :: A, B
    real(dp), intent(out) :: alpha
    character(3), intent(in), optional :: label
    call ms_check(msw_mm_dtrace(A%h, B%h, alpha, c3(label)), 'mm_trace')
  end subroutine mm_dtrace

  subroutine m_dscale(C, beta, label)
    type(matrix), intent(inout) :: C
    real(dp), intent(in) :: beta
    character(3), intent(in), optional :: label
    call ms_check(msw_m_dscale(C%h, beta, c3(label)), 'm_scale')
  end subroutine m_dscale

  subroutine m_dset(C, seC, alpha, beta, label)
    type(matrix), intent(inout) :: C
    character(1), intent(in) :: seC
    real(dp), intent(in) :: alpha, beta
    character(3), intent(in), optional :: label
    call ms_check(msw_m_dset(C%h, seC, alpha, beta, c3(label)), 'm_set')
  end subroutine m_dset

  subroutine m_dset_element(C, i, j, alpha, beta, label)
    type(matrix), intent(inout) :: C
    integer, intent(in) :: i, j
    real(dp), intent(in) :: alpha, beta
    character(3), intent(in), optional :: label
    call ms_check(msw_m_dset_element(C%h, int(i, c_int), int(j, c_int), alpha, beta, c3(label)), 'm_set_element')
  end subroutine m_dset_element

  subroutine m_dget_element(C, i, j, alpha, label)
    type(matrix), intent(in) :: C
    integer, intent(in) :: i, j
    real(dp), intent(out) :: alpha
    character(3), intent(in), optional :: label
    call ms_check(msw_m_dget_element(C%h, int(i, c_int), int(j, c_int), alpha, c3(label)), 'm_get_element')
  end subroutine m_dget_element

  subroutine psp_dgemspm(M, N, K, A, opA, B, opB, C, alpha, beta)
    integer, intent(in) :: M, N, K
    type(matrix), intent(in) :: A, B
    type(matrix), intent(inout) :: C
    character(1), intent(in) :: opA, opB
    real(dp), intent(in) :: alpha, beta
    call ms_check(psp_gpu_dgemspm(int(M, c_int), int(N, c_int), int(K, c_int), A%h, opA, B%h, opB, C%h, alpha, &
                                  beta), 'psp_gemspm')
  end subroutine psp_dgemspm

  subroutine psp_dgespmm(M, N, K, A, opA, B, opB, C, alpha, beta)
    integer, intent(in) :: M, N, K
    type(matrix), intent(in) :: A, B
    type(matrix), intent(inout) :: C
    character(1), intent(in) :: opA, opB
    real(dp), intent(in) :: alpha, beta
    call ms_check(psp_gpu_dgespmm(int(M, c_int), int(N, c_int), int(K, c_int), A%h, opA, B%h, opB, C%h, alpha, &
                                  beta), 'psp_gespmm')
  end subroutine psp_dgespmm

  subroutine m_register_szden(m_name, A)
    type(matrix), intent(inout) :: m_name
    complex(dp), intent(inout), target :: A(:, :)
    call ms_check(msw_register_sden(m_name%h, int(size(A, 1), c_int), int(size(A, 2), c_int), c_loc(A), 1_c_int), &
                  'm_register_sden')
    m_name%is_initialized = .true.
    m_name%is_real = .false.
    m_name%dim1 = size(A, 1)
    m_name%dim2 = size(A, 2)
  end subroutine m_register_szden

  subroutine m_register_pzcsc(m_name, idx1, idx2, val, desc)
    type(matrix), intent(inout) :: m_name
    integer, intent(in), target :: idx1(:), idx2(:)
    complex(dp), intent(in), target :: val(:)
    integer, intent(in) :: desc(9)
    call ms_check(msw_register_csc(m_name%h, c5('pzcsc'), int(desc(3), c_int), int(desc(4), c_int), &
                                   int(size(val), c_int), c_loc(idx2), c_loc(idx1), c_loc(val), 1_c_int), &
                  'm_register_pcsc')
    m_name%is_initialized = .true.
    m_name%is_real = .false.
    m_name%dim1 = desc(3)
    m_name%dim2 = desc(4)
  end subroutine m_register_pzcsc

  subroutine mm_zmultiply(A, opA, B, opB, C, alpha, beta, label)
    type(matrix), intent(in) :: A, B
    type(matrix), intent(inout) :: C
    character(1), intent(in) :: opA, opB
    complex(dp), intent(in) :: alpha, beta
    character(3), intent(in), optional :: label
    call ms_check(msw_mm_zmultiply(A%h, opA, B%h, opB, C%h, alpha, beta, c3(label)), 'mm_multiply')
  end subroutine mm_zmultiply

  subroutine m_zadd(A, opA, C, alpha, beta, label)
    type(matrix), intent(in) :: A
    type(matrix), intent(inout) :: C
    character(1), intent(in) :: opA
    complex(dp), intent(in) :: alpha, beta
    character(3), intent(in), optional :: label
    call ms_check(msw_m_zadd(A%h, opA, C%h, alpha, beta, c3(label)), 'm_add')
  end subroutine m_zadd

  subroutine m_ztrace(A, alpha, label)
    type(matrix), intent(in) :: A
    complex(dp), intent(out) :: alpha
    character(3), intent(in), optional :: label
    call ms_check(msw_m_ztrace(A%h, alpha, c3(label)), 'm_trace')
  end subroutine m_ztrace

  subroutine mm_ztrace(A, B, alpha, label)
    type(matrix), intent(in) :: A, B
    complex(dp), intent(out) :: alpha
    character(3), intent(in), optional :: label
    call ms_check(msw_mm_ztrace(A%h, B%h, alpha, c3(label)), 'mm_trace')
  end subroutine mm_ztrace

  subroutine m_zscale(C, beta, label)
    type(matrix), intent(inout) :: C
    complex(dp), intent(in) :: beta
    character(3), intent(in), optional :: label
    call ms_check(msw_m_zscale(C%h, beta, c3(label)), 'm_scale')
  end subroutine m_zscale

  subroutine m_zset(C, seC, alpha, beta, label)
    type(matrix), intent(inout) :: C
    character(1), intent(in) :: seC
    complex(dp), intent(in) :: alpha, beta
    character(3), intent(in), optional :: label
    call ms_check(msw_m_zset(C%h, seC, alpha, beta, c3(label)), 'm_set')
  end subroutine m_zset

  subroutine m_zset_element(C, i, j, alpha, beta, label)
    type(matrix), intent(inout) :: C
    integer, intent(in) :: i, j
    complex(dp), intent(in) :: alpha, beta
    character(3), intent(in), optional :: label
    call ms_check(msw_m_zset_element(C%h, int(i, c_int), int(j, c_int), alpha, beta, c3(label)), 'm_set_element')
  end subroutine m_zset_element

  subroutine m_zget_element(C, i, j, alpha, label)
    type(matrix), intent(in) :: C
    integer, intent(in) :: i, j
    complex(dp), intent(out) :: alpha
    character(3), intent(in), optional :: label
    call ms_check(msw_m_zget_element(C%h, int(i, c_int), int(j, c_int), alpha, c3(label)), 'm_get_element')
  end subroutine m_zget_element

  subroutine psp_zgemspm(M, N, K, A, opA, B, opB, C, alpha, beta)
    integer, intent(in) :: M, N, K
    type(matrix), intent(in) :: A, B
    type(matrix), intent(inout) :: C
    character(1), intent(in) :: opA, opB
    complex(dp), intent(in) :: alpha, beta
    call ms_check(psp_gpu_zgemspm(int(M, c_int), int(N, c_int), int(K, c_int), A%h, opA, B%h, opB, C%h, alpha, &
                                  beta), 'psp_gemspm')
  end subroutine psp_zgemspm

  subroutine psp_zgespmm(M, N, K, A, opA, B, opB, C, alpha, beta)
    integer, intent(in) :: M, N, K
    type(matrix), intent(in) :: A, B
    type(matrix), intent(inout) :: C
    character(1), intent(in) :: opA, opB
    complex(dp), intent(in) :: alpha, beta
    call ms_check(psp_gpu_zgespmm(int(M, c_int), int(N, c_int), int(K, c_int), A%h, opA, B%h, opB, C%h, alpha, &
                                  beta), 'psp_gespmm')
  end subroutine psp_zgespmm

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

! The string-key layer (MatrixSwitch/src/MatrixSwitch_wrapper.F90, MatrixSwitch_wrapper_params.F90):
! matrices named by keys of at most 10 characters, held by the C library's key table.
module MatrixSwitch_wrapper
  use iso_c_binding
  use MatrixSwitch, only: ms_check, c3, ckey
  implicit none
  private

  integer, parameter :: dp = selected_real_kind(15, 300)

  public :: ms_wrapper_open, ms_wrapper_close, m_allocate, m_deallocate, mm_multiply, m_add, m_trace, mm_trace
  public :: m_scale, m_set, m_set_element, m_get_element, m_register_sden, m_register_pcsc, omm_wrapper

  interface mm_multiply
    module procedure mm_dmultiply, mm_zmultiply
  end interface mm_multiply
  interface m_add
    module procedure m_dadd, m_zadd
  end interface m_add
  interface m_trace
    module procedure m_dtrace, m_ztrace
  end interface m_trace
  interface mm_trace
    module procedure mm_dtrace, mm_ztrace
  end interface mm_trace
  interface m_scale
    module procedure m_dscale, m_zscale
  end interface m_scale
  interface m_set
    module procedure m_dset, m_zset
  end interface m_set
  interface m_set_element
    module procedure m_dset_element, m_zset_element
  end interface m_set_element
  interface m_get_element
    module procedure m_dget_element, m_zget_element
  end interface m_get_element
  interface m_register_sden
    module procedure m_register_sdden, m_register_szden
  end interface m_register_sden
  interface m_register_pcsc
    module procedure m_register_pdcsc, m_register_pzcsc
  end interface m_register_pcsc

  interface
    integer(c_int) function c_ms_wrapper_open(num, keys) bind(c, name="ms_wrapper_open")
      import :: c_int, c_ptr
      integer(c_int), value :: num
      type(c_ptr), dimension(*), intent(in) :: keys
    end function
    integer(c_int) function c_ms_wrapper_close() bind(c, name="ms_wrapper_close")
      import :: c_int
    end function
    integer(c_int) function c_ms_m_allocate(key, i, j, label) bind(c, name="ms_m_allocate")
      import :: c_int, c_char
      character(kind=c_char), dimension(*), intent(in) :: key
      integer(c_int), value :: i, j
      character(kind=c_char), dimension(5), intent(in) :: label
    end function
    integer(c_int) function c_ms_m_deallocate(key) bind(c, name="ms_m_deallocate")
      import :: c_int, c_char
      character(kind=c_char), dimension(*), intent(in) :: key
    end function
    integer(c_int) function c_ms_mm_dmultiply(A, opA, B, opB, C, alpha, beta, label) bind(c, name="ms_mm_dmultiply")
      import :: c_int, c_char, c_double
      character(kind=c_char), dimension(*), intent(in) :: A, B, C
      character(kind=c_char), value :: opA, opB
      real(c_double), value :: alpha, beta
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function c_ms_mm_zmultiply(A, opA, B, opB, C, alpha, beta, label) bind(c, name="ms_mm_zmultiply")
      import :: c_int, c_char, c_double_complex
      character(kind=c_char), dimension(*), intent(in) :: A, B, C
      character(kind=c_char), value :: opA, opB
      complex(c_double_complex), intent(in) :: alpha, beta
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function c_ms_m_dadd(A, opA, C, alpha, beta, label) bind(c, name="ms_m_dadd")
      import :: c_int, c_char, c_double
      character(kind=c_char), dimension(*), intent(in) :: A, C
      character(kind=c_char), value :: opA
      real(c_double), value :: alpha, beta
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function c_ms_m_zadd(A, opA, C, alpha, beta, label) bind(c, name="ms_m_zadd")
      import :: c_int, c_char, c_double_complex
      character(kind=c_char), dimension(*), intent(in) :: A, C
      character(kind=c_char), value :: opA
      complex(c_double_complex), intent(in) :: alpha, beta
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function c_ms_m_dtrace(A, alpha, label) bind(c, name="ms_m_dtrace")
      import :: c_int, c_char, c_double
      character(kind=c_char), dimension(*), intent(in) :: A
      real(c_double), intent(out) :: alpha
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function c_ms_m_ztrace(A, alpha, label) bind(c, name="ms_m_ztrace")
      import :: c_int, c_char, c_double_complex
      character(kind=c_char), dimension(*), intent(in) :: A
      complex(c_double_complex), intent(out) :: alpha
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function c_ms_mm_dtrace(A, B, alpha, label) bind(c, name="ms_mm_dtrace")
      import :: c_int, c_char, c_double
      character(kind=c_char), dimension(*), intent(in) :: A, B
      real(c_double), intent(out) :: alpha
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function c_ms_mm_ztrace(A, B, alpha, label) bind(c, name="ms_mm_ztrace")
      import :: c_int, c_char, c_double_complex
      character(kind=c_char), dimension(*), intent(in) :: A, B
      complex(c_double_complex), intent(out) :: alpha
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function c_ms_m_dscale(C, beta, label) bind(c, name="ms_m_dscale")
      import :: c_int, c_char, c_double
      character(kind=c_char), dimension(*), intent(in) :: C
      real(c_double), value :: beta
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function c_ms_m_zscale(C, beta, label) bind(c, name="ms_m_zscale")
      import :: c_int, c_char, c_double_complex
      character(kind=c_char), dimension(*), intent(in) :: C
      complex(c_double_complex), intent(in) :: beta
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function c_ms_m_dset(C, seC, alpha, beta, label) bind(c, name="ms_m_dset")
      import :: c_int, c_char, c_double
      character(kind=c_char), dimension(*), intent(in) :: C
      character(kind=c_char), value :: seC
      real(c_double), value :: alpha, beta
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function c_ms_m_zset(C, seC, alpha, beta, label) bind(c, name="ms_m_zset")
      import :: c_int, c_char, c_double_complex
      character(kind=c_char), dimension(*), intent(in) :: C
      character(kind=c_char), value :: seC
      complex(c_double_complex), intent(in) :: alpha, beta
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function c_ms_m_dset_element(C, i, j, alpha, beta, label) bind(c, name="ms_m_dset_element")
      import :: c_int, c_char, c_double
      character(kind=c_char), dimension(*), intent(in) :: C
      integer(c_int), value :: i, j
      real(c_double), value :: alpha, beta
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function c_ms_m_zset_element(C, i, j, alpha, beta, label) bind(c, name="ms_m_zset_element")
      import :: c_int, c_char, c_double_complex
      character(kind=c_char), dimension(*), intent(in) :: C
      integer(c_int), value :: i, j
      complex(c_double_complex), intent(in) :: alpha, beta
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function c_ms_m_dget_element(C, i, j, alpha, label) bind(c, name="ms_m_dget_element")
      import :: c_int, c_char, c_double
      character(kind=c_char), dimension(*), intent(in) :: C
      integer(c_int), value :: i, j
      real(c_double), intent(out) :: alpha
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function c_ms_m_zget_element(C, i, j, alpha, label) bind(c, name="ms_m_zget_element")
      import :: c_int, c_char, c_double_complex
      character(kind=c_char), dimension(*), intent(in) :: C
      integer(c_int), value :: i, j
      complex(c_double_complex), intent(out) :: alpha
      character(kind=c_char), dimension(3), intent(in) :: label
    end function
    integer(c_int) function c_ms_m_register_sdden(key, d1, d2, A) bind(c, name="ms_m_register_sdden")
      import :: c_int, c_char, c_ptr
      character(kind=c_char), dimension(*), intent(in) :: key
      integer(c_int), value :: d1, d2
      type(c_ptr), value :: A
    end function
    integer(c_int) function c_ms_m_register_szden(key, d1, d2, A) bind(c, name="ms_m_register_szden")
      import :: c_int, c_char, c_ptr
      character(kind=c_char), dimension(*), intent(in) :: key
      integer(c_int), value :: d1, d2
      type(c_ptr), value :: A
    end function
    integer(c_int) function c_ms_m_register_pdcsc(key, idx1, idx2, val, desc) bind(c, name="ms_m_register_pdcsc")
      import :: c_int, c_char, c_ptr
      character(kind=c_char), dimension(*), intent(in) :: key
      type(c_ptr), value :: idx1, idx2, val
      integer(c_int), dimension(9), intent(in) :: desc
    end function
    integer(c_int) function c_ms_m_register_pzcsc(key, idx1, idx2, val, desc) bind(c, name="ms_m_register_pzcsc")
      import :: c_int, c_char, c_ptr
      character(kind=c_char), dimension(*), intent(in) :: key
      type(c_ptr), value :: idx1, idx2, val
      integer(c_int), dimension(9), intent(in) :: desc
    end function
    integer(c_int) function c_omm_wrapper(m, n, H, S, new_S, e_min, D_min, calc_ED, eta, C_min, init_C, T, scale_T, &
        flavour, np, ip, cg_tol, long_out, dealloc, m_storage, m_operation) bind(c, name="omm_wrapper")
      import :: c_int, c_char, c_double, c_bool
      integer(c_int), value :: m, n, flavour, np, ip
      character(kind=c_char), dimension(*), intent(in) :: H, S, D_min, C_min, T
      logical(c_bool), value :: new_S, calc_ED, init_C, long_out, dealloc
      real(c_double), intent(out) :: e_min
      real(c_double), value :: eta, scale_T, cg_tol
      character(kind=c_char), dimension(5), intent(in) :: m_storage
      character(kind=c_char), dimension(3), intent(in) :: m_operation
    end function
  end interface

contains

  ! ms_wrapper_open (MatrixSwitch_wrapper.F90:219-236): keys are passed to C as NUL-terminated copies
  subroutine ms_wrapper_open(num_matrices, keys)
    integer, intent(in) :: num_matrices
    character(*), intent(in) :: keys(num_matrices)
    character(kind=c_char, len=len(keys) + 1), allocatable, target :: buf(:)
    type(c_ptr), allocatable :: ptrs(:)
    integer :: i
    allocate(buf(num_matrices), ptrs(num_matrices))
    do i = 1, num_matrices
      buf(i) = trim(keys(i))//c_null_char
      ptrs(i) = c_loc(buf(i))
    end do
    call ms_check(c_ms_wrapper_open(int(num_matrices, c_int), ptrs), 'ms_wrapper_open')
  end subroutine ms_wrapper_open

  subroutine ms_wrapper_close()
    call ms_check(c_ms_wrapper_close(), 'ms_wrapper_close')
  end subroutine ms_wrapper_close

  subroutine m_allocate(m_name, i, j, label)
    character(*), intent(in) :: m_name
    integer, intent(in) :: i, j
    character(5), intent(in), optional :: label
    character(5) :: lab
    integer :: k
    character(kind=c_char), dimension(5) :: c
    lab = 'sdden'  ! MatrixSwitch.F90:344-347
    if (present(label)) lab = label
    do k = 1, 5
      c(k) = lab(k:k)
    end do
    call ms_check(c_ms_m_allocate(ckey(m_name), int(i, c_int), int(j, c_int), c), 'm_allocate')
  end subroutine m_allocate

  subroutine m_deallocate(m_name)
    character(*), intent(in) :: m_name
    call ms_check(c_ms_m_deallocate(ckey(m_name)), 'm_deallocate')
  end subroutine m_deallocate

  subroutine mm_dmultiply(A, opA, B, opB, C, alpha, beta, label)
    character(*), intent(in) :: A, B, C
    character(1), intent(in) :: opA, opB
    real(dp), intent(in) :: alpha, beta
    character(3), intent(in), optional :: label
    call ms_check(c_ms_mm_dmultiply(ckey(A), opA, ckey(B), opB, ckey(C), alpha, beta, c3(label)), 'mm_multiply')
  end subroutine mm_dmultiply

  subroutine mm_zmultiply(A, opA, B, opB, C, alpha, beta, label)
    character(*), intent(in) :: A, B, C
    character(1), intent(in) :: opA, opB
    complex(dp), intent(in) :: alpha, beta
    character(3), intent(in), optional :: label
    call ms_check(c_ms_mm_zmultiply(ckey(A), opA, ckey(B), opB, ckey(C), alpha, beta, c3(label)), 'mm_multiply')
  end subroutine mm_zmultiply

  subroutine m_dadd(A, opA, C, alpha, beta, label)
    character(*), intent(in) :: A, C
    character(1), intent(in) :: opA
    real(dp), intent(in) :: alpha, beta
    character(3), intent(in), optional :: label
    call ms_check(c_ms_m_dadd(ckey(A), opA, ckey(C), alpha, beta, c3(label)), 'm_add')
  end subroutine m_dadd

  subroutine m_zadd(A, opA, C, alpha, beta, label)
    character(*), intent(in) :: A, C
    character(1), intent(in) :: opA
    complex(dp), intent(in) :: alpha, beta
    character(3), intent(in), optional :: label
    call ms_check(c_ms_m_zadd(ckey(A), opA, ckey(C), alpha, beta, c3(label)), 'm_add')
  end subroutine m_zadd

  subroutine m_dtrace(A, alpha, label)
    character(*), intent(in) :: A
    real(dp), intent(out) :: alpha
    character(3), intent(in), optional :: label
    call ms_check(c_ms_m_dtrace(ckey(A), alpha, c3(label)), 'm_trace')
  end subroutine m_dtrace

  subroutine m_ztrace(A, alpha, label)
    character(*), intent(in) :: A
    complex(dp), intent(out) :: alpha
    character(3), intent(in), optional :: label
    call ms_check(c_ms_m_ztrace(ckey(A), alpha, c3(label)), 'm_trace')
  end subroutine m_ztrace

  subroutine mm_dtrace(A, B, alpha, label)
    character(*), intent(in) :: A, B
    real(dp), intent(out) :: alpha
    character(3), intent(in), optional :: label
    call ms_check(c_ms_mm_dtrace(ckey(A), ckey(B), alpha, c3(label)), 'mm_trace')
  end subroutine mm_dtrace

  subroutine mm_ztrace(A, B, alpha, label)
    character(*), intent(in) :: A, B
    complex(dp), intent(out) :: alpha
    character(3), intent(in), optional :: label
    call ms_check(c_ms_mm_ztrace(ckey(A), ckey(B), alpha, c3(label)), 'mm_trace')
  end subroutine mm_ztrace

  subroutine m_dscale(C, beta, label)
    character(*), intent(in) :: C
    real(dp), intent(in) :: beta
    character(3), intent(in), optional :: label
    call ms_check(c_ms_m_dscale(ckey(C), beta, c3(label)), 'm_scale')
  end subroutine m_dscale

  subroutine m_zscale(C, beta, label)
    character(*), intent(in) :: C
    complex(dp), intent(in) :: beta
    character(3), intent(in), optional :: label
    call ms_check(c_ms_m_zscale(ckey(C), beta, c3(label)), 'm_scale')
  end subroutine m_zscale

  subroutine m_dset(C, seC, alpha, beta, label)
    character(*), intent(in) :: C
    character(1), intent(in) :: seC
    real(dp), intent(in) :: alpha, beta
    character(3), intent(in), optional :: label
    call ms_check(c_ms_m_dset(ckey(C), seC, alpha, beta, c3(label)), 'm_set')
  end subroutine m_dset

  subroutine m_zset(C, seC, alpha, beta, label)
    character(*), intent(in) :: C
    character(1), intent(in) :: seC
    complex(dp), intent(in) :: alpha, beta
    character(3), intent(in), optional :: label
    call ms_check(c_ms_m_zset(ckey(C), seC, alpha, beta, c3(label)), 'm_set')
  end subroutine m_zset

  subroutine m_dset_element(C, i, j, alpha, beta, label)
    character(*), intent(in) :: C
    integer, intent(in) :: i, j
    real(dp), intent(in) :: alpha, beta
    character(3), intent(in), optional :: label
    call ms_check(c_ms_m_dset_element(ckey(C), int(i, c_int), int(j, c_int), alpha, beta, c3(label)), &
                  'm_set_element')
  end subroutine m_dset_element

  subroutine m_zset_element(C, i, j, alpha, beta, label)
    character(*), intent(in) :: C
    integer, intent(in) :: i, j
    complex(dp), intent(in) :: alpha, beta
    character(3), intent(in), optional :: label
    call ms_check(c_ms_m_zset_element(ckey(C), int(i, c_int), int(j, c_int), alpha, beta, c3(label)), &
                  'm_set_element')
  end subroutine m_zset_element

  subroutine m_dget_element(C, i, j, alpha, label)
    character(*), intent(in) :: C
    integer, intent(in) :: i, j
    real(dp), intent(out) :: alpha
    character(3), intent(in), optional :: label
    call ms_check(c_ms_m_dget_element(ckey(C), int(i, c_int), int(j, c_int), alpha, c3(label)), 'm_get_element')
  end subroutine m_dget_element

  subroutine m_zget_element(C, i, j, alpha, label)
    character(*), intent(in) :: C
    integer, intent(in) :: i, j
    complex(dp), intent(out) :: alpha
    character(3), intent(in), optional :: label
    call ms_check(c_ms_m_zget_element(ckey(C), int(i, c_int), int(j, c_int), alpha, c3(label)), 'm_get_element')
  end subroutine m_zget_element

  subroutine m_register_sdden(m_name, A)
    character(*), intent(in) :: m_name
    real(dp), intent(inout), target :: A(:, :)
    call ms_check(c_ms_m_register_sdden(ckey(m_name), int(size(A, 1), c_int), int(size(A, 2), c_int), c_loc(A)), &
                  'm_register_sden')
  end subroutine m_register_sdden

  subroutine m_register_szden(m_name, A)
    character(*), intent(in) :: m_name
    complex(dp), intent(inout), target :: A(:, :)
    call ms_check(c_ms_m_register_szden(ckey(m_name), int(size(A, 1), c_int), int(size(A, 2), c_int), c_loc(A)), &
                  'm_register_sden')
  end subroutine m_register_szden

  subroutine m_register_pdcsc(m_name, idx1, idx2, val, desc)
    character(*), intent(in) :: m_name
    integer, intent(in), target :: idx1(:), idx2(:)
    real(dp), intent(in), target :: val(:)
    integer, intent(in) :: desc(9)
    call ms_check(c_ms_m_register_pdcsc(ckey(m_name), c_loc(idx1), c_loc(idx2), c_loc(val), int(desc, c_int)), &
                  'm_register_pcsc')
  end subroutine m_register_pdcsc

  subroutine m_register_pzcsc(m_name, idx1, idx2, val, desc)
    character(*), intent(in) :: m_name
    integer, intent(in), target :: idx1(:), idx2(:)
    complex(dp), intent(in), target :: val(:)
    integer, intent(in) :: desc(9)
    call ms_check(c_ms_m_register_pzcsc(ckey(m_name), c_loc(idx1), c_loc(idx2), c_loc(val), int(desc, c_int)), &
                  'm_register_pcsc')
  end subroutine m_register_pzcsc

  ! omm_wrapper (libOMM/src/omm_wrapper.F90:5-96), CBIND form: c_bool logicals
  subroutine omm_wrapper(m, n, H, S, new_S, e_min, D_min, calc_ED, eta, C_min, init_C, T, scale_T, flavour, np, ip, &
                         cg_tol, long_out, dealloc, m_storage, m_operation)
    integer, intent(in) :: m, n, flavour, np, ip
    character(*), intent(in) :: H, S, D_min, C_min, T
    logical(c_bool), intent(in) :: new_S, calc_ED, init_C, long_out, dealloc
    real(dp), intent(out) :: e_min
    real(dp), intent(in) :: eta, scale_T, cg_tol
    character(5), intent(in) :: m_storage
    character(3), intent(in) :: m_operation
    character(kind=c_char), dimension(5) :: st
    character(kind=c_char), dimension(3) :: op
    integer :: k
    do k = 1, 5
      st(k) = m_storage(k:k)
    end do
    do k = 1, 3
      op(k) = m_operation(k:k)
    end do
    call ms_check(c_omm_wrapper(int(m, c_int), int(n, c_int), ckey(H), ckey(S), new_S, e_min, ckey(D_min), calc_ED, &
                                eta, ckey(C_min), init_C, ckey(T), scale_T, int(flavour, c_int), int(np, c_int), &
                                int(ip, c_int), cg_tol, long_out, dealloc, st, op), 'omm_wrapper')
  end subroutine omm_wrapper

end module MatrixSwitch_wrapper

! tomato_TB (tomato/src/tomato_TB.F90:1-636): the reference's external subroutine, same argument
! list and in/out meaning, running tomato_gpu_TB.  H and S come back as matrices of the library
! (S left uninitialised when the template has no overlap, both when build_matrix is false).
subroutine tomato_TB(template_basedir, system_label, switch1, frac_occ, num_orbs_per_atom, switch2, num_orbs, &
                     num_cells_dir, switch3, sparsity, orb_r_cut, num_occ_states, gamma_point, k_point, defect, &
                     defect_perturbation, H, S, m_storage, build_matrix)
  use iso_c_binding
  use MatrixSwitch
  implicit none
  integer, parameter :: dp = selected_real_kind(15, 300)
  character(*), intent(in) :: template_basedir, system_label
  character(5), intent(in) :: m_storage
  logical, intent(in) :: switch1, switch2, switch3, gamma_point, build_matrix, defect
  real(dp), intent(in) :: defect_perturbation
  integer, intent(out) :: num_occ_states
  integer, intent(inout) :: num_orbs_per_atom, num_orbs, num_cells_dir(3)
  real(dp), intent(inout) :: frac_occ, sparsity, orb_r_cut, k_point(3)
  type(matrix), intent(inout) :: H, S
  interface
    integer(c_int) function c_tomato_tb(template_basedir, system_label, switch1, frac_occ, num_orbs_per_atom, &
        switch2, num_orbs, num_cells_dir, switch3, sparsity, orb_r_cut, num_occ_states, gamma_point, k_point, &
        defect, defect_perturbation, H, S, m_storage, build_matrix) bind(c, name="tomato_gpu_TB")
      import :: c_int, c_char, c_double, c_bool, c_ptr
      character(kind=c_char), dimension(*), intent(in) :: template_basedir, system_label
      logical(c_bool), value :: switch1, switch2, switch3, gamma_point, defect, build_matrix
      real(c_double), intent(inout) :: frac_occ, sparsity, orb_r_cut
      integer(c_int), intent(inout) :: num_orbs_per_atom, num_orbs
      integer(c_int), dimension(3), intent(inout) :: num_cells_dir
      integer(c_int), intent(out) :: num_occ_states
      real(c_double), dimension(3), intent(inout) :: k_point
      real(c_double), value :: defect_perturbation
      type(c_ptr), intent(inout) :: H, S
      character(kind=c_char), dimension(5), intent(in) :: m_storage
    end function
  end interface
  integer(c_int) :: nopa, no, ncd(3), nocc
  character(kind=c_char), dimension(5) :: st
  integer :: k
  nopa = num_orbs_per_atom
  no = num_orbs
  ncd = num_cells_dir
  do k = 1, 5
    st(k) = m_storage(k:k)
  end do
  call ms_check(c_tomato_tb(ckey(template_basedir), ckey(system_label), logical(switch1, c_bool), frac_occ, nopa, &
                            logical(switch2, c_bool), no, ncd, logical(switch3, c_bool), sparsity, orb_r_cut, nocc, &
                            logical(gamma_point, c_bool), k_point, logical(defect, c_bool), defect_perturbation, &
                            H%h, S%h, st, logical(build_matrix, c_bool)), 'tomato_TB')
  num_orbs_per_atom = nopa
  num_orbs = no
  num_cells_dir = ncd
  num_occ_states = nocc
  if (c_associated(H%h)) then
    H%is_initialized = .true.
    H%is_real = gamma_point
    H%dim1 = num_orbs
    H%dim2 = num_orbs
  end if
  if (c_associated(S%h)) then
    S%is_initialized = .true.
    S%is_real = gamma_point
    S%dim1 = num_orbs
    S%dim2 = num_orbs
  end if
end subroutine tomato_TB
