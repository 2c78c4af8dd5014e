! rf_gpu.f90 -- Fortran binding of the B200 random-field generator.
!
! Gives Fortran callers the reference's documented entry point
!   createStandardGaussianFieldUnstruct(xPoints, corrMod, margiFirst, corrL,
!                                       fieldAvg, fieldVar, Nmc, method, randField)
! (cottereau/randomField README.md:58-92) on top of the C-ABI in
! include/randomfield_b200.h through iso_c_binding.  Arrays keep the
! reference's layouts: xPoints(nDim, n), randField(n, Nmc).  corrMod and
! margiFirst are the README's strings ("gaussian"; "gaussian" or
! "lognormal"); method is 1 (isotropic), 2 (Shinozuka-Deodatis) or 3
! (randomization).
!
! Errors: with the optional `status` argument present the C status code is
! returned (0 = success, negative RF_E* codes otherwise); without it an error
! prints the library's message and stops, as the reference does.
!
! Build: compile this file with any Fortran 2003 compiler and link
! randomfield_b200/librf_b200.so, e.g.
!   gfortran -c rf_gpu.f90 && gfortran app.f90 rf_gpu.o -L<dir> -lrf_b200
module rf_gpu
  use, intrinsic :: iso_c_binding
  implicit none
  private

  ! constants_RF.f90:12-21
  integer, parameter, public :: RF_ISOTROPIC = 1, RF_SHINOZUKA = 2, RF_RANDOMIZATION = 3
  integer, parameter, public :: RF_CM_GAUSSIAN = 1, RF_CM_COS = 2
  integer, parameter, public :: RF_FOM_GAUSSIAN = 1, RF_FOM_LOGNORMAL = 2
  ! precision forms of the contraction
  integer, parameter, public :: RF_PREC_BF16 = 0, RF_PREC_FP16 = 1, RF_PREC_FP32 = 2, RF_PREC_BF16_FAST = 3

  ! rf_options (include/randomfield_b200.h), same member order and types
  type, bind(C), public :: rf_options_t
    integer(c_int32_t) :: size
    integer(c_int32_t) :: precision
    integer(c_int64_t) :: seed_start
    integer(c_int32_t) :: k_nstep(3)
    integer(c_int32_t) :: iso_n_radial
    integer(c_int32_t) :: iso_n_dir
    integer(c_int32_t) :: literal
    integer(c_int32_t) :: normalize
    real(c_double) :: x_range(3)
    integer(c_int32_t) :: device
    integer(c_int32_t) :: reserved0
    type(c_ptr) :: draws            ! c_loc of real(c_double) draws(n_draws), or c_null_ptr
    integer(c_int64_t) :: n_draws
    integer(c_int32_t) :: reserved(2)
  end type rf_options_t

  ! rf_result_attributes (include/randomfield_b200.h): write_HDF5_attributes' parameters
  type, bind(C), public :: rf_result_attributes_t
    integer(c_int32_t) :: nb_procs = 1, nDim = 0, Nmc = 0, method = 0, seedStart = 0, corrMod = 0, &
                          margiFirst = 0, localizationLevel = 0
    integer(c_int32_t) :: kNStep(3) = 0, nFields(3) = 1
    real(c_double) :: xMinGlob(3) = 0d0, xMaxGlob(3) = 0d0, xStep(3) = 0d0, corrL(3) = 0d0, overlap(3) = 0d0, &
                      procExtent(3) = 0d0, kMax_out(3) = 0d0
  end type rf_result_attributes_t

  public :: createStandardGaussianFieldUnstruct, createStandardGaussianFieldGrid, rf_options_init
  public :: writeResultGrid

  interface
    subroutine rf_options_init(opt) bind(C, name="rf_options_init")
      import :: rf_options_t
      type(rf_options_t), intent(out) :: opt
    end subroutine rf_options_init

    integer(c_int) function c_create(xPoints, nDim, n, corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc, &
                                     method, randField, opt) bind(C, name="rf_create_standard_gaussian_field_unstruct")
      import :: c_int, c_int64_t, c_double, rf_options_t
      real(c_double), intent(in) :: xPoints(*)
      integer(c_int), value :: nDim
      integer(c_int64_t), value :: n
      integer(c_int), value :: corrMod, margiFirst
      real(c_double), intent(in) :: corrL(*)
      real(c_double), value :: fieldAvg, fieldVar
      integer(c_int), value :: Nmc, method
      real(c_double), intent(inout) :: randField(*)
      type(rf_options_t), intent(in) :: opt
    end function c_create

    integer(c_int) function c_create_grid(nDim, xMin, xStep, xNStep, corrMod, margiFirst, corrL, fieldAvg, &
                                          fieldVar, Nmc, method, randField, opt) &
                                          bind(C, name="rf_create_standard_gaussian_field_grid")
      import :: c_int, c_int64_t, c_double, rf_options_t
      integer(c_int), value :: nDim
      real(c_double), intent(in) :: xMin(*), xStep(*)
      integer(c_int64_t), intent(in) :: xNStep(*)
      integer(c_int), value :: corrMod, margiFirst
      real(c_double), intent(in) :: corrL(*)
      real(c_double), value :: fieldAvg, fieldVar
      integer(c_int), value :: Nmc, method
      real(c_double), intent(inout) :: randField(*)
      type(rf_options_t), intent(in) :: opt
    end function c_create_grid

    integer(c_int) function c_write_result_grid(folder, fileName, nDim, xMin, xMax, xStep, field, attr) &
                                                bind(C, name="rf_write_result_grid")
      import :: c_int, c_double, c_char, rf_result_attributes_t
      character(kind=c_char), intent(in) :: folder(*), fileName(*)
      integer(c_int), value :: nDim
      real(c_double), intent(in) :: xMin(*), xMax(*), xStep(*), field(*)
      type(rf_result_attributes_t), intent(in) :: attr
    end function c_write_result_grid

    type(c_ptr) function c_last_error() bind(C, name="rf_last_error")
      import :: c_ptr
    end function c_last_error

    integer(c_size_t) function c_strlen(s) bind(C, name="strlen")
      import :: c_ptr, c_size_t
      type(c_ptr), value :: s
    end function c_strlen
  end interface

contains

  ! The documented entry point (README.md:58-92).  Optional arguments beyond
  ! the reference's: seedStart (>= 0, the reference's seedStart), options
  ! (a full rf_options_t) and status.
  subroutine createStandardGaussianFieldUnstruct(xPoints, corrMod, margiFirst, corrL, fieldAvg, fieldVar, &
                                                 Nmc, method, randField, seedStart, options, status)
    double precision, intent(in) :: xPoints(:, :)
    character(len=*), intent(in) :: corrMod, margiFirst
    double precision, intent(in) :: corrL(:)
    double precision, intent(in) :: fieldAvg, fieldVar
    integer, intent(in) :: Nmc, method
    double precision, intent(inout) :: randField(:, :)
    integer, intent(in), optional :: seedStart
    type(rf_options_t), intent(in), optional :: options
    integer, intent(out), optional :: status

    type(rf_options_t) :: opt
    integer(c_int) :: rc, cm, fom

    if (present(options)) then
      opt = options
    else
      call rf_options_init(opt)
    end if
    if (present(seedStart)) opt%seed_start = int(seedStart, c_int64_t)

    select case (trim(adjustl(corrMod)))
    case ("gaussian")
      cm = RF_CM_GAUSSIAN
    case ("cos")
      cm = RF_CM_COS
    case default
      cm = -1
    end select
    select case (trim(adjustl(margiFirst)))
    case ("gaussian")
      fom = RF_FOM_GAUSSIAN
    case ("lognormal")
      fom = RF_FOM_LOGNORMAL
    case default
      fom = -1
    end select

    if (size(randField, 1) /= size(xPoints, 2) .or. size(randField, 2) /= Nmc) then
      rc = -9  ! RF_EINVAL_ARG
    else
      rc = c_create(xPoints, int(size(xPoints, 1), c_int), int(size(xPoints, 2), c_int64_t), cm, fom, corrL, &
                    real(fieldAvg, c_double), real(fieldVar, c_double), int(Nmc, c_int), int(method, c_int), &
                    randField, opt)
    end if

    if (present(status)) then
      status = int(rc)
    else if (rc /= 0) then
      write (*, *) "createStandardGaussianFieldUnstruct: error ", rc, " ", last_error()
      stop 1
    end if
  end subroutine createStandardGaussianFieldUnstruct

  ! The same field on the structured grid xMin + j xStep (xNStep points per
  ! axis, axis 1 fastest), i.e. on the points set_XPoints would build
  ! (mesh_RF.f90:17-64), without building them: the sum runs axis by axis in
  ! FP64 (rf_create_standard_gaussian_field_grid).  Method 2 only; randField
  ! is (product(xNStep), Nmc).
  subroutine createStandardGaussianFieldGrid(xMin, xStep, xNStep, corrMod, margiFirst, corrL, fieldAvg, fieldVar, &
                                             Nmc, method, randField, seedStart, options, status)
    double precision, intent(in) :: xMin(:), xStep(:)
    integer, intent(in) :: xNStep(:)
    character(len=*), intent(in) :: corrMod, margiFirst
    double precision, intent(in) :: corrL(:)
    double precision, intent(in) :: fieldAvg, fieldVar
    integer, intent(in) :: Nmc, method
    double precision, intent(inout) :: randField(:, :)
    integer, intent(in), optional :: seedStart
    type(rf_options_t), intent(in), optional :: options
    integer, intent(out), optional :: status

    type(rf_options_t) :: opt
    integer(c_int) :: rc
    integer(c_int64_t) :: nsteps(3)
    integer :: d, nd

    if (present(options)) then
      opt = options
    else
      call rf_options_init(opt)
    end if
    if (present(seedStart)) opt%seed_start = int(seedStart, c_int64_t)
    nd = size(xNStep)
    nsteps = 1
    do d = 1, min(nd, 3)
      nsteps(d) = int(xNStep(d), c_int64_t)
    end do

    if (nd < 1 .or. nd > 3 .or. size(xMin) /= nd .or. size(xStep) /= nd .or. size(corrL) /= nd .or. &
        size(randField, 1) /= product(nsteps) .or. size(randField, 2) /= Nmc) then
      rc = -9  ! RF_EINVAL_ARG
    else
      rc = c_create_grid(int(nd, c_int), xMin, xStep, nsteps, corrmod_id(corrMod), margi_id(margiFirst), corrL, &
                         real(fieldAvg, c_double), real(fieldVar, c_double), int(Nmc, c_int), int(method, c_int), &
                         randField, opt)
    end if

    if (present(status)) then
      status = int(rc)
    else if (rc /= 0) then
      write (*, *) "createStandardGaussianFieldGrid: error ", rc, " ", last_error()
      stop 1
    end if
  end subroutine createStandardGaussianFieldGrid

  ! The result files of one realization, as write_MONO_proc_result writes
  ! them (writeResultFile_RF.f90:737-829): <folder>/h5/<fileName>.h5 with
  ! the dataset "samples" and the attributes, <folder>/xmf/<fileName>.xmf.
  subroutine writeResultGrid(folder, fileName, xMin, xMax, xStep, field, attributes, status)
    character(len=*), intent(in) :: folder, fileName
    double precision, intent(in) :: xMin(:), xMax(:), xStep(:), field(:)
    type(rf_result_attributes_t), intent(in) :: attributes
    integer, intent(out), optional :: status
    integer(c_int) :: rc
    rc = c_write_result_grid(trim(folder)//c_null_char, trim(fileName)//c_null_char, int(size(xMin), c_int), &
                             xMin, xMax, xStep, field, attributes)
    if (present(status)) then
      status = int(rc)
    else if (rc /= 0) then
      write (*, *) "writeResultGrid: error ", rc, " ", last_error()
      stop 1
    end if
  end subroutine writeResultGrid

  integer(c_int) function corrmod_id(name)
    character(len=*), intent(in) :: name
    select case (trim(adjustl(name)))
    case ("gaussian")
      corrmod_id = RF_CM_GAUSSIAN
    case ("cos")
      corrmod_id = RF_CM_COS
    case default
      corrmod_id = -1
    end select
  end function corrmod_id

  integer(c_int) function margi_id(name)
    character(len=*), intent(in) :: name
    select case (trim(adjustl(name)))
    case ("gaussian")
      margi_id = RF_FOM_GAUSSIAN
    case ("lognormal")
      margi_id = RF_FOM_LOGNORMAL
    case default
      margi_id = -1
    end select
  end function margi_id

  function last_error() result(msg)
    character(len=:), allocatable :: msg
    type(c_ptr) :: p
    character(kind=c_char), pointer :: chars(:)
    integer :: i, n
    p = c_last_error()
    n = int(c_strlen(p))
    call c_f_pointer(p, chars, [n])
    allocate (character(len=n) :: msg)
    do i = 1, n
      msg(i:i) = chars(i)
    end do
  end function last_error

end module rf_gpu
