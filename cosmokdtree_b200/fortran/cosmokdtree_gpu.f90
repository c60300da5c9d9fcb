! cosmokdtree_gpu -- Fortran front end of libckd.so (the B200 k-d tree).
!
! The procedures keep the call shapes of the reference module cosmokdtree
! (src/cosmokdtree.f90) so that Fortran codes that call it directly can switch:
!
!   tree  = build_kdtree(points_in, L_in, leaf)   ! :124-238, points_in(n, ndim);
!                                                 ! L_in present = periodic tree
!   query = knn_search(tree, targett, k, sorted)  ! :504-540, query%idx, query%dist
!   query = ball_search(tree, targett, radius, sorted)   ! :1015-1072
!   query = box_search(tree, box)                 ! :1220-1253, box(2*ndim)
!   call deallocate_kdtree(tree)
!
! Differences: the tree is a value of type KDTreeGPU (assign with `=`, not `=>`),
! the box side travels with each tree instead of a module global (:87), errors
! are reported through `stat` arguments or stop with the library's message
! instead of STOP codes, and batched forms (knn_search_many, ball_search_many,
! box_search_many) serve many queries per call, which is what the GPU needs to be
! fast.  Ids are 1-based positions in points_in, as in the reference; a missing
! neighbour (k > n) has idx -1 and dist sqrt(HUGE(0.0)), as in the reference.
!
! Link with libckd.so (built by cosmokdtree_b200/csrc/Makefile); the C entry
! points it binds are declared in include/ckd.h.
module cosmokdtree_gpu
  use iso_c_binding
  implicit none
  private

  public :: KDTreeGPU, KDTreeResult
  public :: build_kdtree, deallocate_kdtree
  public :: knn_search, knn_search_many, ball_search, ball_search_many
  public :: box_search, box_search_many, ckd_error_message

  integer, parameter :: dp = c_double

  type :: KDTreeGPU
    type(c_ptr) :: h = c_null_ptr
    integer :: ndim = 0
  end type KDTreeGPU

  type :: KDTreeResult
    integer(kind=c_int64_t), allocatable :: idx(:)
    real(kind=dp), allocatable :: dist(:)
  end type KDTreeResult

  interface
    function c_build(pts, n, d, dtype, leaf, boxsize, on_dev, stream, out) &
        bind(C, name="ckd_build") result(st)
      import :: c_ptr, c_int, c_int64_t, c_double
      real(c_double), intent(in) :: pts(*)
      integer(c_int64_t), value :: n
      integer(c_int), value :: d, dtype, leaf
      type(c_ptr), value :: boxsize
      integer(c_int), value :: on_dev
      type(c_ptr), value :: stream
      type(c_ptr), intent(out) :: out
      integer(c_int) :: st
    end function c_build

    function c_free(tree) bind(C, name="ckd_free") result(st)
      import :: c_ptr, c_int
      type(c_ptr), value :: tree
      integer(c_int) :: st
    end function c_free

    function c_last_error() bind(C, name="ckd_last_error") result(msg)
      import :: c_ptr
      type(c_ptr) :: msg
    end function c_last_error

    function c_knn_host(tree, q, nq, k, sorted, dist, idx, stream) &
        bind(C, name="ckd_knn_host") result(st)
      import :: c_ptr, c_int, c_int64_t, c_double
      type(c_ptr), value :: tree
      real(c_double), intent(in) :: q(*)
      integer(c_int64_t), value :: nq
      integer(c_int), value :: k, sorted
      real(c_double), intent(out) :: dist(*)
      integer(c_int64_t), intent(out) :: idx(*)
      type(c_ptr), value :: stream
      integer(c_int) :: st
    end function c_knn_host

    function c_ball_count_host(tree, q, nq, radius, offsets, stream) &
        bind(C, name="ckd_ball_count_host") result(st)
      import :: c_ptr, c_int, c_int64_t, c_double
      type(c_ptr), value :: tree
      real(c_double), intent(in) :: q(*)
      integer(c_int64_t), value :: nq
      real(c_double), value :: radius
      integer(c_int64_t), intent(out) :: offsets(*)
      type(c_ptr), value :: stream
      integer(c_int) :: st
    end function c_ball_count_host

    function c_ball_fill_host(tree, q, nq, radius, sorted, offsets, idx, dist, stream) &
        bind(C, name="ckd_ball_fill_host") result(st)
      import :: c_ptr, c_int, c_int64_t, c_double
      type(c_ptr), value :: tree
      real(c_double), intent(in) :: q(*)
      integer(c_int64_t), value :: nq
      real(c_double), value :: radius
      integer(c_int), value :: sorted
      integer(c_int64_t), intent(in) :: offsets(*)
      integer(c_int64_t), intent(out) :: idx(*)
      real(c_double), intent(out) :: dist(*)
      type(c_ptr), value :: stream
      integer(c_int) :: st
    end function c_ball_fill_host

    function c_box_count_host(tree, boxes, nb, offsets, stream) &
        bind(C, name="ckd_box_count_host") result(st)
      import :: c_ptr, c_int, c_int64_t, c_double
      type(c_ptr), value :: tree
      real(c_double), intent(in) :: boxes(*)
      integer(c_int64_t), value :: nb
      integer(c_int64_t), intent(out) :: offsets(*)
      type(c_ptr), value :: stream
      integer(c_int) :: st
    end function c_box_count_host

    function c_box_fill_host(tree, boxes, nb, offsets, idx, stream) &
        bind(C, name="ckd_box_fill_host") result(st)
      import :: c_ptr, c_int, c_int64_t, c_double
      type(c_ptr), value :: tree
      real(c_double), intent(in) :: boxes(*)
      integer(c_int64_t), value :: nb
      integer(c_int64_t), intent(in) :: offsets(*)
      integer(c_int64_t), intent(out) :: idx(*)
      type(c_ptr), value :: stream
      integer(c_int) :: st
    end function c_box_fill_host

    function c_strlen(s) bind(C, name="strlen") result(n)
      import :: c_ptr, c_size_t
      type(c_ptr), value :: s
      integer(c_size_t) :: n
    end function c_strlen
  end interface

contains

  ! message of the library's last failure on this thread
  function ckd_error_message() result(msg)
    character(len=:), allocatable :: msg
    type(c_ptr) :: p
    character(kind=c_char), pointer :: chars(:)
    integer :: n, i
    p = c_last_error()
    if (.not. c_associated(p)) then
      msg = ''
      return
    end if
    n = int(c_strlen(p))
    call c_f_pointer(p, chars, [n])
    allocate(character(len=n) :: msg)
    do i = 1, n
      msg(i:i) = chars(i)
    end do
  end function ckd_error_message

  subroutine check(st, stat)
    integer(c_int), intent(in) :: st
    integer, intent(out), optional :: stat
    if (present(stat)) then
      stat = int(st)
    else if (st /= 0) then
      write(*, '(a)') 'cosmokdtree_gpu: ' // ckd_error_message()
      error stop 1
    end if
  end subroutine check

  ! points_in(n, ndim) as in the reference; L_in(ndim) makes the tree periodic
  ! with coordinates in [-L/2, L/2] (:177-190)
  function build_kdtree(points_in, L_in, leaf, stat) result(tree)
    real(dp), intent(in) :: points_in(:, :)
    real(dp), intent(in), optional :: L_in(:)
    integer, intent(in), optional :: leaf
    integer, intent(out), optional :: stat
    type(KDTreeGPU) :: tree
    real(c_double), allocatable :: pts(:, :)
    real(c_double), allocatable, target :: lbox(:)
    type(c_ptr) :: bp, h
    integer(c_int) :: lf, st
    lf = 16
    if (present(leaf)) lf = int(leaf, c_int)
    pts = transpose(points_in)  ! (ndim, n): each point's coordinates contiguous
    bp = c_null_ptr
    if (present(L_in)) then
      lbox = L_in
      bp = c_loc(lbox)
    end if
    st = c_build(pts, int(size(points_in, 1), c_int64_t), int(size(points_in, 2), c_int), &
                 0_c_int, lf, bp, 0_c_int, c_null_ptr, h)
    call check(st, stat)
    if (st == 0) then
      tree%h = h
      tree%ndim = size(points_in, 2)
    end if
  end function build_kdtree

  subroutine deallocate_kdtree(tree)
    type(KDTreeGPU), intent(inout) :: tree
    integer(c_int) :: st
    if (c_associated(tree%h)) st = c_free(tree%h)
    tree%h = c_null_ptr
    tree%ndim = 0
  end subroutine deallocate_kdtree

  ! targets(ntar, ndim); dist(ntar, k), idx(ntar, k), as pyknn_search returns them
  ! (cosmokdtree2py.f90:103-147) but with 1-based ids
  subroutine knn_search_many(tree, targets, k, dist, idx, sorted, stat)
    type(KDTreeGPU), intent(in) :: tree
    real(dp), intent(in) :: targets(:, :)
    integer, intent(in) :: k
    real(dp), allocatable, intent(out) :: dist(:, :)
    integer(c_int64_t), allocatable, intent(out) :: idx(:, :)
    logical, intent(in), optional :: sorted
    integer, intent(out), optional :: stat
    real(c_double), allocatable :: q(:, :), d(:, :)
    integer(c_int64_t), allocatable :: ii(:, :)
    integer(c_int) :: srt, st
    integer(c_int64_t) :: nq
    srt = 1
    if (present(sorted)) then
      if (.not. sorted) srt = 0
    end if
    nq = size(targets, 1)
    q = transpose(targets)
    allocate(d(k, nq), ii(k, nq))
    st = c_knn_host(tree%h, q, nq, int(k, c_int), srt, d, ii, c_null_ptr)
    call check(st, stat)
    if (st /= 0) return
    dist = transpose(d)
    idx = transpose(ii) + 1_c_int64_t
  end subroutine knn_search_many

  function knn_search(tree, targett, k, sorted) result(query)
    type(KDTreeGPU), intent(in) :: tree
    real(dp), intent(in) :: targett(:)
    integer, intent(in) :: k
    logical, intent(in), optional :: sorted
    type(KDTreeResult) :: query
    real(dp), allocatable :: d(:, :)
    integer(c_int64_t), allocatable :: ii(:, :)
    call knn_search_many(tree, reshape(targett, [1, size(targett)]), k, d, ii, sorted)
    query%idx = ii(1, :)
    query%dist = d(1, :)
  end function knn_search

  ! targets(ntar, ndim); CSR rows: results of target i are offsets(i)+1 .. offsets(i+1)
  subroutine ball_search_many(tree, targets, radius, offsets, idx, dist, sorted, stat)
    type(KDTreeGPU), intent(in) :: tree
    real(dp), intent(in) :: targets(:, :)
    real(dp), intent(in) :: radius
    integer(c_int64_t), allocatable, intent(out) :: offsets(:), idx(:)
    real(dp), allocatable, intent(out) :: dist(:)
    logical, intent(in), optional :: sorted
    integer, intent(out), optional :: stat
    real(c_double), allocatable :: q(:, :)
    integer(c_int) :: srt, st
    integer(c_int64_t) :: nq, total
    srt = 0
    if (present(sorted)) then
      if (sorted) srt = 1
    end if
    nq = size(targets, 1)
    q = transpose(targets)
    allocate(offsets(nq + 1))
    st = c_ball_count_host(tree%h, q, nq, real(radius, c_double), offsets, c_null_ptr)
    call check(st, stat)
    if (st /= 0) return
    total = offsets(nq + 1)
    allocate(idx(max(total, 1_c_int64_t)), dist(max(total, 1_c_int64_t)))
    st = c_ball_fill_host(tree%h, q, nq, real(radius, c_double), srt, offsets, idx, dist, &
                          c_null_ptr)
    call check(st, stat)
    if (st /= 0) return
    idx = idx(1:total) + 1_c_int64_t
    dist = dist(1:total)
  end subroutine ball_search_many

  function ball_search(tree, targett, radius, sorted) result(query)
    type(KDTreeGPU), intent(in) :: tree
    real(dp), intent(in) :: targett(:)
    real(dp), intent(in) :: radius
    logical, intent(in), optional :: sorted
    type(KDTreeResult) :: query
    integer(c_int64_t), allocatable :: off(:), ii(:)
    real(dp), allocatable :: d(:)
    call ball_search_many(tree, reshape(targett, [1, size(targett)]), radius, off, ii, d, sorted)
    query%idx = ii
    query%dist = d
  end function ball_search

  ! boxes(nbox, 2*ndim), each row (xmin, xmax, ymin, ymax, ...)
  subroutine box_search_many(tree, boxes, offsets, idx, stat)
    type(KDTreeGPU), intent(in) :: tree
    real(dp), intent(in) :: boxes(:, :)
    integer(c_int64_t), allocatable, intent(out) :: offsets(:), idx(:)
    integer, intent(out), optional :: stat
    real(c_double), allocatable :: b(:, :)
    integer(c_int) :: st
    integer(c_int64_t) :: nb, total
    nb = size(boxes, 1)
    b = transpose(boxes)
    allocate(offsets(nb + 1))
    st = c_box_count_host(tree%h, b, nb, offsets, c_null_ptr)
    call check(st, stat)
    if (st /= 0) return
    total = offsets(nb + 1)
    allocate(idx(max(total, 1_c_int64_t)))
    st = c_box_fill_host(tree%h, b, nb, offsets, idx, c_null_ptr)
    call check(st, stat)
    if (st /= 0) return
    idx = idx(1:total) + 1_c_int64_t
  end subroutine box_search_many

  function box_search(tree, box) result(query)
    type(KDTreeGPU), intent(in) :: tree
    real(dp), intent(in) :: box(:)
    type(KDTreeResult) :: query
    integer(c_int64_t), allocatable :: off(:), ii(:)
    call box_search_many(tree, reshape(box, [1, size(box)]), off, ii)
    query%idx = ii
  end function box_search

end module cosmokdtree_gpu
