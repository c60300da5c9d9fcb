! Brute-force check of the Fortran front end (built and run by
! tests/test_gpu_fortran.py when a Fortran compiler is available): periodic kNN,
! ball and box searches on seeded points against direct evaluation, in the
! manner of the reference's demos (demos/cosmokdtree/periodic/tree_test.f90:79-139,
! demos/cosmokdtree/box_search/tree_test.f90:85-97).  Prints "OK" on success.
program test_cosmokdtree_gpu
  use iso_c_binding
  use cosmokdtree_gpu
  implicit none
  integer, parameter :: n = 20000, nd = 3, k = 8, nq = 50
  real(c_double) :: pts(n, nd), lbox(nd), q(nd), d2(n), box(2 * nd), r, dx
  type(KDTreeGPU) :: tree
  type(KDTreeResult) :: res
  integer :: i, j, t, cnt, bad, order(n)
  integer(c_int64_t), allocatable :: off(:), idx(:)
  real(c_double), allocatable :: dist(:)
  real(c_double) :: targets(nq, nd)
  call random_seed_fixed()
  call random_number(pts)
  pts = pts - 0.5_c_double
  lbox = 1.0_c_double
  tree = build_kdtree(pts, lbox, 16)
  bad = 0
  do t = 1, nq
    q = pts(t * 37, :)
    targets(t, :) = q
    do i = 1, n
      d2(i) = 0
      do j = 1, nd
        dx = abs(pts(i, j) - q(j))
        dx = min(dx, lbox(j) - dx)
        d2(i) = d2(i) + dx * dx
      end do
    end do
    call rank_order(d2, order)
    res = knn_search(tree, q, k)
    do i = 1, k
      if (res%idx(i) /= order(i)) bad = bad + 1
      if (res%dist(i) /= sqrt(d2(order(i)))) bad = bad + 1
    end do
    r = 0.03_c_double
    res = ball_search(tree, q, r, .true.)
    cnt = count(d2 <= r * r)
    if (size(res%idx) /= cnt) bad = bad + 1
    do i = 1, min(cnt, size(res%idx))
      if (res%idx(i) /= order(i)) bad = bad + 1
    end do
    box = [q(1) - 0.05_c_double, q(1) + 0.05_c_double, q(2) - 0.05_c_double, &
           q(2) + 0.05_c_double, q(3) - 0.05_c_double, q(3) + 0.05_c_double]
    res = box_search(tree, box)
    cnt = 0
    do i = 1, n
      if (all(pts(i, :) >= box(1::2)) .and. all(pts(i, :) <= box(2::2))) cnt = cnt + 1
    end do
    if (size(res%idx) /= cnt) bad = bad + 1
  end do
  call ball_search_many(tree, targets, 0.03_c_double, off, idx, dist, .true.)
  if (size(off) /= nq + 1) bad = bad + 1
  call deallocate_kdtree(tree)
  if (bad == 0) then
    write(*, '(a)') 'OK'
  else
    write(*, '(a, i0)') 'FAILED ', bad
    error stop 1
  end if
contains
  subroutine random_seed_fixed()
    integer :: m
    integer, allocatable :: seed(:)
    call random_seed(size=m)
    allocate(seed(m))
    seed = 12345
    call random_seed(put=seed)
  end subroutine random_seed_fixed

  ! indices sorting d (ascending, ties by lower index): insertion of the k + few
  ! smallest is enough here, but a full selection keeps it simple
  subroutine rank_order(d, ord)
    real(c_double), intent(in) :: d(:)
    integer, intent(out) :: ord(:)
    integer :: a, b, tmp
    do a = 1, size(d)
      ord(a) = a
    end do
    do a = 1, min(size(d), 400)
      do b = a + 1, size(d)
        if (d(ord(b)) < d(ord(a)) .or. (d(ord(b)) == d(ord(a)) .and. ord(b) < ord(a))) then
          tmp = ord(a)
          ord(a) = ord(b)
          ord(b) = tmp
        end if
      end do
    end do
  end subroutine rank_order
end program test_cosmokdtree_gpu
