! w2d_iface.f90 -- ISO_C_BINDING interface of libw2d.so (include/w2d.h) for
! the reference's Fortran host (Walicxe-2D, src/*.f90).
!
! A host keeps its main loop (src/main.f90) and its block tree (admesh,
! markref, critneighup/down, updatelpup/down, locatebounds, basegrid) and
! replaces the bodies of timestep, tstep and the u motion of refine/coarse
! with the calls below.  Every function returns 0 (W2D_OK) or a W2D_ERR_*
! status; w2d_last_error then holds the block, cell and message.
!
! Arrays are passed as the reference holds them: lp(nbmin:,1:8),
! icoord(nbmin:,1:2) and innerbounds(:,1:3) column-major with their leading
! dimension, leaf as 4-byte integers (merge(1,0,leaf)), u(nbmin:nbmaxtot,
! neq,-1:18,-1:18) for the *_u_fortran calls.  Scalars go by value.
module w2d_iface
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: W2D_OK = 0, W2D_ERR_ARG = 1, W2D_ERR_CUDA = 2, &
       W2D_ERR_HLLC = 3, W2D_ERR_CAPACITY = 4, W2D_ERR_TOPOLOGY = 5, W2D_ERR_TIMEOUT = 6, &
       W2D_ERR_STATE = 7, W2D_ERR_NOMEM = 8
  integer(c_int32_t), parameter :: W2D_HLLC = 0, W2D_HLL = 1, W2D_HLL_HLLC = 2
  integer(c_int32_t), parameter :: W2D_ADIABATIC = 0, W2D_COOLINGH = 1, W2D_COOLINGDMC = 2
  integer(c_int32_t), parameter :: W2D_BC_OUTFLOW = 0, W2D_BC_REFLECTIVE = 1
  integer(c_int32_t), parameter :: W2D_USERBC_NONE = 0, W2D_USERBC_JET = 1
  integer(c_int32_t), parameter :: W2D_GEOM_CARTESIAN = 0, W2D_GEOM_CYLINDRICAL = 1
  integer(c_int32_t), parameter :: W2D_COMPAT_HLLC_STAR = 1, W2D_COMPAT_OUTFYB = 2

  ! W2dParams of include/w2d.h, field for field (src/parameters.f90 and the
  ! -D flags of JET/Makefile:27-62 as run-time values)
  type, bind(C) :: w2d_params
    integer(c_int32_t) :: neq, npas, nx, ny, nlevs, nbroot_x, nbroot_y, nblocks
    integer(c_int32_t) :: solver, limiter, cooling
    integer(c_int32_t) :: bc_left, bc_right, bc_bottom, bc_top, otherb, compat
    integer(c_int32_t) :: precision, geometry
    real(c_double) :: cv, gamma, cfl, eta
    real(c_double) :: xmax, ymax
    real(c_double) :: tempsc, psc, tsc, rsc
    real(c_double) :: tol, tol2
    real(c_double) :: jet_rj, jet_lj, jet_posx, jet_posy
    real(c_double) :: jet_den, jet_temp, jet_v0, jet_dv, jet_tau
  end type w2d_params

  ! W2dError of include/w2d.h
  type, bind(C) :: w2d_error
    integer(c_int32_t) :: code, block, i, j
    character(kind=c_char) :: message(240)
  end type w2d_error

  ! W2dInit of include/w2d.h: the set-up of the library's own main-loop
  ! driver (basegrid and the initial conditions of src/initmain.f90)
  type, bind(C) :: w2d_init
    integer(c_int32_t) :: kind, init_levels, startup_admesh, pad_
    real(c_double) :: rho0, p0
    real(c_double) :: e_dep
    real(c_double) :: xc, yc, rb
    real(c_double) :: xh0
    real(c_double) :: extra(8)
  end type w2d_init

  interface
    ! ---- lifecycle (after the allocate()s of src/initmain.f90:76-81) ----
    integer(c_int) function w2d_create(p, ctx) bind(C, name="w2d_create")
      import :: c_int, c_ptr, w2d_params
      type(w2d_params), intent(in) :: p
      type(c_ptr), intent(out) :: ctx
    end function w2d_create

    integer(c_int) function w2d_destroy(ctx) bind(C, name="w2d_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function w2d_destroy

    integer(c_int) function w2d_last_error(ctx, err) bind(C, name="w2d_last_error")
      import :: c_int, c_ptr, w2d_error
      type(c_ptr), value :: ctx
      type(w2d_error), intent(out) :: err
    end function w2d_last_error

    ! the DMC table as src/initmain.f90:83-98 reads it: n rows of
    ! (log10 T, -log10 Lambda)
    integer(c_int) function w2d_set_cooltab(ctx, log_t, neg_log_l, n) bind(C, name="w2d_set_cooltab")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: log_t(*), neg_log_l(*)
      integer(c_int), value :: n
    end function w2d_set_cooltab

    integer(c_int) function w2d_wait_selftest(ctx) bind(C, name="w2d_wait_selftest")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function w2d_wait_selftest

    ! ---- topology: lp, leaf, icoord (src/globals.f90:19-24), dx, dy ----
    integer(c_int) function w2d_set_topology(ctx, lp, ld_lp, leaf, icoord, ld_icoord, nbmax, dx, dy) &
         bind(C, name="w2d_set_topology")
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), intent(in) :: lp(*), leaf(*), icoord(*)
      integer(c_int), value :: ld_lp, ld_icoord, nbmax
      real(c_double), intent(in) :: dx(*), dy(*)
    end function w2d_set_topology

    ! innerbounds(1:ninternal,1:3) of locatebounds (src/locatebounds.f90:29-540)
    integer(c_int) function w2d_set_bounds(ctx, innerbounds, ld, ninternal) bind(C, name="w2d_set_bounds")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), intent(in) :: innerbounds(*)
      integer(c_int), value :: ld, ninternal
    end function w2d_set_bounds

    ! ---- block data ----
    integer(c_int) function w2d_put_blocks(ctx, ids, n, u) bind(C, name="w2d_put_blocks")
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), intent(in) :: ids(*)
      integer(c_int), value :: n
      real(c_double), intent(in) :: u(*)
    end function w2d_put_blocks

    integer(c_int) function w2d_get_blocks(ctx, ids, n, u) bind(C, name="w2d_get_blocks")
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), intent(in) :: ids(*)
      integer(c_int), value :: n
      real(c_double), intent(out) :: u(*)
    end function w2d_get_blocks

    ! u(nbmin:nbmaxtot,neq,-1:18,-1:18) with ld = nbmaxtot-nbmin+1: basegrid
    ! ends with the put, output starts with the get
    integer(c_int) function w2d_put_u_fortran(ctx, u, ld, nbmin, ids, n) bind(C, name="w2d_put_u_fortran")
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: u(*)
      integer(c_int), value :: ld, nbmin, n
      integer(c_int32_t), intent(in) :: ids(*)
    end function w2d_put_u_fortran

    integer(c_int) function w2d_get_u_fortran(ctx, u, ld, nbmin, ids, n) bind(C, name="w2d_get_u_fortran")
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(inout) :: u(*)
      integer(c_int), value :: ld, nbmin, n
      integer(c_int32_t), intent(in) :: ids(*)
    end function w2d_get_u_fortran

    integer(c_int) function w2d_get_primit(ctx, ids, n, prim) bind(C, name="w2d_get_primit")
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), intent(in) :: ids(*)
      integer(c_int), value :: n
      real(c_double), intent(out) :: prim(*)
    end function w2d_get_primit

    ! ---- the per-step block update (src/main.f90:87-98) ----
    ! timestep(dt), src/timestep.f90:7-61; may follow w2d_refine/w2d_coarse
    ! directly (the device rebuilds its leaf list)
    integer(c_int) function w2d_timestep(ctx, dt) bind(C, name="w2d_timestep")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: dt
    end function w2d_timestep

    ! tstep(time,dt), src/tstep.f90:4-126, after the plans of this step
    ! (w2d_set_topology + w2d_set_bounds, or w2d_locate_bounds)
    integer(c_int) function w2d_tstep(ctx, time, dt) bind(C, name="w2d_tstep")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: time, dt
    end function w2d_tstep

    ! criteria, src/criteria.f90:16-50: grad(nb) for nb = 1..nbmax (-1 for
    ! non-leaves)
    integer(c_int) function w2d_criteria(ctx, grad) bind(C, name="w2d_criteria")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: grad(*)
    end function w2d_criteria

    ! ---- the tree's flag loops and locatebounds on the device ----
    ! lp(nb,k) = lp(1 + (nb-1)*row_stride + (k-1)*col_stride); rows =
    ! c_null_ptr sends blocks 1..nbmax, else c_loc of nrows block IDs
    integer(c_int) function w2d_set_links(ctx, lp, row_stride, col_stride, rows, nrows) &
         bind(C, name="w2d_set_links")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), intent(in) :: lp(*)
      integer(c_int), value :: row_stride, col_stride, nrows
      type(c_ptr), value :: rows
    end function w2d_set_links

    integer(c_int) function w2d_admesh_flags(ctx, refine, cap_refine, nrefine, coarsen, cap_coarsen, ncoarsen) &
         bind(C, name="w2d_admesh_flags")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), intent(out) :: refine(*), coarsen(*)
      integer(c_int), value :: cap_refine, cap_coarsen
      integer(c_int), intent(out) :: nrefine, ncoarsen
    end function w2d_admesh_flags

    integer(c_int) function w2d_locate_bounds(ctx) bind(C, name="w2d_locate_bounds")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function w2d_locate_bounds

    ! ---- the u motion of refine / coarse: quads(1:5,k) = (nb|dad, s1..s4) ----
    integer(c_int) function w2d_refine(ctx, quads, n) bind(C, name="w2d_refine")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), intent(in) :: quads(*)
      integer(c_int), value :: n
    end function w2d_refine

    integer(c_int) function w2d_coarse(ctx, quads, n) bind(C, name="w2d_coarse")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), intent(in) :: quads(*)
      integer(c_int), value :: n
    end function w2d_coarse

    ! ---- the routines alone (hosts that split tstep) ----
    integer(c_int) function w2d_boundaryI(ctx, time) bind(C, name="w2d_boundaryI")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: time
    end function w2d_boundaryI

    integer(c_int) function w2d_boundaryII(ctx, time) bind(C, name="w2d_boundaryII")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: time
    end function w2d_boundaryII

    integer(c_int) function w2d_calcprim(ctx) bind(C, name="w2d_calcprim")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function w2d_calcprim

    integer(c_int) function w2d_coolingh(ctx, dt_s) bind(C, name="w2d_coolingh")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: dt_s
    end function w2d_coolingh

    integer(c_int) function w2d_coolingdmc(ctx, dt_s) bind(C, name="w2d_coolingdmc")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: dt_s
    end function w2d_coolingdmc

    integer(c_int) function w2d_sync(ctx) bind(C, name="w2d_sync")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function w2d_sync

    ! ---- the allocation-free time step (no counterpart in the reference):
    ! u and lev are device addresses (c_loc of the device copies, e.g. under
    ! !$acc host_data use_device(u, lev)), dx and dy host arrays
    integer(c_int) function w2d_timestep_noalloc(p, u, lev, nblocks, dx, dy, dt) &
         bind(C, name="w2d_timestep_noalloc")
      import :: c_int, c_ptr, c_double, w2d_params
      type(w2d_params), intent(in) :: p
      type(c_ptr), value :: u, lev
      integer(c_int), value :: nblocks
      real(c_double), intent(in) :: dx(*), dy(*)
      real(c_double), intent(out) :: dt
    end function w2d_timestep_noalloc

    ! ---- one run split by blocks over several GPUs (the -DMPIP build's
    ! counterpart): rank 0 makes the NCCL id, mpi_bcast hands it to all,
    ! every rank creates its part on its GPU and runs the main loop
    integer(c_int) function w2d_part_nccl_id(id, bytes) bind(C, name="w2d_part_nccl_id")
      import :: c_int, c_int8_t
      integer(c_int8_t), intent(out) :: id(*)
      integer(c_int), value :: bytes
    end function w2d_part_nccl_id

    integer(c_int) function w2d_part_create(p, ic, nranks, rank, nccl_id, part) bind(C, name="w2d_part_create")
      import :: c_int, c_int8_t, c_ptr, w2d_params, w2d_init
      type(w2d_params), intent(in) :: p
      type(w2d_init), intent(in) :: ic
      integer(c_int), value :: nranks, rank
      integer(c_int8_t), intent(in) :: nccl_id(*)
      type(c_ptr), intent(out) :: part
    end function w2d_part_create

    integer(c_int) function w2d_part_run(part, nsteps) bind(C, name="w2d_part_run")
      import :: c_int, c_ptr
      type(c_ptr), value :: part
      integer(c_int), value :: nsteps
    end function w2d_part_run

    integer(c_int) function w2d_part_destroy(part) bind(C, name="w2d_part_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: part
    end function w2d_part_destroy
  end interface

  ! the host's one context (w2d_create in initmain)
  type(c_ptr), save :: w2d_ctx = c_null_ptr

end module w2d_iface
