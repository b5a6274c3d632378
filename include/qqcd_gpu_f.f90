! qqcd_gpu_f.f90 -- Fortran 2003 (ISO_C_BINDING) binding of the B200 solver library.
!
! Two modules, compiled into the reference's own build (it needs its modules kinds,
! latdims, basics and gmresrhs):
!
!   qqcd_gpu       one bind(C) interface per prototype of qqcd_gpu.h, with the derived
!                  types of the C structs and the status codes;
!   qqcd_gpu_shim  drop-in procedures with the reference's names and argument lists --
!                  Hsingle, Hdouble, Hdbletm (Q/diracops.f90:264-550, 554-599), gmresdr,
!                  psc, bicgstab (Q/inverters.f90:302-487, 2871-3572, 4310-4465) and
!                  fermprop (Q/quark.f90:458-842) -- so a call site needs no edit: only
!                  its `use diracops` / `use inverters` / `use quark` import of these
!                  names changes to `use qqcd_gpu_shim`.  The shim accepts the MPI table
!                  arguments (vecbl, vecblinv, myid, nn, ldiv, nms, lvbc, ib, lbd, iblv,
!                  MRT, MRT2) and validates them against the single-process layout the
!                  GPU library recomputes on the device; it stops with the reference's
!                  kind of message (a `stop`) where the reference would, and on any
!                  library error.
!
! Array arguments are passed as the reference's contiguous real(KR) arrays; the C side
! receives their first element's address.  Opaque handles (qq_ctx, qq_defl, qq_net) are
! type(c_ptr) values.  Output strings of qq_last_error are C strings (qqgpu_last_error
! converts).
module qqcd_gpu
  use, intrinsic :: iso_c_binding
  implicit none
  public

  integer(c_int), parameter :: QQ_OK = 0, QQ_NOT_CONVERGED = 1, QQ_NAN = 2, QQ_BAD_ARG = 3, &
                               QQ_CUDA_ERR = 4, QQ_ABORTED = 5, QQ_NO_DEVICE = 6, QQ_SINGULAR = 7

  type, bind(C) :: qq_geom
    integer(c_int) :: nx, ny, nz, nt
    integer(c_int) :: bc(4)
    real(c_double) :: c1(4)
    real(c_double) :: c2(4)
  end type qq_geom

  type, bind(C) :: qq_solve_info
    integer(c_int) :: status
    integer(c_int) :: itercount
    integer(c_int) :: mvp
    integer(c_int) :: ncycles
    real(c_double) :: true_rel
    real(c_double) :: seconds
    integer(c_int) :: nhist
    real(c_double) :: hist(1024)
    integer(c_int) :: hist_mvp(1024)
    integer(c_int) :: nritz
    real(c_double) :: ritz(1024)
    integer(c_int) :: fallback
    integer(c_int) :: finished_by
    integer(c_int) :: restarts
  end type qq_solve_info

  type, bind(C) :: qq_method
    integer(c_int) :: m, k
    integer(c_int) :: precision
    integer(c_int) :: rhs_block
    real(c_double) :: tol
    integer(c_int) :: max_outer
    integer(c_int) :: solver
    integer(c_int) :: deflate
    real(c_double) :: defl_tol
    integer(c_int) :: stall_window
  end type qq_method

  type, bind(C) :: qq_uneven_group
    type(c_ptr) :: ctx
    integer(c_int) :: nrhs
    real(c_double) :: kappa(2)
    type(c_ptr) :: be
    type(c_ptr) :: bo
    type(c_ptr) :: xe
    type(c_ptr) :: xo
    type(c_ptr) :: infos
  end type qq_uneven_group

  interface
    ! ---- context ----
    function qq_ctx_create(geom, device, out) bind(C, name="qq_ctx_create") result(st)
      import :: c_int, c_ptr, qq_geom
      type(qq_geom), intent(in) :: geom
      integer(c_int), value :: device
      type(c_ptr), intent(out) :: out
      integer(c_int) :: st
    end function qq_ctx_create
    function qq_ctx_destroy(ctx) bind(C, name="qq_ctx_destroy") result(st)
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int) :: st
    end function qq_ctx_destroy
    function qq_ctx_dims(ctx, nvhalf, ntotal) bind(C, name="qq_ctx_dims") result(st)
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), intent(out) :: nvhalf, ntotal
      integer(c_int) :: st
    end function qq_ctx_dims
    function qq_last_error() bind(C, name="qq_last_error") result(msg)
      import :: c_ptr
      type(c_ptr) :: msg
    end function qq_last_error
    function qq_set_coact(ctx, c1, c2) bind(C, name="qq_set_coact") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: c1(4), c2(4)
      integer(c_int) :: st
    end function qq_set_coact

    ! ---- gauge field ----
    function qq_gauge_upload(ctx, u_ref, recon) bind(C, name="qq_gauge_upload") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: u_ref(*)
      integer(c_int), value :: recon
      integer(c_int) :: st
    end function qq_gauge_upload
    function qq_heatbath(ctx, beta, nsweeps, seed, u_ref, plaq) bind(C, name="qq_heatbath") result(st)
      import :: c_int, c_ptr, c_double, c_long_long
      type(c_ptr), value :: ctx
      real(c_double), value :: beta
      integer(c_int), value :: nsweeps
      integer(c_long_long), value :: seed
      real(c_double), intent(out) :: u_ref(*)
      real(c_double), intent(out) :: plaq
      integer(c_int) :: st
    end function qq_heatbath

    ! ---- Dirac operator ----
    function qq_hsingle(ctx, gout, gin, idag, gblclr) bind(C, name="qq_hsingle") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: gout(*)
      real(c_double), intent(in) :: gin(*)
      integer(c_int), value :: idag, gblclr
      integer(c_int) :: st
    end function qq_hsingle
    function qq_hdouble(ctx, he, ge, idag, kappa) bind(C, name="qq_hdouble") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: he(*)
      real(c_double), intent(in) :: ge(*)
      integer(c_int), value :: idag
      real(c_double), value :: kappa
      integer(c_int) :: st
    end function qq_hdouble
    function qq_hdbletm(ctx, he, ge, idag, kappa, iflag) bind(C, name="qq_hdbletm") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: he(*)
      real(c_double), intent(in) :: ge(*)
      integer(c_int), value :: idag
      real(c_double), intent(in) :: kappa(2)
      integer(c_int), value :: iflag
      integer(c_int) :: st
    end function qq_hdbletm
    function qq_twmshift(ctx, hwhole, gwhole, idag, kappa, iflag) bind(C, name="qq_twmshift") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: hwhole(*)
      real(c_double), intent(in) :: gwhole(*)
      integer(c_int), value :: idag
      real(c_double), intent(in) :: kappa(2)
      integer(c_int), value :: iflag
      integer(c_int) :: st
    end function qq_twmshift
    function qq_gamma5mult(ctx, he, ge, idag, kappa, iflag) bind(C, name="qq_gamma5mult") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: he(*)
      real(c_double), intent(in) :: ge(*)
      integer(c_int), value :: idag
      real(c_double), intent(in) :: kappa(2)
      integer(c_int), value :: iflag
      integer(c_int) :: st
    end function qq_gamma5mult
    function qq_vecdot(ctx, a, b, adb) bind(C, name="qq_vecdot") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: a(*), b(*)
      real(c_double), intent(out) :: adb(2)
      integer(c_int) :: st
    end function qq_vecdot
    function qq_vecdot_noalloc(ctx, a, b, adb) bind(C, name="qq_vecdot_noalloc") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: a(*), b(*)
      real(c_double), intent(out) :: adb(2)
      integer(c_int) :: st
    end function qq_vecdot_noalloc

    ! ---- inverters ----
    function qq_defl_create(ctx, nmax, kmax, out) bind(C, name="qq_defl_create") result(st)
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: nmax, kmax
      type(c_ptr), intent(out) :: out
      integer(c_int) :: st
    end function qq_defl_create
    function qq_defl_destroy(d) bind(C, name="qq_defl_destroy") result(st)
      import :: c_int, c_ptr
      type(c_ptr), value :: d
      integer(c_int) :: st
    end function qq_defl_destroy
    function qq_defl_size(d) bind(C, name="qq_defl_size") result(k)
      import :: c_int, c_ptr
      type(c_ptr), value :: d
      integer(c_int) :: k
    end function qq_defl_size
    function qq_defl_vector(d, j, v) bind(C, name="qq_defl_vector") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: d
      integer(c_int), value :: j
      real(c_double), intent(out) :: v(*)
      integer(c_int) :: st
    end function qq_defl_vector
    function qq_gmresdr(ctx, phi, x, GMRES, resmax, itermin, kappa, iflag, defl, info) &
        bind(C, name="qq_gmresdr") result(st)
      import :: c_int, c_ptr, c_double, qq_solve_info
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: phi(*)
      real(c_double), intent(inout) :: x(*)
      integer(c_int), intent(in) :: GMRES(2)
      real(c_double), value :: resmax
      integer(c_int), value :: itermin
      real(c_double), intent(in) :: kappa(2)
      integer(c_int), value :: iflag
      type(c_ptr), value :: defl
      type(qq_solve_info), intent(out) :: info
      integer(c_int) :: st
    end function qq_gmresdr
    function qq_gmresproj(ctx, b, x, GMRES, resmax, itermin, kappa, iflag, defl, info) &
        bind(C, name="qq_gmresproj") result(st)
      import :: c_int, c_ptr, c_double, qq_solve_info
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: b(*)
      real(c_double), intent(inout) :: x(*)
      integer(c_int), intent(in) :: GMRES(2)
      real(c_double), value :: resmax
      integer(c_int), value :: itermin
      real(c_double), intent(in) :: kappa(2)
      integer(c_int), value :: iflag
      type(c_ptr), value :: defl
      type(qq_solve_info), intent(out) :: info
      integer(c_int) :: st
    end function qq_gmresproj
    function qq_psc(ctx, b, x, GMRES, resmax, itermin, kappa, iflag, isignal, defl, info) &
        bind(C, name="qq_psc") result(st)
      import :: c_int, c_ptr, c_double, qq_solve_info
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: b(*)
      real(c_double), intent(inout) :: x(*)
      integer(c_int), intent(in) :: GMRES(2)
      real(c_double), value :: resmax
      integer(c_int), value :: itermin
      real(c_double), intent(in) :: kappa(2)
      integer(c_int), value :: iflag, isignal
      type(c_ptr), value :: defl
      type(qq_solve_info), intent(out) :: info
      integer(c_int) :: st
    end function qq_psc
    function qq_gmresdrshift(ctx, b, xshift, nshifts, sigma, GMRES, resmax, itermin, kappa, iflag, resid, info) &
        bind(C, name="qq_gmresdrshift") result(st)
      import :: c_int, c_ptr, c_double, qq_solve_info
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: b(*)
      real(c_double), intent(out) :: xshift(*)
      integer(c_int), value :: nshifts
      real(c_double), intent(in) :: sigma(*)
      integer(c_int), intent(in) :: GMRES(2)
      real(c_double), value :: resmax
      integer(c_int), value :: itermin
      real(c_double), intent(in) :: kappa(2)
      integer(c_int), value :: iflag
      real(c_double), intent(out) :: resid(*)
      type(qq_solve_info), intent(out) :: info
      integer(c_int) :: st
    end function qq_gmresdrshift
    function qq_bicgstab(ctx, phi, x, resmax, itermin, kappa, iflag, maxiter, info) &
        bind(C, name="qq_bicgstab") result(st)
      import :: c_int, c_ptr, c_double, qq_solve_info
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: phi(*)
      real(c_double), intent(inout) :: x(*)
      real(c_double), value :: resmax
      integer(c_int), value :: itermin
      real(c_double), intent(in) :: kappa(2)
      integer(c_int), value :: iflag, maxiter
      type(qq_solve_info), intent(out) :: info
      integer(c_int) :: st
    end function qq_bicgstab

    ! ---- propagators ----
    function qq_fermprop(ctx, be, bo, kappa, inverter, resmax, itermin, nGMRES, xe, xo, ntmqcd, isignal, defl, &
                         info) bind(C, name="qq_fermprop") result(st)
      import :: c_int, c_ptr, c_double, qq_solve_info
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: be(*), bo(*)
      real(c_double), intent(in) :: kappa(2)
      integer(c_int), value :: inverter
      real(c_double), value :: resmax
      integer(c_int), value :: itermin
      integer(c_int), intent(in) :: nGMRES(2)
      real(c_double), intent(out) :: xe(*), xo(*)
      integer(c_int), value :: ntmqcd, isignal
      type(c_ptr), value :: defl
      type(qq_solve_info), intent(out) :: info
      integer(c_int) :: st
    end function qq_fermprop
    function qq_pointsource(ctx, be, bo, src, icsrc, idsrc) bind(C, name="qq_pointsource") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: be(*), bo(*)
      integer(c_int), intent(in) :: src(4)
      integer(c_int), value :: icsrc, idsrc
      integer(c_int) :: st
    end function qq_pointsource
    function qq_fermprop_batch(ctx, nrhs, be, bo, kappa, method, xe, xo, infos) &
        bind(C, name="qq_fermprop_batch") result(st)
      import :: c_int, c_ptr, c_double, qq_method, qq_solve_info
      type(c_ptr), value :: ctx
      integer(c_int), value :: nrhs
      real(c_double), intent(in) :: be(*), bo(*)
      real(c_double), intent(in) :: kappa(2)
      type(qq_method), intent(in) :: method
      real(c_double), intent(out) :: xe(*), xo(*)
      type(qq_solve_info), intent(out) :: infos(*)
      integer(c_int) :: st
    end function qq_fermprop_batch
    function qq_fermprop_uneven(ngroups, groups, method, concurrent, seconds) &
        bind(C, name="qq_fermprop_uneven") result(st)
      import :: c_int, c_double, qq_method, qq_uneven_group
      integer(c_int), value :: ngroups
      type(qq_uneven_group), intent(in) :: groups(*)
      type(qq_method), intent(in) :: method
      integer(c_int), value :: concurrent
      real(c_double), intent(out) :: seconds
      integer(c_int) :: st
    end function qq_fermprop_uneven

    ! ---- noise sources and loop traces ----
    function qq_initlagfib(myid, iseed) bind(C, name="qq_initlagfib") result(st)
      import :: c_int
      integer(c_int), value :: myid, iseed
      integer(c_int) :: st
    end function qq_initlagfib
    function qq_rnds(m, rn) bind(C, name="qq_rnds") result(st)
      import :: c_int, c_double
      integer(c_int), value :: m
      real(c_double), intent(out) :: rn(*)
      integer(c_int) :: st
    end function qq_rnds
    function qq_z2source(ctx, be, bo) bind(C, name="qq_z2source") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: be(*), bo(*)
      integer(c_int) :: st
    end function qq_z2source
    function qq_z4source(ctx, be, bo) bind(C, name="qq_z4source") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: be(*), bo(*)
      integer(c_int) :: st
    end function qq_z4source
    function qq_twaverage_level0(ctx, be, bo, xe, xo, kappa, delta, dobndry, J) &
        bind(C, name="qq_twaverage_level0") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: be(*), bo(*), xe(*), xo(*)
      real(c_double), value :: kappa, delta
      integer(c_int), value :: dobndry
      real(c_double), intent(out) :: J(*)
      integer(c_int) :: st
    end function qq_twaverage_level0
    function qq_discon_traces(ctx, noise_kind, nnoise, kappa, method, delta, dobndry, J, infos) &
        bind(C, name="qq_discon_traces") result(st)
      import :: c_int, c_ptr, c_double, qq_method, qq_solve_info
      type(c_ptr), value :: ctx
      integer(c_int), value :: noise_kind, nnoise
      real(c_double), intent(in) :: kappa(2)
      type(qq_method), intent(in) :: method
      real(c_double), value :: delta
      integer(c_int), value :: dobndry
      real(c_double), intent(out) :: J(*)
      type(qq_solve_info), intent(out) :: infos(*)
      integer(c_int) :: st
    end function qq_discon_traces
    function qq_twaverage(ctx, be, bo, xe, xo, kappa, delta, io, dobndry, ir, nsub, nmom, nop, Jave) &
        bind(C, name="qq_twaverage") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: be(*), bo(*), xe(*), xo(*)
      real(c_double), value :: kappa, delta
      integer(c_int), intent(in) :: io(3)
      integer(c_int), value :: dobndry, ir, nsub, nmom, nop
      real(c_double), intent(out) :: Jave(*)
      integer(c_int) :: st
    end function qq_twaverage
    function qq_twistdiscon(ctx, noise_kind, nnoise, kappa, method, delta, io, dobndry, ir, nsub, nmom, nop, &
                            Jtotal, Jnoise, infos) bind(C, name="qq_twistdiscon") result(st)
      import :: c_int, c_ptr, c_double, qq_method, qq_solve_info
      type(c_ptr), value :: ctx
      integer(c_int), value :: noise_kind, nnoise
      real(c_double), intent(in) :: kappa(2)
      type(qq_method), intent(in) :: method
      real(c_double), value :: delta
      integer(c_int), intent(in) :: io(3)
      integer(c_int), value :: dobndry, ir, nsub, nmom, nop
      real(c_double), intent(out) :: Jtotal(*), Jnoise(*)
      type(qq_solve_info), intent(out) :: infos(*)
      integer(c_int) :: st
    end function qq_twistdiscon
    function qq_vev(ctx, kappa, io, Jvev, plaq, psi) bind(C, name="qq_vev") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: kappa
      integer(c_int), intent(in) :: io(3)
      real(c_double), intent(out) :: Jvev(*), plaq, psi
      integer(c_int) :: st
    end function qq_vev
    function qq_discon(ctx, noise_kind, nnoise, kappa, method, io, nsub, nmom, nop, Jtotal, Jvev, infos) &
        bind(C, name="qq_discon") result(st)
      import :: c_int, c_ptr, c_double, qq_method, qq_solve_info
      type(c_ptr), value :: ctx
      integer(c_int), value :: noise_kind, nnoise
      real(c_double), value :: kappa
      type(qq_method), intent(in) :: method
      integer(c_int), intent(in) :: io(3)
      integer(c_int), value :: nsub, nmom, nop
      real(c_double), intent(out) :: Jtotal(*), Jvev(*)
      type(qq_solve_info), intent(out) :: infos(*)
      integer(c_int) :: st
    end function qq_discon
    function qq_average(ctx, be, bo, xe, xo, kappa, nsub, nmom, nop, momfac, Jtime) &
        bind(C, name="qq_average") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: be(*), bo(*), xe(*), xo(*)
      real(c_double), value :: kappa
      integer(c_int), value :: nsub, nmom, nop
      real(c_double), intent(in) :: momfac(*)
      real(c_double), intent(out) :: Jtime(*)
      integer(c_int) :: st
    end function qq_average
    function qq_momfacs(dims, io, momfac) bind(C, name="qq_momfacs") result(st)
      import :: c_int, c_double
      integer(c_int), intent(in) :: dims(4), io(3)
      real(c_double), intent(out) :: momfac(*)
      integer(c_int) :: st
    end function qq_momfacs

    function qq_smear(ctx, he, ho, ge, go, asmear, nsmear) bind(C, name="qq_smear") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: he(*), ho(*)
      real(c_double), intent(in) :: ge(*), go(*)
      real(c_double), value :: asmear
      integer(c_int), value :: nsmear
      integer(c_int) :: st
    end function qq_smear
    function qq_mesoncorr(ctx, q, qbar, src, channels, corrRe, corrIm) bind(C, name="qq_mesoncorr") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: q(*), qbar(*)
      integer(c_int), intent(in) :: src(4)
      integer(c_int), value :: channels
      real(c_double), intent(out) :: corrRe(*), corrIm(*)
      integer(c_int) :: st
    end function qq_mesoncorr

    ! ---- eigenmode subtraction of the Wilson loop driver ----
    function qq_eigmodes(ctx, kind, nGMRES, ncycles, kappa, se, so, eig, numEV, evals) &
        bind(C, name="qq_eigmodes") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: kind
      integer(c_int), intent(in) :: nGMRES(2)
      integer(c_int), value :: ncycles
      real(c_double), intent(in) :: kappa(2)
      real(c_double), intent(in) :: se(*), so(*)
      type(c_ptr), intent(out) :: eig
      integer(c_int), intent(out) :: numEV
      real(c_double), intent(out) :: evals(*)
      integer(c_int) :: st
    end function qq_eigmodes
    function qq_eig_destroy(eig) bind(C, name="qq_eig_destroy") result(st)
      import :: c_int, c_ptr
      type(c_ptr), value :: eig
      integer(c_int) :: st
    end function qq_eig_destroy
    function qq_eig_info(eig, kind, numEV, cycles, mvp, evals, ritz) bind(C, name="qq_eig_info") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: eig
      integer(c_int), intent(out) :: kind, numEV, cycles, mvp
      real(c_double), intent(out) :: evals(*), ritz(*)
      integer(c_int) :: st
    end function qq_eig_info
    function qq_eig_vector(eig, j, left, ve, vo) bind(C, name="qq_eig_vector") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: eig
      integer(c_int), value :: j, left
      real(c_double), intent(out) :: ve(*), vo(*)
      integer(c_int) :: st
    end function qq_eig_vector
    function qq_xigenerator(ctx, eig, kappa, xiinv) bind(C, name="qq_xigenerator") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx, eig
      real(c_double), value :: kappa
      real(c_double), intent(out) :: xiinv(*)
      integer(c_int) :: st
    end function qq_xigenerator
    function qq_eigaverage(ctx, eig, ze, zo, kappa, scal, eigstart, eigstep, Jtime) &
        bind(C, name="qq_eigaverage") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx, eig
      real(c_double), intent(in) :: ze(*), zo(*)
      real(c_double), value :: kappa
      real(c_double), intent(in) :: scal(*)
      integer(c_int), value :: eigstart, eigstep
      real(c_double), intent(out) :: Jtime(*)
      integer(c_int) :: st
    end function qq_eigaverage
    function qq_ppcoeffs(ctx, be, bo, kappa, p, co) bind(C, name="qq_ppcoeffs") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: be(*), bo(*)
      real(c_double), value :: kappa
      integer(c_int), value :: p
      real(c_double), intent(out) :: co(*)
      integer(c_int) :: st
    end function qq_ppcoeffs
    function qq_ppaverage(ctx, p, co, be, bo, xe, xo, kappa, nsub, Jtime) bind(C, name="qq_ppaverage") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: p
      real(c_double), intent(in) :: co(*)
      real(c_double), intent(in) :: be(*), bo(*), xe(*), xo(*)
      real(c_double), value :: kappa
      integer(c_int), value :: nsub
      real(c_double), intent(out) :: Jtime(*)
      integer(c_int) :: st
    end function qq_ppaverage
    function qq_xipolygenerator(ctx, eig, kappa, co, xiinv) bind(C, name="qq_xipolygenerator") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx, eig
      real(c_double), value :: kappa
      real(c_double), intent(in) :: co(*)
      real(c_double), intent(out) :: xiinv(*)
      integer(c_int) :: st
    end function qq_xipolygenerator
    function qq_generalaverage(ctx, m, mp, ze, zo, xe, xo, kappa, eigstart, eigstep, co11, co8, co5, copoly, &
        Jave) bind(C, name="qq_generalaverage") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx, m, mp
      real(c_double), intent(in) :: ze(*), zo(*), xe(*), xo(*)
      real(c_double), value :: kappa
      integer(c_int), value :: eigstart, eigstep
      real(c_double), intent(in) :: co11(*), co8(*), co5(*), copoly(*)
      real(c_double), intent(out) :: Jave(*)
      integer(c_int) :: st
    end function qq_generalaverage

    ! ---- file formats ----
    function qq_gfwrite(path, u, nvhalf, ntotal, gaction, beta, alat, tad, icfgsave, myid) &
        bind(C, name="qq_gfwrite") result(st)
      import :: c_int, c_double, c_char
      character(kind=c_char), intent(in) :: path(*)
      real(c_double), intent(inout) :: u(*)
      integer(c_int), value :: nvhalf, ntotal
      integer(c_int), intent(in) :: gaction(4)
      real(c_double), value :: beta
      real(c_double), intent(in) :: alat(4), tad(4)
      integer(c_int), value :: icfgsave, myid
      integer(c_int) :: st
    end function qq_gfwrite
    function qq_gfread(path, u, nvhalf, ntotal, gaction, beta, alat, tad, icfgsave, myid) &
        bind(C, name="qq_gfread") result(st)
      import :: c_int, c_double, c_char
      character(kind=c_char), intent(in) :: path(*)
      real(c_double), intent(out) :: u(*)
      integer(c_int), value :: nvhalf, ntotal
      integer(c_int), intent(out) :: gaction(4)
      real(c_double), intent(out) :: beta
      real(c_double), intent(out) :: alat(4), tad(4)
      integer(c_int), intent(out) :: icfgsave, myid
      integer(c_int) :: st
    end function qq_gfread
    function qq_fpwrite(path, xe, xo, nvhalf, ntotal, kappa, tmqcd, cSW, icsrc, idsrc, icfg, myid) &
        bind(C, name="qq_fpwrite") result(st)
      import :: c_int, c_double, c_char
      character(kind=c_char), intent(in) :: path(*)
      real(c_double), intent(in) :: xe(*), xo(*)
      integer(c_int), value :: nvhalf, ntotal
      real(c_double), value :: kappa, tmqcd, cSW
      integer(c_int), value :: icsrc, idsrc, icfg, myid
      integer(c_int) :: st
    end function qq_fpwrite
    function qq_fpread(path, xe, xo, nvhalf, ntotal, kappa, tmqcd, cSW, icsrc, idsrc, icfg, myid) &
        bind(C, name="qq_fpread") result(st)
      import :: c_int, c_double, c_char
      character(kind=c_char), intent(in) :: path(*)
      real(c_double), intent(out) :: xe(*), xo(*)
      integer(c_int), value :: nvhalf, ntotal
      real(c_double), intent(out) :: kappa, tmqcd, cSW
      integer(c_int), intent(out) :: icsrc, idsrc, icfg, myid
      integer(c_int) :: st
    end function qq_fpread

    ! ---- measurement ----
    function qq_ctx_stream(ctx, stream) bind(C, name="qq_ctx_stream") result(st)
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      type(c_ptr), intent(out) :: stream
      integer(c_int) :: st
    end function qq_ctx_stream
    function qq_launch_count() bind(C, name="qq_launch_count") result(n)
      import :: c_long_long
      integer(c_long_long) :: n
    end function qq_launch_count
    function qq_profile_hop(ctx, enable) bind(C, name="qq_profile_hop") result(st)
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: enable
      integer(c_int) :: st
    end function qq_profile_hop
    function qq_profile_hop_read(ctx, launches, ms_total, bytes_total) bind(C, name="qq_profile_hop_read") result(st)
      import :: c_int, c_ptr, c_double, c_long_long
      type(c_ptr), value :: ctx
      integer(c_long_long), intent(out) :: launches
      real(c_double), intent(out) :: ms_total, bytes_total
      integer(c_int) :: st
    end function qq_profile_hop_read
    function qq_profile_hop_select(ctx, precision, nrhs, launches, ms_total, bytes_total, flops_total) &
        bind(C, name="qq_profile_hop_select") result(st)
      import :: c_int, c_ptr, c_double, c_long_long
      type(c_ptr), value :: ctx
      integer(c_int), value :: precision, nrhs
      integer(c_long_long), intent(out) :: launches
      real(c_double), intent(out) :: ms_total, bytes_total, flops_total
      integer(c_int) :: st
    end function qq_profile_hop_select
    function qq_bench_hsingle(ctx, precision, nrhs, tps, niter, flush_l2, ms_per_call, bytes_per_call) &
        bind(C, name="qq_bench_hsingle") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: precision, nrhs, tps, niter, flush_l2
      real(c_double), intent(out) :: ms_per_call, bytes_per_call
      integer(c_int) :: st
    end function qq_bench_hsingle

    ! ---- local meson correlators, perturbative VEVs ----
    function qq_pionrho(ctx, xe, xo, idsrc, pion, rho, decay) bind(C, name="qq_pionrho") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: xe(*), xo(*)
      integer(c_int), value :: idsrc
      real(c_double), intent(inout) :: pion(*), rho(*), decay(*)
      integer(c_int) :: st
    end function qq_pionrho
    function qq_twvev(ctx, kappa, delta, io, dobndry, ir, nsub, nmom, nop, Jvev) bind(C, name="qq_twvev") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: kappa, delta
      integer(c_int), intent(in) :: io(3)
      integer(c_int), value :: dobndry, ir, nsub, nmom, nop
      real(c_double), intent(out) :: Jvev(*)
      integer(c_int) :: st
    end function qq_twvev

    ! ---- learned preconditioner ----
    function qq_net_create(nlayers, channels, seed, scale, out) bind(C, name="qq_net_create") result(st)
      import :: c_int, c_ptr, c_double, c_long_long
      integer(c_int), value :: nlayers
      integer(c_int), intent(in) :: channels(*)
      integer(c_long_long), value :: seed
      real(c_double), value :: scale
      type(c_ptr), intent(out) :: out
      integer(c_int) :: st
    end function qq_net_create
    function qq_net_destroy(net) bind(C, name="qq_net_destroy") result(st)
      import :: c_int, c_ptr
      type(c_ptr), value :: net
      integer(c_int) :: st
    end function qq_net_destroy
    function qq_net_nweights(net) bind(C, name="qq_net_nweights") result(n)
      import :: c_int, c_ptr
      type(c_ptr), value :: net
      integer(c_int) :: n
    end function qq_net_nweights
    function qq_net_get_weights(net, w) bind(C, name="qq_net_get_weights") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: net
      real(c_double), intent(out) :: w(*)
      integer(c_int) :: st
    end function qq_net_get_weights
    function qq_net_set_weights(net, w) bind(C, name="qq_net_set_weights") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: net
      real(c_double), intent(in) :: w(*)
      integer(c_int) :: st
    end function qq_net_set_weights
    function qq_net_apply(ctx, net, in, out) bind(C, name="qq_net_apply") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx, net
      real(c_double), intent(in) :: in(*)
      real(c_double), intent(out) :: out(*)
      integer(c_int) :: st
    end function qq_net_apply
    function qq_net_grad(ctx, net, nsamples, b, x, loss, grad) bind(C, name="qq_net_grad") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx, net
      integer(c_int), value :: nsamples
      real(c_double), intent(in) :: b(*), x(*)
      real(c_double), intent(out) :: loss
      real(c_double), intent(out) :: grad(*)
      integer(c_int) :: st
    end function qq_net_grad
    function qq_net_train(ctx, net, kappa, nsamples, nsteps, lr, seed, losses) bind(C, name="qq_net_train") result(st)
      import :: c_int, c_ptr, c_double, c_long_long
      type(c_ptr), value :: ctx, net
      real(c_double), intent(in) :: kappa(2)
      integer(c_int), value :: nsamples, nsteps
      real(c_double), value :: lr
      integer(c_long_long), value :: seed
      real(c_double), intent(out) :: losses(*)
      integer(c_int) :: st
    end function qq_net_train
    function qq_net_train_pairs(ctx, net, nsamples, b, x, nsteps, lr, losses) &
        bind(C, name="qq_net_train_pairs") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx, net
      integer(c_int), value :: nsamples
      real(c_double), intent(in) :: b(*), x(*)
      integer(c_int), value :: nsteps
      real(c_double), value :: lr
      real(c_double), intent(out) :: losses(*)
      integer(c_int) :: st
    end function qq_net_train_pairs
    function qq_fgmres(ctx, net, phi, x, m, resmax, max_cycles, kappa, info) bind(C, name="qq_fgmres") result(st)
      import :: c_int, c_ptr, c_double, qq_solve_info
      type(c_ptr), value :: ctx, net
      real(c_double), intent(in) :: phi(*)
      real(c_double), intent(inout) :: x(*)
      integer(c_int), value :: m
      real(c_double), value :: resmax
      integer(c_int), value :: max_cycles
      real(c_double), intent(in) :: kappa(2)
      type(qq_solve_info), intent(out) :: info
      integer(c_int) :: st
    end function qq_fgmres
    function qq_fgmresdr(ctx, net, phi, x, GMRES, resmax, max_cycles, kappa, info) &
        bind(C, name="qq_fgmresdr") result(st)
      import :: c_int, c_ptr, c_double, qq_solve_info
      type(c_ptr), value :: ctx, net
      real(c_double), intent(in) :: phi(*)
      real(c_double), intent(inout) :: x(*)
      integer(c_int), intent(in) :: GMRES(2)
      real(c_double), value :: resmax
      integer(c_int), value :: max_cycles
      real(c_double), intent(in) :: kappa(2)
      type(qq_solve_info), intent(out) :: info
      integer(c_int) :: st
    end function qq_fgmresdr

    ! ---- kernel shapes ----
    function qq_hop_tuned_shape(ctx, precision, nrhs, shape) bind(C, name="qq_hop_tuned_shape") result(st)
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: precision, nrhs
      integer(c_int), intent(out) :: shape
      integer(c_int) :: st
    end function qq_hop_tuned_shape
    function qq_hsingle_block(ctx, precision, nrhs, shape, gout, gin, idag, gblclr) &
        bind(C, name="qq_hsingle_block") result(st)
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: precision, nrhs, shape
      real(c_double), intent(out) :: gout(*)
      real(c_double), intent(in) :: gin(*)
      integer(c_int), value :: idag, gblclr
      integer(c_int) :: st
    end function qq_hsingle_block
  end interface

contains

  ! The text of qq_last_error as a Fortran string.
  function qqgpu_last_error() result(msg)
    character(len=512) :: msg
    character(kind=c_char), pointer :: p(:)
    type(c_ptr) :: cp
    integer :: i
    msg = ""
    cp = qq_last_error()
    if (.not. c_associated(cp)) return
    call c_f_pointer(cp, p, [512])
    do i = 1, 512
      if (p(i) == c_null_char) exit
      msg(i:i) = p(i)
    end do
  end function qqgpu_last_error
end module qqcd_gpu


! ---------------------------------------------------------------------------------------
! The reference's procedure names and argument lists on the GPU library.  One library
! context per process, created on first use from latdims (nx, ny, nz, nt), bc and coact;
! the gauge field is uploaded on first use and again whenever the caller passes a
! different u (its address, or a sample of its entries, changed).
module qqcd_gpu_shim
  use, intrinsic :: iso_c_binding
  use kinds
  use latdims
  use basics
  use gmresrhs, only: isignal
  use qqcd_gpu
  implicit none
  private
  public :: Hsingle, Hdouble, Hdbletm, gmresdr, psc, bicgstab, fermprop, qqgpu_finalize

  type(c_ptr), save :: qqctx = c_null_ptr
  type(c_ptr), save :: qqdefl = c_null_ptr
  integer(c_intptr_t), save :: u_addr = 0
  real(c_double), save :: u_sig = 0.0_c_double
  real(c_double), save :: cur_c1(4) = 0.0_c_double, cur_c2(4) = 0.0_c_double

contains

  ! Stop with the library's message, as the reference stops on an argument error.
  subroutine qqgpu_check(st, what)
    integer(c_int), intent(in) :: st
    character(len=*), intent(in) :: what
    if (st == QQ_OK .or. st == QQ_NOT_CONVERGED) return
    write(*, "(a, a, a, i0, a, a)") "qqcd_gpu ", what, ": status ", st, " ", trim(qqgpu_last_error())
    stop
  end subroutine qqgpu_check

  ! The MPI tables of the reference describe a single process here (nps = 1): the GPU
  ! library holds the whole lattice and recomputes neighbours and blocks on the device.
  ! Reject anything else instead of computing on a different decomposition.
  subroutine qqgpu_validate(gin, bc, vecbl, vecblinv, myid, nn, ldiv, nms, lvbc, ib, lbd, iblv)
    real(kind=KR), intent(in), dimension(:,:,:,:,:) :: gin
    integer(kind=KI), intent(in), dimension(:) :: bc, nms
    integer(kind=KI), intent(in), dimension(:,:) :: vecbl, vecblinv, nn, iblv
    integer(kind=KI), intent(in) :: myid
    logical, intent(in), dimension(:) :: ldiv
    integer(kind=KI), intent(in), dimension(:,:,:) :: lvbc
    integer(kind=KI), intent(in), dimension(:,:,:,:) :: ib
    logical, intent(in), dimension(:,:) :: lbd
    integer(kind=KI), parameter :: even(8) = [1, 4, 6, 7, 10, 11, 13, 16]
    integer(kind=KI) :: mu, i
    if (nps /= 1 .or. myid /= 0) then
      write(*, *) "qqcd_gpu: one process per lattice (nps = 1, myid = 0) required"
      stop
    end if
    if (size(gin, 1) /= 6 .or. size(gin, 2) /= ntotal .or. size(gin, 3) /= 4 .or. size(gin, 4) /= 2 .or. &
        size(gin, 5) /= 8) then
      write(*, *) "qqcd_gpu: Dirac vector is not g(6,ntotal,4,2,8)"
      stop
    end if
    if (size(bc) < 4 .or. size(nms) < 4 .or. size(ldiv) < 4 .or. size(vecbl, 2) < 8 .or. size(vecblinv, 2) < 16 &
        .or. size(nn, 1) < 4 .or. size(iblv, 1) < 16 .or. size(lbd, 1) < 16 .or. size(lvbc, 1) < nvhalf .or. &
        size(ib, 1) < 1) then
      write(*, *) "qqcd_gpu: MPI tables have the wrong shape"
      stop
    end if
    do i = 1, 8
      if (vecbl(1, i) /= even(i)) then
        write(*, *) "qqcd_gpu: vecbl is not the reference's global checkerboard"
        stop
      end if
    end do
    do mu = 1, 4
      if (ldiv(mu)) then
        write(*, *) "qqcd_gpu: the lattice is divided among processes (ldiv)"
        stop
      end if
      if (bc(mu) < -1 .or. bc(mu) > 1) then
        write(*, *) "qqcd_gpu: bc must be 1, -1 or 0"
        stop
      end if
    end do
  end subroutine qqgpu_validate

  ! Create the context on first use, keep coact and the gauge field current.
  subroutine qqgpu_prepare(u, coact, bc)
    real(kind=KR), intent(in), dimension(:,:,:,:,:), target :: u
    real(kind=KR), intent(in), dimension(:,:,:) :: coact
    integer(kind=KI), intent(in), dimension(:) :: bc
    type(qq_geom) :: geom
    real(c_double) :: c1(4), c2(4), sig
    integer(c_intptr_t) :: addr
    integer :: mu, i, n
    real(kind=KR), pointer :: flat(:)
    do mu = 1, 4
      c1(mu) = coact(3, 1, mu)
      c2(mu) = coact(3, 2, mu)
    end do
    if (.not. c_associated(qqctx)) then
      geom%nx = nx
      geom%ny = ny
      geom%nz = nz
      geom%nt = nt
      geom%bc = int(bc(1:4), c_int)
      geom%c1 = c1
      geom%c2 = c2
      call qqgpu_check(qq_ctx_create(geom, 0_c_int, qqctx), "ctx_create")
      cur_c1 = c1
      cur_c2 = c2
    else if (any(c1 /= cur_c1) .or. any(c2 /= cur_c2)) then
      call qqgpu_check(qq_set_coact(qqctx, c1, c2), "set_coact")
      cur_c1 = c1
      cur_c2 = c2
    end if
    n = size(u)
    call c_f_pointer(c_loc(u), flat, [n])
    sig = 0.0_c_double
    do i = 1, n, max(1, n / 64)
      sig = sig + real(i, c_double) * flat(i)
    end do
    addr = transfer(c_loc(u), addr)
    if (addr /= u_addr .or. sig /= u_sig) then
      call qqgpu_check(qq_gauge_upload(qqctx, flat, 0_c_int), "gauge_upload")
      u_addr = addr
      u_sig = sig
    end if
  end subroutine qqgpu_prepare

  subroutine qqgpu_finalize()
    integer(c_int) :: st
    if (c_associated(qqdefl)) st = qq_defl_destroy(qqdefl)
    if (c_associated(qqctx)) st = qq_ctx_destroy(qqctx)
    qqdefl = c_null_ptr
    qqctx = c_null_ptr
    u_addr = 0
  end subroutine qqgpu_finalize

  ! Hsingle Q/diracops.f90:554-599
  subroutine Hsingle(gout, u, gin, idag, coact, bc, gblclr, vecbl, vecblinv, myid, nn, ldiv, nms, lvbc, ib, lbd, &
                     iblv, MRT)
    real(kind=KR), intent(out), dimension(:,:,:,:,:) :: gout
    real(kind=KR), intent(in), dimension(:,:,:,:,:), target :: u
    real(kind=KR), intent(inout), dimension(:,:,:,:,:) :: gin
    integer(kind=KI), intent(in), dimension(:) :: bc, nms
    integer(kind=KI), intent(in) :: idag, gblclr, myid, MRT
    real(kind=KR), intent(in), dimension(:,:,:) :: coact
    integer(kind=KI), intent(in), dimension(:,:) :: vecbl, vecblinv
    integer(kind=KI), intent(in), dimension(:,:) :: nn, iblv
    logical, intent(in), dimension(:) :: ldiv
    integer(kind=KI), intent(in), dimension(:,:,:) :: lvbc
    integer(kind=KI), intent(in), dimension(:,:,:,:) :: ib
    logical, intent(in), dimension(:,:) :: lbd
    call qqgpu_validate(gin, bc, vecbl, vecblinv, myid, nn, ldiv, nms, lvbc, ib, lbd, iblv)
    call qqgpu_prepare(u, coact, bc)
    call qqgpu_check(qq_hsingle(qqctx, gout, gin, int(idag, c_int), int(gblclr, c_int)), "Hsingle")
  end subroutine Hsingle

  ! Hdouble Q/diracops.f90:264-346
  subroutine Hdouble(he, u, ge, idag, coact, kappa, bc, vecbl, vecblinv, myid, nn, ldiv, nms, lvbc, ib, lbd, iblv, &
                     MRT)
    real(kind=KR), intent(out), dimension(:,:,:,:,:) :: he
    real(kind=KR), intent(in), dimension(:,:,:,:,:), target :: u
    real(kind=KR), intent(inout), dimension(:,:,:,:,:) :: ge
    integer(kind=KI), intent(in) :: idag, myid, MRT
    real(kind=KR), intent(in), dimension(:,:,:) :: coact
    real(kind=KR), intent(in) :: kappa
    integer(kind=KI), intent(in), dimension(:) :: bc, nms
    integer(kind=KI), intent(in), dimension(:,:) :: vecbl, vecblinv, nn, iblv
    logical, intent(in), dimension(:) :: ldiv
    integer(kind=KI), intent(in), dimension(:,:,:) :: lvbc
    integer(kind=KI), intent(in), dimension(:,:,:,:) :: ib
    logical, intent(in), dimension(:,:) :: lbd
    call qqgpu_validate(ge, bc, vecbl, vecblinv, myid, nn, ldiv, nms, lvbc, ib, lbd, iblv)
    call qqgpu_prepare(u, coact, bc)
    call qqgpu_check(qq_hdouble(qqctx, he, ge, int(idag, c_int), real(kappa, c_double)), "Hdouble")
  end subroutine Hdouble

  ! Hdbletm Q/diracops.f90:435-550 (iflag = -1; the clover branch stops)
  subroutine Hdbletm(he, u, GeeGooinv, ge, idag, coact, kappa, iflag, bc, vecbl, vecblinv, myid, nn, ldiv, nms, &
                     lvbc, ib, lbd, iblv, MRT)
    real(kind=KR), intent(out), dimension(:,:,:,:,:) :: he
    real(kind=KR), intent(in), dimension(:,:,:,:,:), target :: u
    real(kind=KR), intent(in), dimension(:,:,:,:,:) :: GeeGooinv
    real(kind=KR), intent(inout), dimension(:,:,:,:,:) :: ge
    integer(kind=KI), intent(in) :: idag, iflag, myid, MRT
    real(kind=KR), intent(in), dimension(:,:,:) :: coact
    real(kind=KR), intent(in), dimension(:) :: kappa
    integer(kind=KI), intent(in), dimension(:) :: bc, nms
    integer(kind=KI), intent(in), dimension(:,:) :: vecbl, vecblinv, nn, iblv
    logical, intent(in), dimension(:) :: ldiv
    integer(kind=KI), intent(in), dimension(:,:,:) :: lvbc
    integer(kind=KI), intent(in), dimension(:,:,:,:) :: ib
    logical, intent(in), dimension(:,:) :: lbd
    real(c_double) :: k2(2)
    call qqgpu_validate(ge, bc, vecbl, vecblinv, myid, nn, ldiv, nms, lvbc, ib, lbd, iblv)
    call qqgpu_prepare(u, coact, bc)
    k2 = real(kappa(1:2), c_double)
    call qqgpu_check(qq_hdbletm(qqctx, he, ge, int(idag, c_int), k2, int(iflag, c_int)), "Hdbletm")
  end subroutine Hdbletm

  ! gmresdr Q/inverters.f90:2871-3572 (the deflation space is kept for psc)
  subroutine gmresdr(rwdir, phi, x, GMRES, resmax, itermin, itercount, u, GeeGooinv, iflag, kappa, coact, bc, &
                     vecbl, vecblinv, myid, nn, ldiv, nms, lvbc, ib, lbd, iblv, MRT, MRT2)
    character(len=*), intent(in), dimension(:) :: rwdir
    real(kind=KR), intent(in), dimension(:,:,:,:,:) :: phi
    real(kind=KR), intent(inout), dimension(:,:,:,:,:) :: x
    integer(kind=KI), intent(in), dimension(:) :: GMRES, bc, nms
    integer(kind=KI), intent(in) :: itermin, iflag, myid, MRT, MRT2
    real(kind=KR), intent(in) :: resmax
    integer(kind=KI), intent(out) :: itercount
    real(kind=KR), intent(in), dimension(:,:,:,:,:), target :: u
    real(kind=KR), intent(in), dimension(:,:,:,:,:) :: GeeGooinv
    real(kind=KR), intent(in), dimension(:) :: kappa
    real(kind=KR), intent(in), dimension(:,:,:) :: coact
    integer(kind=KI), intent(in), dimension(:,:) :: vecbl, vecblinv, nn, iblv
    logical, intent(in), dimension(:) :: ldiv
    integer(kind=KI), intent(in), dimension(:,:,:) :: lvbc
    integer(kind=KI), intent(in), dimension(:,:,:,:) :: ib
    logical, intent(in), dimension(:,:) :: lbd
    type(qq_solve_info) :: info
    integer(c_int) :: g2(2)
    real(c_double) :: k2(2)
    call qqgpu_validate(x, bc, vecbl, vecblinv, myid, nn, ldiv, nms, lvbc, ib, lbd, iblv)
    call qqgpu_prepare(u, coact, bc)
    call qqgpu_defl(GMRES)
    g2 = int(GMRES(1:2), c_int)
    k2 = real(kappa(1:2), c_double)
    call qqgpu_check(qq_gmresdr(qqctx, phi, x, g2, real(resmax, c_double), int(itermin, c_int), k2, &
                                int(iflag, c_int), qqdefl, info), "gmresdr")
    itercount = info%itercount
  end subroutine gmresdr

  ! psc Q/inverters.f90:4310-4465: isignal from the reference's gmresrhs module
  subroutine psc(rwdir, b, x, GMRES, resmax, itermin, itercount, u, GeeGooinv, iflag, kappa, coact, bc, vecbl, &
                 vecblinv, myid, nn, ldiv, nms, lvbc, ib, lbd, iblv, MRT, MRT2)
    character(len=*), intent(in), dimension(:) :: rwdir
    real(kind=KR), intent(in), dimension(:,:,:,:,:) :: b
    real(kind=KR), intent(inout), dimension(:,:,:,:,:) :: x
    integer(kind=KI), intent(in), dimension(:) :: GMRES, bc, nms
    integer(kind=KI), intent(in) :: itermin, iflag, myid, MRT, MRT2
    real(kind=KR), intent(in) :: resmax
    integer(kind=KI), intent(out) :: itercount
    real(kind=KR), intent(in), dimension(:,:,:,:,:), target :: u
    real(kind=KR), intent(in), dimension(:,:,:,:,:) :: GeeGooinv
    real(kind=KR), intent(in), dimension(:) :: kappa
    real(kind=KR), intent(in), dimension(:,:,:) :: coact
    integer(kind=KI), intent(in), dimension(:,:) :: vecbl, vecblinv, nn, iblv
    logical, intent(in), dimension(:) :: ldiv
    integer(kind=KI), intent(in), dimension(:,:,:) :: lvbc
    integer(kind=KI), intent(in), dimension(:,:,:,:) :: ib
    logical, intent(in), dimension(:,:) :: lbd
    type(qq_solve_info) :: info
    integer(c_int) :: g2(2)
    real(c_double) :: k2(2)
    call qqgpu_validate(x, bc, vecbl, vecblinv, myid, nn, ldiv, nms, lvbc, ib, lbd, iblv)
    call qqgpu_prepare(u, coact, bc)
    call qqgpu_defl(GMRES)
    g2 = int(GMRES(1:2), c_int)
    k2 = real(kappa(1:2), c_double)
    call qqgpu_check(qq_psc(qqctx, b, x, g2, real(resmax, c_double), int(itermin, c_int), k2, int(iflag, c_int), &
                            int(isignal, c_int), qqdefl, info), "psc")
    itercount = info%itercount
  end subroutine psc

  ! bicgstab Q/inverters.f90:302-487
  subroutine bicgstab(rwdir, phi, x, resmax, itermin, itercount, u, GeeGooinv, iflag, kappa, coact, bc, vecbl, &
                      vecblinv, myid, nn, ldiv, nms, lvbc, ib, lbd, iblv, MRT, MRT2)
    character(len=*), intent(in), dimension(:) :: rwdir
    real(kind=KR), intent(in), dimension(:,:,:,:,:) :: phi
    real(kind=KR), intent(inout), dimension(:,:,:,:,:) :: x
    real(kind=KR), intent(in) :: resmax
    integer(kind=KI), intent(in) :: itermin, iflag, myid, MRT, MRT2
    integer(kind=KI), intent(out) :: itercount
    real(kind=KR), intent(in), dimension(:,:,:,:,:), target :: u
    real(kind=KR), intent(in), dimension(:,:,:,:,:) :: GeeGooinv
    real(kind=KR), intent(in), dimension(:) :: kappa
    real(kind=KR), intent(in), dimension(:,:,:) :: coact
    integer(kind=KI), intent(in), dimension(:) :: bc, nms
    integer(kind=KI), intent(in), dimension(:,:) :: vecbl, vecblinv, nn, iblv
    logical, intent(in), dimension(:) :: ldiv
    integer(kind=KI), intent(in), dimension(:,:,:) :: lvbc
    integer(kind=KI), intent(in), dimension(:,:,:,:) :: ib
    logical, intent(in), dimension(:,:) :: lbd
    type(qq_solve_info) :: info
    real(c_double) :: k2(2)
    call qqgpu_validate(x, bc, vecbl, vecblinv, myid, nn, ldiv, nms, lvbc, ib, lbd, iblv)
    call qqgpu_prepare(u, coact, bc)
    k2 = real(kappa(1:2), c_double)
    call qqgpu_check(qq_bicgstab(qqctx, phi, x, real(resmax, c_double), int(itermin, c_int), k2, &
                                 int(iflag, c_int), 0_c_int, info), "bicgstab")
    itercount = info%itercount
  end subroutine bicgstab

  ! fermprop Q/quark.f90:458-842 for nkappa = -1 (Wilson / twisted mass, cSW = 0): the
  ! reference passes nGMRES = (vectype, kGMRES) to its inverters (:545-547); inverters 0
  ! (bicgstab), 5 (gmresdr) and 6 (psc, isignal from gmresrhs) run on the GPU.
  subroutine fermprop(rwdir, be, bo, nkappa, kappa, cSW, inverter, coact, bc, resmax, itermin, omegaM3R, u, &
                      vectype, kGMRES, xe, xo, myid, nn, ldiv, nms, lvbc, lvcl, ib, lbd, iblv, vecbl, vecblinv, &
                      ntmqcd, hoption, MRT, MRT2)
    character(len=*), intent(in), dimension(:) :: rwdir
    real(kind=KR), intent(in), dimension(:,:,:,:,:) :: be
    real(kind=KR), intent(inout), dimension(:,:,:,:,:) :: bo
    integer(kind=KI), intent(in) :: nkappa, hoption, inverter, kGMRES
    real(kind=KR), intent(in), dimension(:) :: kappa
    real(kind=KR), intent(in) :: cSW, resmax
    real(kind=KR), intent(in), dimension(:,:,:) :: coact
    integer(kind=KI), intent(in) :: ntmqcd
    integer(kind=KI), intent(in), dimension(:) :: bc, nms
    integer(kind=KI), intent(in) :: itermin, myid, MRT, MRT2
    real(kind=KR2), intent(in) :: omegaM3R
    real(kind=KR), intent(inout), dimension(:,:,:,:,:), target :: u
    integer(kind=KI), intent(inout) :: vectype
    real(kind=KR), intent(inout), dimension(:,:,:,:,:,:) :: xe, xo
    integer(kind=KI), intent(in), dimension(:,:) :: nn, iblv, vecbl, vecblinv
    logical, intent(in), dimension(:) :: ldiv
    integer(kind=KI), intent(in), dimension(:,:,:) :: lvbc, lvcl
    integer(kind=KI), intent(in), dimension(:,:,:,:) :: ib
    logical, intent(in), dimension(:,:) :: lbd
    type(qq_solve_info) :: info
    integer(c_int) :: g2(2)
    real(c_double) :: k2(2)
    if (nkappa /= -1) then
      write(*, *) "qqcd_gpu: fermprop supports nkappa = -1 (Wilson / twisted mass) only"
      stop
    end if
    if (inverter /= 0 .and. inverter /= 5 .and. inverter /= 6) then
      write(*, *) "qqcd_gpu: fermprop supports inverter 0, 5 and 6"
      stop
    end if
    call qqgpu_validate(be, bc, vecbl, vecblinv, myid, nn, ldiv, nms, lvbc, ib, lbd, iblv)
    call qqgpu_prepare(u, coact, bc)
    g2(1) = int(vectype, c_int)
    g2(2) = int(kGMRES, c_int)
    if (inverter /= 0) call qqgpu_defl(g2)
    k2 = real(kappa(1:2), c_double)
    call qqgpu_check(qq_fermprop(qqctx, be, bo, k2, int(inverter, c_int), real(resmax, c_double), &
                                 int(itermin, c_int), g2, xe(:,:,:,:,:,1), xo(:,:,:,:,:,1), int(ntmqcd, c_int), &
                                 int(isignal, c_int), qqdefl, info), "fermprop")
  end subroutine fermprop

  ! The deflation handle that replaces the shift module's vtemp / hcnew / beg.
  ! Sized like the reference's shift module (nmaxGMRES, kmaxGMRES of latdims), and at
  ! least as large as this call's GMRES(n, k).
  subroutine qqgpu_defl(GMRES)
    integer, intent(in), dimension(:) :: GMRES
    integer :: nmax, kmax
    if (c_associated(qqdefl)) return
    nmax = max(GMRES(1), nmaxGMRES, 2)
    kmax = max(1, min(nmax - 1, max(GMRES(2), kmaxGMRES)))
    call qqgpu_check(qq_defl_create(qqctx, int(nmax, c_int), int(kmax, c_int), qqdefl), "defl_create")
  end subroutine qqgpu_defl
end module qqcd_gpu_shim
