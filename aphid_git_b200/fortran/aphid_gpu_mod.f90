!======================================================================!
! aphid_gpu_mod.f90 -- ISO_C_BINDING interface to libaphid_gpu.so      !
! (include/aphid_gpu.h) and qmr_gpu, a drop-in for `call qmr` /          !
! `call qmr_mthread` in aphid_main (src/aphid.f90:102-104).             !
!                                                                      !
! qmr_gpu takes the same module data as qmr (module mesh: nx,ny,nz,     !
! dx,dy,dz,dxc,dyc,dzc, k2_*grid, diag_*, rhs_*; module general:        !
! qmr_target, qmr_max_it, pwd, iout), overwrites rhs_* with the         !
! solution, and writes qmr.iter and the stdout summary from the        !
! returned residual history (src/aphid_qmr.f90:161-409).               !
!                                                                      !
! Build (where a Fortran compiler exists):                              !
!   gfortran -c aphid_gpu_mod.f90 (after aphid_mod.f90), link with      !
!   -L<dir> -laphid_gpu -Wl,-rpath,<dir>                                 !
!======================================================================!

      module aphid_gpu
      use iso_c_binding
      implicit none

      integer(c_int), parameter :: APHID_OK = 0
      integer(c_int), parameter :: APHID_CONVERGED = 0
      integer(c_int), parameter :: APHID_MAXIT = 1
      integer(c_int), parameter :: APHID_PREC_FP64 = 0
      integer(c_int), parameter :: APHID_PREC_MIXED = 1
      integer(c_int), parameter :: APHID_PREC_FUSED64 = 2
      integer(c_int), parameter :: APHID_PREC_AUTO = 3

      type, bind(C) :: aphid_opts
        integer(c_int) :: device
        type(c_ptr)    :: stream
        integer(c_int) :: graph_iters
        integer(c_int) :: verbose
        integer(c_int) :: plane_kz
      end type aphid_opts

      type, bind(C) :: aphid_info
        integer(c_int)       :: status, iters, inner_iters, outer_iters
        real(c_double)       :: rhs_norm, recur_resid, true_rel_resid
        real(c_double)       :: seconds
        integer(c_long_long) :: kernel_launches
        integer(c_int)       :: inner64_iters
      end type aphid_info

      ! options of aphid_gpu_sweep (the batched farm of aphid_parallel)
      type, bind(C) :: aphid_sweep_opts
        integer(c_int) :: precision
        real(c_double) :: target
        integer(c_int) :: max_it
        real(c_double) :: inner_tol
        integer(c_int) :: max_outer
        integer(c_int) :: stall_window
        integer(c_int) :: reserved(2)
      end type aphid_sweep_opts

      ! a source of aphid_gpu_sweep_sources: oper_mode 2 / 3 (MT sheet
      ! sources of gen_rhs) or 5 (ndip dipoles, dip_dir "+X".."-Z" and
      ! 1-based tail nodes dip_ijk; c_null_ptr for MT)
      type, bind(C) :: aphid_source
        integer(c_int) :: oper_mode
        integer(c_int) :: ndip
        type(c_ptr)    :: dip_dir
        type(c_ptr)    :: dip_ijk
      end type aphid_source

      interface
        integer(c_int) function aphid_gpu_create(ctx, opts)             &
                       bind(C, name="aphid_gpu_create")
          import :: c_int, c_ptr, aphid_opts
          type(c_ptr), intent(out) :: ctx
          type(aphid_opts), intent(in) :: opts
        end function

        integer(c_int) function aphid_gpu_destroy(ctx)                  &
                       bind(C, name="aphid_gpu_destroy")
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx
        end function

        integer(c_int) function aphid_gpu_set_mesh(ctx, nx, ny, nz,     &
                       dx, dy, dz, dxc, dyc, dzc)                       &
                       bind(C, name="aphid_gpu_set_mesh")
          import :: c_int, c_ptr, c_double
          type(c_ptr), value :: ctx
          integer(c_int), value :: nx, ny, nz
          real(c_double), intent(in) :: dx(*), dy(*), dz(*)
          real(c_double), intent(in) :: dxc(*), dyc(*), dzc(*)
        end function

        integer(c_int) function aphid_gpu_qmr(ctx,                      &
                       k2x, k2y, k2z, k2p, dgx, dgy, dgz, dgp,          &
                       rx, ry, rz, rp, x0x, x0y, x0z, x0p,              &
                       target, max_it, hist, hist_cap, info)            &
                       bind(C, name="aphid_gpu_qmr")
          import :: c_int, c_ptr, c_double, c_double_complex, aphid_info
          type(c_ptr), value :: ctx
          complex(c_double_complex), intent(in) :: k2x(*), k2y(*)
          complex(c_double_complex), intent(in) :: k2z(*), k2p(*)
          complex(c_double_complex), intent(in) :: dgx(*), dgy(*)
          complex(c_double_complex), intent(in) :: dgz(*), dgp(*)
          complex(c_double_complex), intent(inout) :: rx(*), ry(*)
          complex(c_double_complex), intent(inout) :: rz(*), rp(*)
          type(c_ptr), value :: x0x, x0y, x0z, x0p
          real(c_double), value :: target
          integer(c_int), value :: max_it, hist_cap
          real(c_double), intent(out) :: hist(*)
          type(aphid_info), intent(out) :: info
        end function

        ! cell model of a sweep: csig_flag 'R', 'C' or 'I' with the real(4)
        ! cell arrays of read_mesh (c_null_ptr for an absent one)
        integer(c_int) function aphid_gpu_set_model(ctx, csig_flag,     &
                       sig_re, eps_rel)                                 &
                       bind(C, name="aphid_gpu_set_model")
          import :: c_int, c_ptr, c_char
          type(c_ptr), value :: ctx
          character(kind=c_char), value :: csig_flag
          type(c_ptr), value :: sig_re, eps_rel
        end function

        ! every (frequency, source) system of aphid_mpi.freq / .source in
        ! one call: omega(nsys), source_of_system(nsys) (0-based source
        ! index), ndip(nsrc) dipoles per source, dip_dir(2*sum(ndip))
        ! "+X".."-Z", dip_ijk(3*sum(ndip)) 1-based tail nodes; x_out
        ! (nsys concatenated solutions) and x0 may be c_null_ptr
        integer(c_int) function aphid_gpu_sweep(ctx, nsys, omega,        &
                       source_of_system, nsrc, src_ndip, dip_dir,       &
                       dip_ijk, x0, opts, x_out, info)                  &
                       bind(C, name="aphid_gpu_sweep")
          import :: c_int, c_ptr, c_double, c_char, aphid_sweep_opts,   &
                    aphid_info
          type(c_ptr), value :: ctx
          integer(c_int), value :: nsys, nsrc
          real(c_double), intent(in) :: omega(*)
          integer(c_int), intent(in) :: source_of_system(*), src_ndip(*)
          character(kind=c_char), intent(in) :: dip_dir(*)
          integer(c_int), intent(in) :: dip_ijk(*)
          type(c_ptr), value :: x0, x_out
          type(aphid_sweep_opts), intent(in) :: opts
          type(aphid_info), intent(out) :: info(*)
        end function

        ! the same with sources of any kind: the MT farm (aphid_mpi.input
        ! 'MT') passes srcs = [aphid_source(2, ...), aphid_source(3, ...)]
        integer(c_int) function aphid_gpu_sweep_sources(ctx, nsys,      &
                       omega, source_of_system, nsrc, srcs, x0, opts,   &
                       x_out, info)                                     &
                       bind(C, name="aphid_gpu_sweep_sources")
          import :: c_int, c_ptr, c_double, aphid_source,               &
                    aphid_sweep_opts, aphid_info
          type(c_ptr), value :: ctx
          integer(c_int), value :: nsys, nsrc
          real(c_double), intent(in) :: omega(*)
          integer(c_int), intent(in) :: source_of_system(*)
          type(aphid_source), intent(in) :: srcs(*)
          type(c_ptr), value :: x0, x_out
          type(aphid_sweep_opts), intent(in) :: opts
          type(aphid_info), intent(out) :: info(*)
        end function

        ! Cole-Cole cells (csig_flag 'D'): sig_re, eta, tau, cee
        integer(c_int) function aphid_gpu_set_model_cole_cole(ctx,      &
                       sig_re, eta, tau, cee)                           &
                       bind(C, name="aphid_gpu_set_model_cole_cole")
          import :: c_int, c_ptr, c_float
          type(c_ptr), value :: ctx
          real(c_float), intent(in) :: sig_re(*), eta(*), tau(*), cee(*)
        end function

        ! E and H at 1-based interior nodes rec_ijk(3, nrec) for every
        ! system of the last sweep: E, H (3, nrec, nsys)
        integer(c_int) function aphid_gpu_sweep_receivers(ctx, nrec,    &
                       rec_ijk, e, h)                                   &
                       bind(C, name="aphid_gpu_sweep_receivers")
          import :: c_int, c_ptr, c_double_complex
          type(c_ptr), value :: ctx
          integer(c_int), value :: nrec
          integer(c_int), intent(in) :: rec_ijk(*)
          complex(c_double_complex), intent(out) :: e(*), h(*)
        end function
      end interface

      contains

!----------------------------------------------------------------------!
!  Drop-in for `call qmr`: same inputs (module data), same output       !
!  (rhs_* overwritten with the solution), same qmr.iter file.           !
!----------------------------------------------------------------------!
      subroutine qmr_gpu
      use general
      use mesh
      type(c_ptr)       :: ctx
      type(aphid_opts)  :: opts
      type(aphid_info)  :: info
      integer(c_int)    :: rc
      integer           :: i, nh
      real(c_double), allocatable :: hist(:)

      opts%device = 0
      opts%stream = c_null_ptr
      opts%graph_iters = 0
      opts%verbose = 0
      opts%plane_kz = 0
      rc = aphid_gpu_create(ctx, opts)
      if (rc.ne.APHID_OK) then
        write(iout,*) '>> ERROR: no usable GPU for qmr_gpu, code ', rc
        stop
      end if
      rc = aphid_gpu_set_mesh(ctx, nx, ny, nz, dx, dy, dz, dxc, dyc, dzc)
      if (rc.ne.APHID_OK) then
        write(iout,*) '>> ERROR: aphid_gpu_set_mesh failed, code ', rc
        rc = aphid_gpu_destroy(ctx)
        stop
      end if
      allocate(hist(max(1, qmr_max_it)))
      rc = aphid_gpu_qmr(ctx, k2_xgrid, k2_ygrid, k2_zgrid, k2_pgrid,   &
                         diag_x, diag_y, diag_z, diag_p,                &
                         rhs_x, rhs_y, rhs_z, rhs_p,                    &
                         c_null_ptr, c_null_ptr, c_null_ptr, c_null_ptr,&
                         qmr_target, qmr_max_it, hist,                  &
                         int(size(hist), c_int), info)
      if (rc.ne.APHID_OK) then
        write(iout,*) '>> ERROR: aphid_gpu_qmr failed, code ', rc
        stop
      end if

      open(unit=11,file=trim(pwd)//'/qmr.iter',status='unknown')
      nh = min(info%inner_iters, size(hist))
      do i=1,nh
        write(11,*) i, hist(i), info%seconds
      end do
      close(11)

      if (info%status.eq.APHID_CONVERGED) then
        write(iout,*) 'Solution converged in ',info%iters,' iterations'
      else
        write(iout,*) '********** WARNING ************'
        write(iout,*) '  Maximum iterations exceeded  '
        write(iout,*) '*******************************'
      end if
      write(iout,'(a,1x,e11.4)') '   Residual:',info%recur_resid
      write(iout,*) 'Time spent in QMR [s]: ', info%seconds
      write(iout,*) 'Seconds per iteration:    ',                       &
                    info%seconds/real(max(1,info%iters))
      deallocate(hist)
      rc = aphid_gpu_destroy(ctx)
      end subroutine qmr_gpu

      end module aphid_gpu
