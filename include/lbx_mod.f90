! lbx_mod.f90 -- ISO_C_BINDING interface of include/lbx.h for a Fortran host.
!
! A Fortran driver shaped like LBcuda's `program TestLB` (main.CUF) uses this
! module instead of launching CUDA Fortran kernels on module-global arrays:
!
!   use lbx_mod
!   type(lbx_params) :: p
!   type(c_ptr)      :: ctx
!   call lbx_default_params(p, 128, 128, 128)
!   ierr = lbx_create(p, ctx)
!   ierr = lbx_set_fields(ctx, rhoR, rhoB, vx, vy, vz)   ! setupRho_Pops
!   do step = 1, nIter
!     ierr = lbx_step(ctx, 1)                              ! main.CUF:130-271
!     if (mod(step, nIterVTK) == 0) ierr = lbx_get_fields(ctx, rhoR, rhoB, vel, phase)
!   end do
!   ierr = lbx_destroy(ctx)
!
! Arrays are passed by reference in Fortran order (x fastest), exactly the
! layout of the reference's host arrays rhoR(1:nx,1:ny,1:nz) and
! vel(3,1:nx,1:ny,1:nz) (write_output.f90:975-1041).
module lbx_mod
  use iso_c_binding
  implicit none

  integer(c_int32_t), parameter :: LBX_MODEL_BGK = 0, LBX_MODEL_CG = 1, LBX_MODEL_CG_DIFFDENS = 2
  integer(c_int32_t), parameter :: LBX_MODEL_CG_D3Q27 = 3, LBX_MODEL_CG_DIFFDENS_D3Q27 = 4
  integer(c_int32_t), parameter :: LBX_STORE_F32 = 0, LBX_STORE_F16 = 1, LBX_STORE_BF16 = 2, LBX_STORE_F64 = 3
  integer(c_int32_t), parameter :: LBX_STORE_F16_SD = 4, LBX_STORE_BF16_SD = 5
  integer(c_int32_t), parameter :: LBX_WET_JANUS = 0, LBX_WET_NEUTRAL = 1

  type, bind(C) :: lbx_params
    integer(c_int32_t) :: nx, ny, nz
    integer(c_int32_t) :: model, storage, wetting, lrotate, max_particles
    real(c_float) :: tau, tauR, tauB, sigma, beta, rho0R, rho0B
    real(c_float) :: radius, rmass, max_vel
    real(c_float) :: ext_force(3), ext_torque(3)
    real(c_float) :: hz_k, hz_rmin, hz_rcap
    integer(c_int32_t) :: lubrication
    real(c_float) :: lubric_k, lubric_rmin, lubric_rcap
    integer(c_int32_t) :: kinematic, closure
    real(c_float) :: closure_gap_min, closure_gap_max, closure_vmax
    integer(c_int32_t) :: exact_tiles
    real(c_float) :: densR, densB   ! namelist &fluid (DIFFDENS build)
  end type lbx_params

  interface
    subroutine lbx_default_params(p, nx, ny, nz) bind(C, name="lbx_default_params")
      import :: lbx_params, c_int32_t
      type(lbx_params), intent(out) :: p
      integer(c_int32_t), value :: nx, ny, nz
    end subroutine
    integer(c_int) function lbx_create(p, ctx) bind(C, name="lbx_create")
      import :: lbx_params, c_int, c_ptr
      type(lbx_params), intent(in) :: p
      type(c_ptr), intent(out) :: ctx
    end function
    integer(c_int) function lbx_destroy(ctx) bind(C, name="lbx_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function lbx_set_fields(ctx, rhoR, rhoB, vx, vy, vz) bind(C, name="lbx_set_fields")
      import :: c_int, c_ptr, c_float
      type(c_ptr), value :: ctx
      real(c_float), intent(in) :: rhoR(*), rhoB(*)
      real(c_float), value :: vx, vy, vz
    end function
    integer(c_int) function lbx_set_pops(ctx, popsR, popsB) bind(C, name="lbx_set_pops")
      import :: c_int, c_ptr, c_float
      type(c_ptr), value :: ctx
      real(c_float), intent(in) :: popsR(*), popsB(*)
    end function
    integer(c_int) function lbx_set_particles(ctx, n, xyz, vel, omega, q) bind(C, name="lbx_set_particles")
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: n
      real(c_double), intent(in) :: xyz(*), vel(*), omega(*), q(*)
    end function
    integer(c_int) function lbx_step(ctx, nsteps) bind(C, name="lbx_step")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: nsteps
    end function
    integer(c_int) function lbx_get_fields(ctx, rhoR, rhoB, vel, phase) bind(C, name="lbx_get_fields")
      import :: c_int, c_ptr, c_float
      type(c_ptr), value :: ctx
      real(c_float), intent(out) :: rhoR(*), rhoB(*), vel(*), phase(*)
    end function
    integer(c_int) function lbx_get_pops(ctx, popsR, popsB) bind(C, name="lbx_get_pops")
      import :: c_int, c_ptr, c_float
      type(c_ptr), value :: ctx
      real(c_float), intent(out) :: popsR(*), popsB(*)
    end function
    integer(c_int) function lbx_get_flags(ctx, flags) bind(C, name="lbx_get_flags")
      import :: c_int, c_ptr, c_int8_t
      type(c_ptr), value :: ctx
      integer(c_int8_t), intent(out) :: flags(*)
    end function
    integer(c_int) function lbx_get_links(ctx, cell, dir, sphere, cap, n) bind(C, name="lbx_get_links")
      import :: c_int, c_ptr, c_int8_t, c_int32_t, c_int64_t
      type(c_ptr), value :: ctx
      integer(c_int32_t), intent(out) :: cell(*), sphere(*)
      integer(c_int8_t), intent(out) :: dir(*)
      integer(c_int64_t), value :: cap
      integer(c_int64_t), intent(out) :: n
    end function
    integer(c_int) function lbx_get_particles(ctx, xyz, vel, omega, q, force, torque) bind(C, name="lbx_get_particles")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: xyz(*), vel(*), omega(*), q(*), force(*), torque(*)
    end function
    integer(c_int) function lbx_status(ctx, code, step, where) bind(C, name="lbx_status")
      import :: c_int, c_int32_t, c_int64_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), intent(out) :: code, step
      integer(c_int64_t), intent(out) :: where
    end function
    integer(c_int) function lbx_sync(ctx) bind(C, name="lbx_sync")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    ! z-slab decomposition: an MPI host (one rank per slab, as setupMPI.CUF)
    ! packs its boundary planes into a device buffer, passes it to the
    ! neighbour rank (CUDA-aware MPI or NCCL) and unpacks the received halo
    integer(c_int) function lbx_set_zrange(ctx, zlo, zhi) bind(C, name="lbx_set_zrange")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: zlo, zhi
    end function
    integer(c_int) function lbx_plane_bytes(ctx, nplanes, bytes) bind(C, name="lbx_plane_bytes")
      import :: c_int, c_int32_t, c_int64_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: nplanes
      integer(c_int64_t), intent(out) :: bytes
    end function
    integer(c_int) function lbx_pack_planes(ctx, z0, nplanes, dev_buf) bind(C, name="lbx_pack_planes")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: ctx, dev_buf
      integer(c_int32_t), value :: z0, nplanes
    end function
    integer(c_int) function lbx_unpack_planes(ctx, z0, nplanes, dev_buf) bind(C, name="lbx_unpack_planes")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: ctx, dev_buf
      integer(c_int32_t), value :: z0, nplanes
    end function
    integer(c_int) function lbx_get_stream(ctx, stream) bind(C, name="lbx_get_stream")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      type(c_ptr), intent(out) :: stream
    end function
  end interface
end module lbx_mod
