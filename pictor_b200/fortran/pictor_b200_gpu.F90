! pictor_b200_gpu.F90 -- ISO_C_BINDING shim that lets PICTOR's unchanged
! MAIN.F90 drive libpictor_b200.so.  Build PICTOR with -Dgpu and this file in
! place of the CUDA Fortran sources of src/movdep, src/maxwell, src/mem,
! src/init/initialise_gpu.F90 and src/comm/comm_fld_gpu.F90: it provides the
! modules MAIN.F90 uses under `#ifdef gpu` (MAIN.F90:20-28) and the
! argument-less subroutines it calls (MAIN.F90:53-55, 67-69, 91-93, 113-116,
! 128-130, 161-163, 173-175, 189-191, 223-233, 250-252, 263-265).
!
! State stays in the reference's module globals (vars.F90); the library owns
! the device copies.  Host arrays move only in InitAll_gpu and at output
! steps (CopyGPUDataToHostForOutput), as in src/mem/particles_gpu.F90:569-581.

module pictor_b200_capi
   use iso_c_binding
   implicit none

   integer(c_int), parameter :: PIC_MAX_FLVR = 15

   type, bind(C) :: pic_config
      integer(c_int32_t) :: nx, ny, nz, dims, geom, fdtd, precision, nflvr
      real(c_double) :: c, qi, bext(3), qm(0:PIC_MAX_FLVR)
      integer(c_int32_t) :: reorder_period, curr_filter
      integer(c_int64_t) :: capacity
      real(c_double) :: rmin
      integer(c_int32_t) :: inc_axis, brick(3), cyl_modes, slab_x, exact_current, fp64_tiles, exact_charge, &
                            reserved(3)
   end type pic_config

   ! pic_inflow: one 'iflw' face's injection (bc_inflow.F90) with a uniform
   ! density and drift, up to four phase-space properties
   type, bind(C) :: pic_inflow_t
      integer(c_int32_t) :: face
      real(c_double)     :: pos, speed, vmax, epc, density, drift(3)
      integer(c_int32_t) :: nspecies, flv(4)
      real(c_double)     :: temp(4), charge(4)
      integer(c_int32_t) :: seed, call
   end type pic_inflow_t

   interface
      integer(c_int) function pic_create(cfg, h) bind(C, name="pic_create")
         import :: c_int, c_ptr, pic_config
         type(pic_config), intent(in) :: cfg
         type(c_ptr), intent(out) :: h
      end function
      subroutine pic_destroy(h) bind(C, name="pic_destroy")
         import :: c_ptr
         type(c_ptr), value :: h
      end subroutine
      integer(c_int) function pic_load_fields(h, ex, ey, ez, bx, by, bz) bind(C, name="pic_load_fields")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: h
         real(c_double), intent(in) :: ex(*), ey(*), ez(*), bx(*), by(*), bz(*)
      end function
      integer(c_int) function pic_fetch_fields(h, ex, ey, ez, bx, by, bz, jx, jy, jz) bind(C, name="pic_fetch_fields")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: h
         real(c_double), intent(out) :: ex(*), ey(*), ez(*), bx(*), by(*), bz(*), jx(*), jy(*), jz(*)
      end function
      integer(c_int) function pic_load_particles(h, n, q, x, y, z, u, v, w, flv) bind(C, name="pic_load_particles")
         import :: c_int, c_ptr, c_double, c_int64_t, c_int32_t
         type(c_ptr), value :: h
         integer(c_int64_t), value :: n
         real(c_double), intent(in) :: q(*), x(*), y(*), z(*), u(*), v(*), w(*)
         integer(c_int32_t), intent(in) :: flv(*)
      end function
      integer(c_int) function pic_fetch_particles(h, n, q, x, y, z, u, v, w, flv) bind(C, name="pic_fetch_particles")
         import :: c_int, c_ptr, c_double, c_int64_t, c_int32_t
         type(c_ptr), value :: h
         integer(c_int64_t), intent(out) :: n
         real(c_double), intent(out) :: q(*), x(*), y(*), z(*), u(*), v(*), w(*)
         integer(c_int32_t), intent(out) :: flv(*)
      end function
      integer(c_int) function pic_particle_count(h, n) bind(C, name="pic_particle_count")
         import :: c_int, c_ptr, c_int64_t
         type(c_ptr), value :: h
         integer(c_int64_t), intent(out) :: n
      end function
   end interface

   ! the phase entry points share one signature: int f(pic_handle*)
   interface
      integer(c_int) function pic_update_b_half(h) bind(C, name="pic_update_b_half")
         import :: c_int, c_ptr
         type(c_ptr), value :: h
      end function
      integer(c_int) function pic_move_deposit(h) bind(C, name="pic_move_deposit")
         import :: c_int, c_ptr
         type(c_ptr), value :: h
      end function
      integer(c_int) function pic_exchange_particles(h) bind(C, name="pic_exchange_particles")
         import :: c_int, c_ptr
         type(c_ptr), value :: h
      end function
      integer(c_int) function pic_update_e(h) bind(C, name="pic_update_e")
         import :: c_int, c_ptr
         type(c_ptr), value :: h
      end function
      integer(c_int) function pic_fold_current(h) bind(C, name="pic_fold_current")
         import :: c_int, c_ptr
         type(c_ptr), value :: h
      end function
      integer(c_int) function pic_filter_current(h) bind(C, name="pic_filter_current")
         import :: c_int, c_ptr
         type(c_ptr), value :: h
      end function
      integer(c_int) function pic_add_current(h) bind(C, name="pic_add_current")
         import :: c_int, c_ptr
         type(c_ptr), value :: h
      end function
      integer(c_int) function pic_reset_current(h) bind(C, name="pic_reset_current")
         import :: c_int, c_ptr
         type(c_ptr), value :: h
      end function
      integer(c_int) function pic_reorder(h) bind(C, name="pic_reorder")
         import :: c_int, c_ptr
         type(c_ptr), value :: h
      end function
   end interface

   ! Walls: EnforceBC_PostMovDep / EnforceBC_Final (bc.F90) call these for
   ! bc_face(1:4) of type 'refl' / 'cond' (side 0 = low face) and 'remv'.
   interface
      integer(c_int) function pic_bc_reflect_x(h, side, pos) bind(C, name="pic_bc_reflect_x")
         import :: c_int, c_ptr, c_int32_t, c_double
         type(c_ptr), value :: h
         integer(c_int32_t), value :: side
         real(c_double), value :: pos
      end function
      integer(c_int) function pic_bc_conducting_x(h, side, pos) bind(C, name="pic_bc_conducting_x")
         import :: c_int, c_ptr, c_int32_t, c_double
         type(c_ptr), value :: h
         integer(c_int32_t), value :: side
         real(c_double), value :: pos
      end function
      integer(c_int) function pic_bc_reflect_y(h, side, pos) bind(C, name="pic_bc_reflect_y")
         import :: c_int, c_ptr, c_int32_t, c_double
         type(c_ptr), value :: h
         integer(c_int32_t), value :: side
         real(c_double), value :: pos
      end function
      integer(c_int) function pic_bc_conducting_y(h, side, pos) bind(C, name="pic_bc_conducting_y")
         import :: c_int, c_ptr, c_int32_t, c_double
         type(c_ptr), value :: h
         integer(c_int32_t), value :: side
         real(c_double), value :: pos
      end function
      integer(c_int) function pic_bc_remove(h, face, pos) bind(C, name="pic_bc_remove")
         import :: c_int, c_ptr, c_int32_t, c_double
         type(c_ptr), value :: h
         integer(c_int32_t), value :: face
         real(c_double), value :: pos
      end function
   end interface

   ! Field faces of EnforceBC_Final besides 'cond': 'attn' faces
   ! (Attenuate_EM_Vacuum: faces = bit mask of bc_face(1:6), pos and scale
   ! hold bc_face(:)%pos_fld and %attn_scale), an 'iflw' face with a uniform
   ! flow (Attenuate_EM_Flow), 'open' x faces for fields (OpenBC_Fld_*) and
   ! particles (OpenBC_Prtl_*).
   interface
      integer(c_int) function pic_bc_attenuate(h, faces, pos, scale) bind(C, name="pic_bc_attenuate")
         import :: c_int, c_ptr, c_int32_t, c_double
         type(c_ptr), value :: h
         integer(c_int32_t), value :: faces
         real(c_double), intent(in) :: pos(6), scale(6)
      end function
      integer(c_int) function pic_bc_attenuate_flow(h, face, pos, thickness, scale, bflow, drift) &
            bind(C, name="pic_bc_attenuate_flow")
         import :: c_int, c_ptr, c_int32_t, c_double
         type(c_ptr), value :: h
         integer(c_int32_t), value :: face
         real(c_double), value :: pos, thickness, scale
         real(c_double), intent(in) :: bflow(3), drift(3)
      end function
      integer(c_int) function pic_bc_open_x(h, side, pos) bind(C, name="pic_bc_open_x")
         import :: c_int, c_ptr, c_int32_t, c_double
         type(c_ptr), value :: h
         integer(c_int32_t), value :: side
         real(c_double), value :: pos
      end function
      integer(c_int) function pic_bc_open_prtl_x(h, side, pos) bind(C, name="pic_bc_open_prtl_x")
         import :: c_int, c_ptr, c_int32_t, c_double
         type(c_ptr), value :: h
         integer(c_int32_t), value :: side
         real(c_double), value :: pos
      end function
      integer(c_int) function pic_bc_inflow(h, inj) bind(C, name="pic_bc_inflow")
         import :: c_int, c_ptr, pic_inflow_t
         type(c_ptr), value :: h
         type(pic_inflow_t), intent(in) :: inj
      end function
      integer(c_int) function pic_bc_inflow_reflect(h, pos, drift_x) bind(C, name="pic_bc_inflow_reflect")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: h
         real(c_double), value :: pos, drift_x
      end function
      ! 'pml' faces (bc_pml.F90): faces = bit mask of bc_face(1:6), pos and
      ! thickness hold bc_face(:)%pos_fld and %attn_thickness; then
      ! pic_bc_pml_b where MAIN calls UpdateMagFld_PML and pic_bc_pml_e where
      ! it calls UpdateElcFld_PML
      integer(c_int) function pic_bc_pml(h, faces, pos, thickness) bind(C, name="pic_bc_pml")
         import :: c_int, c_ptr, c_int32_t, c_double
         type(c_ptr), value :: h
         integer(c_int32_t), value :: faces
         real(c_double), intent(in) :: pos(6), thickness(6)
      end function
      integer(c_int) function pic_bc_pml_b(h) bind(C, name="pic_bc_pml_b")
         import :: c_int, c_ptr
         type(c_ptr), value :: h
      end function
      integer(c_int) function pic_bc_pml_e(h) bind(C, name="pic_bc_pml_e")
         import :: c_int, c_ptr
         type(c_ptr), value :: h
      end function
   end interface

   ! Slab form (cfg%slab_x = 1): x faces exchanged by the host
   ! between ranks; buffers are device addresses (a CUDA-aware MPI_Sendrecv
   ! takes them as they are), see include/pictor_b200.h.
   interface
      integer(c_int) function pic_slab_face_len(h, n) bind(C, name="pic_slab_face_len")
         import :: c_int, c_ptr, c_int64_t
         type(c_ptr), value :: h
         integer(c_int64_t), intent(out) :: n
      end function
      integer(c_int) function pic_slab_pack_fields(h, which, to_left, to_right) bind(C, name="pic_slab_pack_fields")
         import :: c_int, c_ptr, c_int32_t
         type(c_ptr), value :: h, to_left, to_right
         integer(c_int32_t), value :: which
      end function
      integer(c_int) function pic_slab_unpack_fields(h, which, from_left, from_right) &
            bind(C, name="pic_slab_unpack_fields")
         import :: c_int, c_ptr, c_int32_t
         type(c_ptr), value :: h, from_left, from_right
         integer(c_int32_t), value :: which
      end function
      integer(c_int) function pic_slab_pack_particles(h, out, cap, n_right, n_left) &
            bind(C, name="pic_slab_pack_particles")
         import :: c_int, c_ptr, c_int64_t
         type(c_ptr), value :: h, out
         integer(c_int64_t), value :: cap
         integer(c_int64_t), intent(out) :: n_right, n_left
      end function
      integer(c_int) function pic_slab_unpack_particles(h, in, n) bind(C, name="pic_slab_unpack_particles")
         import :: c_int, c_ptr, c_int64_t
         type(c_ptr), value :: h, in
         integer(c_int64_t), value :: n
      end function
   end interface

   type(c_ptr), save :: pic_h = c_null_ptr

   ! Choices with no counterpart in the reference's parameters.F90, read by
   ! InitAll_gpu from the environment so that no setup file changes:
   !   PICTOR_PRECISION=fp32   the FP32 cell-relative form (default fp64, the
   !                           reference layout and arithmetic)
   !   PICTOR_EXACT_CURRENT=1  FP64: the current summed in the serial CPU
   !                           build's order (bit-exact, reproducible runs)
   integer(c_int32_t), save :: pictor_precision = 0, pictor_exact_current = 0

contains

   subroutine pictor_read_env()
      character(len=16) :: val
      integer :: ln, st
      call get_environment_variable("PICTOR_PRECISION", val, ln, st)
      if (st .eq. 0 .and. (val(1:4) .eq. 'fp32' .or. val(1:4) .eq. 'FP32')) pictor_precision = 1
      call get_environment_variable("PICTOR_EXACT_CURRENT", val, ln, st)
      if (st .eq. 0 .and. val(1:1) .eq. '1') pictor_exact_current = 1
   end subroutine pictor_read_env

   subroutine pic_check(code)
      use communication, only: Abort   ! communication.F90:96-102
      integer(c_int), intent(in) :: code
      if (code .ne. 0) call Abort(int(100 - code))
   end subroutine pic_check

end module pictor_b200_capi

! ---------------------------------------------------------------------------
! Modules named as MAIN.F90 uses them under #ifdef gpu.
! ---------------------------------------------------------------------------
module var_gpu
   use pictor_b200_capi
end module var_gpu

module initialise_gpu
   use parameters
   use vars
   use pictor_b200_capi
   implicit none
contains
   subroutine InitAll_gpu   ! replaces src/init/initialise_gpu.F90:9
      type(pic_config) :: cfg
      integer :: n
      cfg%nx = mx - 5; cfg%ny = my - 5; cfg%nz = max(mz - 5, 1)
#ifdef twoD
      cfg%dims = 2
#else
      cfg%dims = 3
#endif
#ifdef cyl
      cfg%geom = 1
#else
      cfg%geom = 0
#endif
      ! FDTD=Lehe in the reference Makefile only swaps sources (Makefile:70-74):
      ! add -DLehe to the flags of this file in a Lehe build
#ifdef Lehe
      cfg%fdtd = 1
#else
      cfg%fdtd = 0
#endif
      call pictor_read_env()
      cfg%precision = pictor_precision
      cfg%exact_current = pictor_exact_current
      cfg%nflvr = Nflvr
      cfg%c = c; cfg%qi = qi
      cfg%bext = (/ Bx_ext0, By_ext0, Bz_ext0 /)
      cfg%qm = 0
      do n = 1, Nflvr
         cfg%qm(n) = flvrqm(n)
      end do
      cfg%reorder_period = prtl_reorder_period
      cfg%curr_filter = curr_filter
      cfg%capacity = gpu_prtl_arr_size
#ifdef cyl
      ! r of the first interior x cell and whether the axis is on this rank
      ! (cyl_common.F90:19-32, cyl_em_update.F90:145)
      cfg%rmin = xborders(procxind) + rshift
      cfg%inc_axis = merge(1, 0, inc_axis .and. procxind .eq. 0)
#else
      cfg%rmin = 0; cfg%inc_axis = 1
#endif
      cfg%brick = 0; cfg%cyl_modes = 0; cfg%slab_x = 0; cfg%fp64_tiles = 0; cfg%exact_charge = 0; cfg%reserved = 0
      call pic_check(pic_create(cfg, pic_h))
      call pic_check(pic_load_fields(pic_h, Ex, Ey, Ez, Bx, By, Bz))
      call pic_check(pic_load_particles(pic_h, int(used_prtl_arr_size, c_int64_t), qp, xp, yp, zp, up, vp, wp, flvp))
   end subroutine InitAll_gpu

   ! MAIN.F90:390 calls this after InitAll_gpu in a -Dcyl build.  The
   ! reference's version (cyl_common.F90:35-39) allocates the device arrays
   ! of the axis update; pic_create has allocated everything the cylindrical
   ! step needs, so nothing is left to do.  Compile src/cyl/cyl_common.F90
   ! without -Dgpu so that this is the only InitAll_cyl_gpu.
   subroutine InitAll_cyl_gpu
   end subroutine InitAll_cyl_gpu
end module initialise_gpu

module em_update_gpu
   use pictor_b200_capi
   implicit none
contains
   subroutine UpdateBfieldHalfGPU      ! em_update_gpu.F90:44 (+ halo)
      call pic_check(pic_update_b_half(pic_h))
   end subroutine
   subroutine UpdateEfieldGPU          ! em_update_gpu.F90:12 (+ halo)
      call pic_check(pic_update_e(pic_h))
   end subroutine
   subroutine AddCurrentGPU            ! em_update_gpu.F90:92 (+ halo)
      call pic_check(pic_add_current(pic_h))
   end subroutine
end module em_update_gpu

module movdep_gpu
   use pictor_b200_capi
   implicit none
contains
   subroutine MoveDepositPrtlGPU       ! movdep_gpu.F90:14
      call pic_check(pic_move_deposit(pic_h))
   end subroutine
end module movdep_gpu

module particles_gpu
   use vars
   use pictor_b200_capi
   implicit none
contains
   subroutine ExchangePrtlGPU          ! LoadPrtlOutliers + AppendParticles on one periodic rank
      call pic_check(pic_exchange_particles(pic_h))
   end subroutine
   subroutine ReorderPrtlGPU           ! particles_gpu.F90:416
      if (modulo(t, prtl_reorder_period) .eq. 0) call pic_check(pic_reorder(pic_h))
   end subroutine
   subroutine CopyGPUDataToHostForOutput   ! particles_gpu.F90:569
      integer(c_int64_t) :: n
      call pic_check(pic_particle_count(pic_h, n))
      if (n .gt. size(xp)) call ReshapePrtlArr(int(n) + 1000000)
      call pic_check(pic_fetch_particles(pic_h, n, qp, xp, yp, zp, up, vp, wp, flvp))
      used_prtl_arr_size = int(n)
      call pic_check(pic_fetch_fields(pic_h, Ex, Ey, Ez, Bx, By, Bz, Jx, Jy, Jz))
   end subroutine
   subroutine FinishSaveDataGPU
   end subroutine
end module particles_gpu

module fields_gpu
   use pictor_b200_capi
   implicit none
contains
   subroutine ResetCurrentGPU          ! fields_gpu.F90:61
      call pic_check(pic_reset_current(pic_h))
   end subroutine
   subroutine smoothen_current_gpu     ! fields_gpu.F90:120 (filter on the device)
      call pic_check(pic_filter_current(pic_h))
   end subroutine
end module fields_gpu

module comm_fld_gpu
   use pictor_b200_capi
   implicit none
contains
   subroutine UpdateCurrentsAllEdgesGPU    ! ghost current fold on one periodic rank
      call pic_check(pic_fold_current(pic_h))
   end subroutine
   subroutine EMfldExchangeGPU             ! halo: done inside every field update
   end subroutine
end module comm_fld_gpu
