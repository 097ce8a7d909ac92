! gazpart_gpu_iface.f90 -- the Fortran side of the drop-in boundary.
!
! Linked into the reference's own build in place of interp_lag3.o, frozen_interp_lag3.o,
! fluid_force_ellipsoid.o, fluid_torque_ellipsoid.o, adv_particle_new.o, adv_quaternion.o,
! adv_angular_velocity.o, collision*.o, ellipsoid_contact_detection.o and
! collision_response.o (Makefile:56-111).  Every routine below keeps the name and the
! argument list of the one it replaces, so its callers (main.f90:466,483, interpH.f90,
! the statistics routines) are unchanged; each forwards to the C ABI of
! include/gazpart_gpu.h through ISO_C_BINDING interfaces and turns a nonzero status into
! the reference's stop, with the reference's message where it has one.
!
! Not compiled in this repository: neither the build host nor the GPU host has a Fortran
! compiler (gfortran, ifort, ifx and flang are absent), so this file is written against
! the reference's modules (DNS_DIM, GEOMETRIC_VARIABLE, PARAM_PHYS, COLLISION_VARIABLE,
! PARTICLE_PARALLEL, FLUID_VARIABLE, mod_quaternion) and the header, and checked only by
! reading.
!
! How the state moves
!  - COLLISION_INITIATION (called once by main.f90 after the fields and particles are
!    initialised) creates the context, loads the six field components and uploads
!    PART(1:NPART_LOC(J), J) for every class J.  From then on the particles live on the
!    device: ADV_PARTICLE_ELLP and COLLISION step them there.
!  - GAZPART_GPU_SYNC copies the device state back into PART (positions, velocities,
!    quaternions, angular velocities and the interpolated fluid values UFAP..VORTZAP).
!    Call it before anything reads PART on the host: STAT_*, PRINT_PARTICLE,
!    SAVE_PARTICLE (main.f90:402-440,697).
!  - GAZPART_GPU_PUT copies PART back to the device after a host-side change.
!  - GAZPART_GPU_FIELDS_CHANGED tells the interpolation drop-in that the field arrays
!    have new values (after ADV_FLUID in DNS mode); frozen fields never change.
!
! Limits of this wrapper (not of the C ABI)
!  - One context for all classes: GRAVITY, ECP and MUP are taken from class 1, and a run
!    whose classes differ in them stops at COLLISION_INITIATION.
!  - NPROC = 1 (one rank, one GPU): the path runs on one GPU, without the MPI domain
!    decomposition.

module gazpart_gpu
  use iso_c_binding
  implicit none

  integer(c_int32_t), parameter :: GP_LAYOUT_REFERENCE = 1, GP_GHOST_PERIODIC = 0, GP_GHOST_ZERO = 1
  integer(c_int32_t), parameter :: GP_PREC_FP64 = 0

  type, bind(c) :: gp_params
     integer(c_int32_t) :: nx, ny, nz
     real(c_double)     :: lx, ly, lz, visc, rhof, dtime, gravity, ecp, mup, ecw, muw
     integer(c_int32_t) :: periodicity, wall_boundary, interp_scheme, frozen_flow
     integer(c_int32_t) :: precision, store_fluid
     integer(c_int64_t) :: max_particles
  end type gp_params

  interface
     integer(c_int) function gp_ctx_create(p, ctx) bind(c, name='gp_ctx_create')
       import; type(gp_params), intent(in) :: p; type(c_ptr) :: ctx
     end function
     integer(c_int) function gp_ctx_destroy(ctx) bind(c, name='gp_ctx_destroy')
       import; type(c_ptr), value :: ctx
     end function
     integer(c_int) function gp_status(ctx, code, first_id) bind(c, name='gp_status')
       import; type(c_ptr), value :: ctx; integer(c_int32_t) :: code; integer(c_int64_t) :: first_id
     end function
     integer(c_int) function gp_clear_status(ctx) bind(c, name='gp_clear_status')
       import; type(c_ptr), value :: ctx
     end function
     integer(c_int) function gp_set_class(ctx, ig, idp, emaj, apr, rhop) bind(c, name='gp_set_class')
       import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: ig, idp
       real(c_double), value :: emaj, apr, rhop
     end function
     integer(c_int) function gp_set_field(ctx, comp, src, layout, ghost, on_device) bind(c, name='gp_set_field')
       import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: comp, layout, ghost, on_device
       type(c_ptr), value :: src
     end function
     integer(c_int) function gp_upload_classes(ctx, nclass, counts, cols, props, on_device) &
          bind(c, name='gp_upload_classes')
       import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: nclass, on_device
       integer(c_int64_t), intent(in) :: counts(*); type(c_ptr), intent(in) :: cols(13), props(6)
     end function
     integer(c_int) function gp_put_state(ctx, n, cols, on_device) bind(c, name='gp_put_state')
       import; type(c_ptr), value :: ctx; integer(c_int64_t), value :: n
       type(c_ptr), intent(in) :: cols(13); integer(c_int32_t), value :: on_device
     end function
     integer(c_int) function gp_download_state(ctx, n, cols, fluid, on_device) bind(c, name='gp_download_state')
       import; type(c_ptr), value :: ctx; integer(c_int64_t), value :: n
       type(c_ptr), intent(in) :: cols(13), fluid(6); integer(c_int32_t), value :: on_device
     end function
     integer(c_int) function gp_adv_particle_ellp(ctx, ncycle) bind(c, name='gp_adv_particle_ellp')
       import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: ncycle
     end function
     integer(c_int) function gp_collision(ctx, ncycle, time, n_near, n_contact, n_coll) bind(c, name='gp_collision')
       import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: ncycle; real(c_double), value :: time
       type(c_ptr), value :: n_near, n_contact, n_coll
     end function
     integer(c_int) function gp_collision_box_connectivity(ctx, nbox, ncon, con, dims, geom) &
          bind(c, name='gp_collision_box_connectivity')
       import; type(c_ptr), value :: ctx; integer(c_int32_t) :: nbox
       type(c_ptr), value :: ncon, con, dims, geom
     end function
     integer(c_int) function gp_interp_lag3(ctx, comp, nint, xint, yint, zint, uint, on_device) &
          bind(c, name='gp_interp_lag3')
       import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: comp, on_device
       integer(c_int64_t), value :: nint; real(c_double), intent(in) :: xint(*), yint(*), zint(*)
       real(c_double), intent(out) :: uint(*)
     end function
     integer(c_int) function gp_frozen_interp_lag3(ctx, xain, yain, zain, nx, ny, nz, uain, nint, &
          xint, yint, zint, uint) bind(c, name='gp_frozen_interp_lag3')
       import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: nx, ny, nz
       real(c_double), intent(in) :: xain(*), yain(*), zain(*), uain(*), xint(*), yint(*), zint(*)
       integer(c_int64_t), value :: nint; real(c_double), intent(out) :: uint(*)
     end function
     integer(c_int) function gp_fluid_force_ellipsoid(ctx, ig, idp, up, vp, wp, uf, vf, wf, q, fd, fl) &
          bind(c, name='gp_fluid_force_ellipsoid')
       import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: ig, idp
       real(c_double), value :: up, vp, wp, uf, vf, wf; real(c_double), intent(in) :: q(4)
       real(c_double), intent(out) :: fd(3), fl(3)
     end function
     integer(c_int) function gp_fluid_torque_ellipsoid(ctx, ig, idp, ox, oy, oz, q, part_up, part_ufap, &
          part_vort, tpitch, trot) bind(c, name='gp_fluid_torque_ellipsoid')
       import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: ig, idp
       real(c_double), value :: ox, oy, oz; real(c_double), intent(in) :: q(4), part_up(3), part_ufap(3)
       real(c_double), intent(in) :: part_vort(3); real(c_double), intent(out) :: tpitch(3), trot(3)
     end function
     integer(c_int) function gp_quaternion_integration(ctx, q, omgx, omgy, omgz, dt) &
          bind(c, name='gp_quaternion_integration')
       import; type(c_ptr), value :: ctx; real(c_double), intent(inout) :: q(4)
       real(c_double), value :: omgx, omgy, omgz, dt
     end function
     integer(c_int) function gp_euler_integration(ctx, ig, idp, omgx, omgy, omgz) bind(c, name='gp_euler_integration')
       import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: ig, idp
       real(c_double), intent(inout) :: omgx, omgy, omgz
     end function
     integer(c_int) function gp_ellipsoid_contact_detection(ctx, ig, idp1, idp2, ix, iy, iz, iq, &
          jx, jy, jz, jq, flag, e1, e2, cn) bind(c, name='gp_ellipsoid_contact_detection')
       import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: ig, idp1, idp2
       real(c_double), value :: ix, iy, iz, jx, jy, jz; real(c_double), intent(in) :: iq(4), jq(4)
       integer(c_int32_t), intent(out) :: flag; real(c_double), intent(out) :: e1(3), e2(3), cn(3)
     end function
     integer(c_int) function gp_collision_response(ctx, ig, idp, part1, part2, r1, r2, nrm) &
          bind(c, name='gp_collision_response')
       import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: ig, idp
       real(c_double), intent(inout) :: part1(10), part2(10)
       real(c_double), intent(in) :: r1(3), r2(3), nrm(3)
     end function
     ! Launch tuning, optional: a driver may call gp_autotune once after
     ! COLLISION_INITIATION (it times the launch choices on the resident particles and
     ! restores their state); no result depends on these choices.
     integer(c_int) function gp_autotune(ctx, grids) bind(c, name='gp_autotune')
       import; type(c_ptr), value :: ctx; integer(c_int32_t), intent(out) :: grids(5)
     end function
     integer(c_int) function gp_set_contact_order(ctx, on) bind(c, name='gp_set_contact_order')
       import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: on
     end function
     integer(c_int) function gp_set_gather_staging(ctx, mode) bind(c, name='gp_set_gather_staging')
       import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: mode
     end function
  end interface
end module gazpart_gpu


module gazpart_gpu_iface_state
  use iso_c_binding
  use gazpart_gpu
  implicit none
  type(c_ptr), save :: gp = c_null_ptr
  ! field arrays already loaded into the context, by address (INTERP_LAG3's UAIN)
  type(c_ptr), save :: field_src(6) = c_null_ptr
  ! host copies of PART in the C ABI's column order, classes one after another
  real(c_double), allocatable, target, save :: cols(:, :), props(:, :), fluid(:, :)
  integer(c_int64_t), allocatable, save :: counts(:)
  integer(c_int64_t), save :: ntot = 0

contains

  ! The context, created from the reference's module variables on the first call of any
  ! routine here (INITIATION_PARTICLE_VELOCITY interpolates before COLLISION_INITIATION).
  subroutine ensure_ctx()
    use DNS_DIM, only: NX, NY, NZ
    use GEOMETRIC_VARIABLE, only: LXMAX, LYMAX, LZMAX
    use PARAM_PHYS, only: VISC, RHOF, DTIME, GRAVITY, PERIODICITY, WALL_BOUNDARY, INTERP_SCHEME, FROZEN_FLOW
    use COLLISION_VARIABLE, only: ECP, MUP, ECW, MUW
    type(gp_params) :: p
    if (c_associated(gp)) return
    p%nx = NX; p%ny = NY; p%nz = NZ
    p%lx = LXMAX; p%ly = LYMAX; p%lz = LZMAX
    p%visc = VISC; p%rhof = RHOF; p%dtime = DTIME; p%gravity = GRAVITY(1)
    p%ecp = ECP(1); p%mup = MUP(1); p%ecw = ECW; p%muw = MUW
    p%periodicity = merge(1, 0, PERIODICITY); p%wall_boundary = merge(1, 0, WALL_BOUNDARY)
    p%interp_scheme = INTERP_SCHEME; p%frozen_flow = FROZEN_FLOW
    p%precision = GP_PREC_FP64; p%store_fluid = 1; p%max_particles = 0
    call gp_check(gp_ctx_create(p, gp), 'gazpart_gpu context')
  end subroutine ensure_ctx

  ! A ghosted field array (the reference's (NX, NY+4, NZ+4) layout) into component slot
  ! `slot` of the context; `a` is the caller's array, seen here with TARGET so that its
  ! address can be passed on (and remembered for INTERP_LAG3).
  subroutine load_field(slot, a)
    integer, intent(in) :: slot
    real(c_double), target, intent(in) :: a(*)
    call gp_check(gp_set_field(gp, int(slot, c_int32_t), c_loc(a), GP_LAYOUT_REFERENCE, GP_GHOST_PERIODIC, &
                               0_c_int32_t), 'field')
    field_src(slot + 1) = c_loc(a)
  end subroutine load_field

  ! A nonzero status becomes the reference's stop (status codes of gazpart_gpu.h).
  subroutine gp_check(rc, where)
    integer(c_int), intent(in) :: rc
    character(len=*), intent(in) :: where
    integer(c_int32_t) :: code
    integer(c_int64_t) :: id
    code = int(rc, c_int32_t)
    if (code == 0 .and. c_associated(gp)) then
       if (gp_status(gp, code, id) /= 0) code = 8
    end if
    select case (code)
    case (0)
       return
    case (1)
       stop 'In Fluid force'                        ! fluid_force_ellipsoid.f90:157
    case (2)
       write(*,*) 'FLUID_TORQUE_ELLIPSOID: NaN angular velocity'     ! fluid_torque_ellipsoid.f90:178-187
       stop
    case (3)
       write(*,*) ' Error in KE (Total)% above 1e-9 in ', where   ! collision_response.f90:408-435,
       stop                                                       ! wall_ellipsoid_rebound.f90:372-384
    case (4)
       stop 'Matrix is numerically singular!'       ! invert_ndim3_matrix.f90:20
    case (6)
       write(*,*) 'particle outside the collision box grid or the stencil range in ', where
       stop
    case default
       write(*,*) 'gazpart_gpu: status ', code, ' in ', where
       error stop
    end select
  end subroutine gp_check

  ! PART(1:NPART_LOC(J), J) into the column buffers (state, properties).
  subroutine pack_part()
    use DNS_DIM, only: NIG, NPART_LOC
    use PARTICLE_PARALLEL, only: PART
    use PARAM_PHYS, only: EMAJ_PART, APR_PART, RHOP, IPXX, IPYY, IPZZ
    integer :: j, i, idp
    integer(c_int64_t) :: k
    if (.not. allocated(counts)) allocate(counts(NIG))
    counts = int(NPART_LOC(1:NIG), c_int64_t)
    ntot = sum(counts)
    if (allocated(cols)) deallocate(cols, props, fluid)
    allocate(cols(max(ntot, 1_c_int64_t), 13), props(max(ntot, 1_c_int64_t), 6), fluid(max(ntot, 1_c_int64_t), 6))
    k = 0
    do j = 1, NIG
       do i = 1, NPART_LOC(j)
          k = k + 1
          idp = PART(i, j)%IDP
          cols(k, 1:13) = (/ PART(i, j)%XP, PART(i, j)%YP, PART(i, j)%ZP, &
                             PART(i, j)%UP, PART(i, j)%VP, PART(i, j)%WP, &
                             PART(i, j)%ELLQUAT%a, PART(i, j)%ELLQUAT%b, PART(i, j)%ELLQUAT%c, PART(i, j)%ELLQUAT%d, &
                             PART(i, j)%OMEGAX, PART(i, j)%OMEGAY, PART(i, j)%OMEGAZ /)
          props(k, 1:6) = (/ EMAJ_PART(j, idp), APR_PART(j), RHOP(j, idp), IPXX(j, idp), IPYY(j, idp), IPZZ(j, idp) /)
       end do
    end do
  end subroutine pack_part

  subroutine col_ptrs(p13)
    type(c_ptr), intent(out) :: p13(13)
    integer :: c
    do c = 1, 13
       p13(c) = c_loc(cols(1, c))
    end do
  end subroutine col_ptrs

end module gazpart_gpu_iface_state


! COLLISION_INITIATION (collision_initiation.f90:7-192): the box grid is set up inside
! the context from the particles' largest EMAJ, as the reference does
! (collision_initiation.f90:44-103); the module's grid variables and COLBOX are filled
! from it.  Also creates the context, loads the fields and uploads PART.
subroutine COLLISION_INITIATION
  use iso_c_binding
  use gazpart_gpu
  use gazpart_gpu_iface_state
  use DNS_DIM, only: NIG
  use PARAM_PHYS, only: GRAVITY, EMAJ_PART, APR_PART, RHOP, POLYDISP
  use COLLISION_VARIABLE, only: ECP, MUP
  use FLUID_VARIABLE, only: UFLU, VFLU, WFLU, VORTICITY_X, VORTICITY_Y, VORTICITY_Z
  implicit none
  type(c_ptr) :: pc(13), pp(6)
  integer :: j, idp, c
  if (NIG > 1) then
     if (any(GRAVITY(2:NIG) /= GRAVITY(1)) .or. any(ECP(2:NIG) /= ECP(1)) .or. any(MUP(2:NIG) /= MUP(1))) &
        stop 'gazpart_gpu: classes with different GRAVITY, ECP or MUP need one context each'
  end if
  call ensure_ctx()
  do j = 1, NIG
     do idp = 1, POLYDISP(j)
        call gp_check(gp_set_class(gp, int(j, c_int32_t), int(idp, c_int32_t), EMAJ_PART(j, idp), &
                                   APR_PART(j), RHOP(j, idp)), 'COLLISION_INITIATION')
     end do
  end do
  ! the six components in the step's order; the velocity ghosts are the self-exchanged
  ! planes FLUIDCOMM leaves and the vorticity ghosts hold zero (main.f90:255-259), both
  ! already in the arrays
  field_src = c_null_ptr
  call load_field(0, UFLU)
  call load_field(1, VFLU)
  call load_field(2, WFLU)
  call load_field(3, VORTICITY_X)
  call load_field(4, VORTICITY_Y)
  call load_field(5, VORTICITY_Z)
  call pack_part()
  call col_ptrs(pc)
  do c = 1, 6
     pp(c) = c_loc(props(1, c))
  end do
  call gp_check(gp_upload_classes(gp, int(NIG, c_int32_t), counts, pc, pp, 0_c_int32_t), 'COLLISION_INITIATION')
  call COLLISION_BOX_CONNECTIVITY
end subroutine COLLISION_INITIATION


! COLLISION_BOX_CONNECTIVITY (collision_box_connectivity.f90:7-384): the grid variables
! and COLBOX(1:NBOX)%NCON / %CON of the context's box grid (class 1's).
subroutine COLLISION_BOX_CONNECTIVITY
  use iso_c_binding
  use gazpart_gpu
  use gazpart_gpu_iface_state
  use COLLISION_VARIABLE, only: NXBOX, NYBOX, NZBOX, NBOX, DXBOX, DYBOX, DZBOX, XMINBOX, YMINBOX, ZMINBOX, &
                                XMAXBOX, YMAXBOX, ZMAXBOX, DELTA_COLL, COLBOX
  use GEOMETRIC_VARIABLE, only: XMESH, YMESH, ZMESH, DX, DY, DZ
  use DNS_DIM, only: ISTART, IEND
  implicit none
  integer(c_int32_t) :: nb
  integer(c_int32_t), target :: dims(3)
  real(c_double), target :: geom(6)
  integer(c_int32_t), allocatable, target :: ncon(:), con(:, :)
  integer :: b
  call gp_check(gp_collision_box_connectivity(gp, nb, c_null_ptr, c_null_ptr, c_loc(dims), c_loc(geom)), &
                'COLLISION_BOX_CONNECTIVITY')
  allocate(ncon(nb), con(27, nb))
  call gp_check(gp_collision_box_connectivity(gp, nb, c_loc(ncon), c_loc(con), c_null_ptr, c_null_ptr), &
                'COLLISION_BOX_CONNECTIVITY')
  NXBOX = dims(1); NYBOX = dims(2); NZBOX = dims(3); NBOX = nb
  DXBOX = geom(1); DYBOX = geom(2); DZBOX = geom(3)
  XMINBOX = geom(4); YMINBOX = geom(5); ZMINBOX = geom(6)
  ! collision_initiation.f90:83-93 with NPROC = 1 (DELTA_COLL = ZERO)
  DELTA_COLL = YMESH(ISTART(2)) - YMINBOX
  XMAXBOX = XMESH(IEND(1)) + DX
  YMAXBOX = YMESH(IEND(2)) + DY + DELTA_COLL
  ZMAXBOX = ZMESH(IEND(3)) + DZ + DELTA_COLL
  if (allocated(COLBOX)) deallocate(COLBOX)
  allocate(COLBOX(NBOX))
  do b = 1, NBOX
     COLBOX(b)%NCON = ncon(b)
     COLBOX(b)%CON(:) = con(:, b)
  end do
end subroutine COLLISION_BOX_CONNECTIVITY


! INTERP_LAG3(XAIN,YAIN,ZAIN,UAIN,NINT,XINT,YINT,ZINT,UINT)  interp_lag3.f90:11-298.
! UAIN is one of the ghosted field arrays; a new array is loaded into a free component
! slot of the context once and recognised by its address afterwards.
subroutine INTERP_LAG3(XAIN, YAIN, ZAIN, UAIN, NINT, XINT, YINT, ZINT, UINT)
  use iso_c_binding
  use gazpart_gpu
  use gazpart_gpu_iface_state
  use DNS_DIM, only: ISTART, IEND, NGHTCELL
  implicit none
  real(kind=8), dimension(ISTART(1):IEND(1)), intent(in) :: XAIN
  real(kind=8), dimension(ISTART(2):IEND(2)), intent(in) :: YAIN
  real(kind=8), dimension(ISTART(3):IEND(3)), intent(in) :: ZAIN
  real(kind=8), dimension(ISTART(1):IEND(1), ISTART(2)-NGHTCELL:IEND(2)+NGHTCELL, &
                          ISTART(3)-NGHTCELL:IEND(3)+NGHTCELL), intent(in), target :: UAIN
  integer, intent(in) :: NINT
  real(kind=8), dimension(NINT), intent(in) :: XINT, YINT, ZINT
  real(kind=8), dimension(NINT), intent(out) :: UINT
  type(c_ptr) :: a
  integer :: c, slot
  call ensure_ctx()
  a = c_loc(UAIN)
  slot = -1
  do c = 1, 6
     if (c_associated(field_src(c), a)) slot = c - 1
  end do
  if (slot < 0) then
     do c = 1, 6
        if (.not. c_associated(field_src(c))) then
           slot = c - 1
           exit
        end if
     end do
     if (slot < 0) stop 'gazpart_gpu: more than six field arrays interpolated'
     call load_field(slot, UAIN)
  end if
  call gp_check(gp_interp_lag3(gp, int(slot, c_int32_t), int(NINT, c_int64_t), XINT, YINT, ZINT, UINT, 0_c_int32_t), &
                'INTERP_LAG3')
end subroutine INTERP_LAG3


! FROZEN_INTERP_LAG3(XAIN,YAIN,ZAIN,NX,NY,NZ,UAIN,NINT,XINT,YINT,ZINT,UINT)
! frozen_interp_lag3.f90:11-274 (mirror boundaries).
subroutine FROZEN_INTERP_LAG3(XAIN, YAIN, ZAIN, NX, NY, NZ, UAIN, NINT, XINT, YINT, ZINT, UINT)
  use iso_c_binding
  use gazpart_gpu
  use gazpart_gpu_iface_state
  implicit none
  integer, intent(in) :: NX, NY, NZ, NINT
  real(kind=8), intent(in) :: XAIN(NX), YAIN(NY), ZAIN(NZ), UAIN(NX, NY, NZ)
  real(kind=8), intent(in) :: XINT(NINT), YINT(NINT), ZINT(NINT)
  real(kind=8), intent(out) :: UINT(NINT)
  call ensure_ctx()
  call gp_check(gp_frozen_interp_lag3(gp, XAIN, YAIN, ZAIN, int(NX, c_int32_t), int(NY, c_int32_t), &
                                      int(NZ, c_int32_t), UAIN, int(NINT, c_int64_t), XINT, YINT, ZINT, UINT), &
                'FROZEN_INTERP_LAG3')
end subroutine FROZEN_INTERP_LAG3


! FLUID_FORCE_ELLIPSOID  fluid_force_ellipsoid.f90:1-161
subroutine FLUID_FORCE_ELLIPSOID(IG, IDP, UPART, VPART, WPART, UFLUID, VFLUID, WFLUID, quat, FDRAG, FLIFT)
  use iso_c_binding
  use gazpart_gpu
  use gazpart_gpu_iface_state
  use mod_quaternion, only: quaternion
  implicit none
  integer, intent(in) :: IG, IDP
  real(kind=8), intent(in) :: UPART, VPART, WPART, UFLUID, VFLUID, WFLUID
  type(quaternion), intent(in) :: quat
  real(kind=8), dimension(3, 1), intent(inout) :: FDRAG, FLIFT
  real(c_double) :: fd(3), fl(3)
  call ensure_ctx()
  call gp_check(gp_fluid_force_ellipsoid(gp, int(IG, c_int32_t), int(IDP, c_int32_t), UPART, VPART, WPART, &
                                         UFLUID, VFLUID, WFLUID, (/quat%a, quat%b, quat%c, quat%d/), fd, fl), &
                'FLUID_FORCE_ELLIPSOID')
  FDRAG(:, 1) = fd
  FLIFT(:, 1) = fl
end subroutine FLUID_FORCE_ELLIPSOID


! FLUID_TORQUE_ELLIPSOID  fluid_torque_ellipsoid.f90:1-190.  The reference reads
! PART(I,IG)%UP..WP, %UFAP..WFAP and %VORTXAP..VORTZAP from its module (:88-120); they
! are passed on from the host copy of PART.
subroutine FLUID_TORQUE_ELLIPSOID(I, IG, IDP, OX, OY, OZ, QUAT, TORQUE_PITCHING, TORQUE_ROTATION)
  use iso_c_binding
  use gazpart_gpu
  use gazpart_gpu_iface_state
  use mod_quaternion, only: quaternion
  use PARTICLE_PARALLEL, only: PART
  implicit none
  integer, intent(in) :: I, IG, IDP
  real(kind=8), intent(in) :: OX, OY, OZ
  type(quaternion), intent(in) :: QUAT
  real(kind=8), dimension(3, 1), intent(inout) :: TORQUE_PITCHING, TORQUE_ROTATION
  real(c_double) :: tp(3), tr(3)
  call ensure_ctx()
  call gp_check(gp_fluid_torque_ellipsoid(gp, int(IG, c_int32_t), int(IDP, c_int32_t), OX, OY, OZ, &
                (/QUAT%a, QUAT%b, QUAT%c, QUAT%d/), (/PART(I, IG)%UP, PART(I, IG)%VP, PART(I, IG)%WP/), &
                (/PART(I, IG)%UFAP, PART(I, IG)%VFAP, PART(I, IG)%WFAP/), &
                (/PART(I, IG)%VORTXAP, PART(I, IG)%VORTYAP, PART(I, IG)%VORTZAP/), tp, tr), 'FLUID_TORQUE_ELLIPSOID')
  TORQUE_PITCHING(:, 1) = tp
  TORQUE_ROTATION(:, 1) = tr
end subroutine FLUID_TORQUE_ELLIPSOID


! QUATERNION_INTEGRATION(qp_n, omgx, omgy, omgz, dt)  adv_quaternion.f90:1-117
subroutine QUATERNION_INTEGRATION(qp_n, omgx, omgy, omgz, dt)
  use iso_c_binding
  use gazpart_gpu
  use gazpart_gpu_iface_state
  use mod_quaternion, only: quaternion
  implicit none
  type(quaternion), intent(inout) :: qp_n
  real(kind=8), intent(in) :: omgx, omgy, omgz, dt
  real(c_double) :: q(4)
  q = (/qp_n%a, qp_n%b, qp_n%c, qp_n%d/)
  call ensure_ctx()
  call gp_check(gp_quaternion_integration(gp, q, omgx, omgy, omgz, dt), 'QUATERNION_INTEGRATION')
  qp_n%a = q(1); qp_n%b = q(2); qp_n%c = q(3); qp_n%d = q(4)
end subroutine QUATERNION_INTEGRATION


! EULER_INTEGRATION(IG, IDP, omgx, omgy, omgz)  adv_angular_velocity.f90:1-168
subroutine EULER_INTEGRATION(IG, IDP, omgx, omgy, omgz)
  use iso_c_binding
  use gazpart_gpu
  use gazpart_gpu_iface_state
  implicit none
  integer, intent(in) :: IG, IDP
  real(kind=8), intent(inout) :: omgx, omgy, omgz
  call ensure_ctx()
  call gp_check(gp_euler_integration(gp, int(IG, c_int32_t), int(IDP, c_int32_t), omgx, omgy, omgz), &
                'EULER_INTEGRATION')
end subroutine EULER_INTEGRATION


! ADV_PARTICLE_ELLP(NCYCLE)  adv_particle_new.f90:7-704, on the device-resident state
subroutine ADV_PARTICLE_ELLP(NCYCLE)
  use iso_c_binding
  use gazpart_gpu
  use gazpart_gpu_iface_state
  implicit none
  integer, intent(in) :: NCYCLE
  call gp_check(gp_adv_particle_ellp(gp, int(NCYCLE, c_int32_t)), 'ADV_PARTICLE_ELLP')
end subroutine ADV_PARTICLE_ELLP


! COLLISION(NCYCLE, TIME)  collision.f90:7-200 (NPROC = 1), on the device-resident state
subroutine COLLISION(NCYCLE, TIME)
  use iso_c_binding
  use gazpart_gpu
  use gazpart_gpu_iface_state
  implicit none
  integer, intent(in) :: NCYCLE
  real(kind=8), intent(in) :: TIME
  call gp_check(gp_collision(gp, int(NCYCLE, c_int32_t), TIME, c_null_ptr, c_null_ptr, c_null_ptr), 'COLLISION')
end subroutine COLLISION


! ellipsoid_contact_detection  ellipsoid_contact_detection.f90:1-187 (lmder1 inside)
subroutine ellipsoid_contact_detection(IG, IDP1, IDP2, IXP, IYP, IZP, IQUAT, JXP, JYP, JZP, JQUAT, &
                                       flag, EPT1, EPT2, cnormal)
  use iso_c_binding
  use gazpart_gpu
  use gazpart_gpu_iface_state
  use mod_quaternion, only: quaternion
  implicit none
  integer, intent(in) :: IG, IDP1, IDP2
  real(kind=8), intent(in) :: IXP, IYP, IZP, JXP, JYP, JZP
  type(quaternion), intent(in) :: IQUAT, JQUAT
  logical, intent(inout) :: flag
  real(kind=8), dimension(3, 1), intent(inout) :: EPT1, EPT2, cnormal
  integer(c_int32_t) :: f
  real(c_double) :: e1(3), e2(3), cn(3)
  call ensure_ctx()
  call gp_check(gp_ellipsoid_contact_detection(gp, int(IG, c_int32_t), int(IDP1, c_int32_t), int(IDP2, c_int32_t), &
                IXP, IYP, IZP, (/IQUAT%a, IQUAT%b, IQUAT%c, IQUAT%d/), JXP, JYP, JZP, &
                (/JQUAT%a, JQUAT%b, JQUAT%c, JQUAT%d/), f, e1, e2, cn), 'ellipsoid_contact_detection')
  flag = (f /= 0)
  EPT1(:, 1) = e1
  EPT2(:, 1) = e2
  cnormal(:, 1) = cn
end subroutine ellipsoid_contact_detection


! COLLISION_RESPONSE(IG, IDP, part1, part2, R_impact1, R_impact2, normal)
! collision_response.f90:1-437: the inertia of class (IG, IDP) for both bodies (Q8).
subroutine COLLISION_RESPONSE(IG, IDP, part1, part2, R_impact1, R_impact2, normal)
  use iso_c_binding
  use gazpart_gpu
  use gazpart_gpu_iface_state
  use PARTICLE_PARALLEL, only: PARTTYPE
  implicit none
  integer, intent(in) :: IG, IDP
  type(PARTTYPE), intent(inout) :: part1, part2
  real(kind=8), dimension(3, 1), intent(in) :: R_impact1, R_impact2, normal
  real(c_double) :: p1(10), p2(10)
  call ensure_ctx()
  p1 = (/part1%UP, part1%VP, part1%WP, part1%OMEGAX, part1%OMEGAY, part1%OMEGAZ, &
         part1%ELLQUAT%a, part1%ELLQUAT%b, part1%ELLQUAT%c, part1%ELLQUAT%d/)
  p2 = (/part2%UP, part2%VP, part2%WP, part2%OMEGAX, part2%OMEGAY, part2%OMEGAZ, &
         part2%ELLQUAT%a, part2%ELLQUAT%b, part2%ELLQUAT%c, part2%ELLQUAT%d/)
  call gp_check(gp_collision_response(gp, int(IG, c_int32_t), int(IDP, c_int32_t), p1, p2, &
                R_impact1(:, 1), R_impact2(:, 1), normal(:, 1)), 'COLLISION_RESPONSE')
  part1%UP = p1(1); part1%VP = p1(2); part1%WP = p1(3)
  part1%OMEGAX = p1(4); part1%OMEGAY = p1(5); part1%OMEGAZ = p1(6)
  part2%UP = p2(1); part2%VP = p2(2); part2%WP = p2(3)
  part2%OMEGAX = p2(4); part2%OMEGAY = p2(5); part2%OMEGAZ = p2(6)
end subroutine COLLISION_RESPONSE


! The device state back into PART(1:NPART_LOC(J), J), with the fluid values of the last
! step (UFAP..VORTZAP): before statistics, snapshots and restart files read PART.
subroutine GAZPART_GPU_SYNC
  use iso_c_binding
  use gazpart_gpu
  use gazpart_gpu_iface_state
  use DNS_DIM, only: NIG, NPART_LOC
  use PARTICLE_PARALLEL, only: PART
  implicit none
  type(c_ptr) :: pc(13), pf(6)
  integer :: j, i, c
  integer(c_int64_t) :: k
  call col_ptrs(pc)
  do c = 1, 6
     pf(c) = c_loc(fluid(1, c))
  end do
  call gp_check(gp_download_state(gp, ntot, pc, pf, 0_c_int32_t), 'GAZPART_GPU_SYNC')
  k = 0
  do j = 1, NIG
     do i = 1, NPART_LOC(j)
        k = k + 1
        PART(i, j)%XP = cols(k, 1); PART(i, j)%YP = cols(k, 2); PART(i, j)%ZP = cols(k, 3)
        PART(i, j)%UP = cols(k, 4); PART(i, j)%VP = cols(k, 5); PART(i, j)%WP = cols(k, 6)
        PART(i, j)%ELLQUAT%a = cols(k, 7); PART(i, j)%ELLQUAT%b = cols(k, 8)
        PART(i, j)%ELLQUAT%c = cols(k, 9); PART(i, j)%ELLQUAT%d = cols(k, 10)
        PART(i, j)%OMEGAX = cols(k, 11); PART(i, j)%OMEGAY = cols(k, 12); PART(i, j)%OMEGAZ = cols(k, 13)
        PART(i, j)%UFAP = fluid(k, 1); PART(i, j)%VFAP = fluid(k, 2); PART(i, j)%WFAP = fluid(k, 3)
        PART(i, j)%VORTXAP = fluid(k, 4); PART(i, j)%VORTYAP = fluid(k, 5); PART(i, j)%VORTZAP = fluid(k, 6)
     end do
  end do
end subroutine GAZPART_GPU_SYNC


! PART back to the device after the host changed it (same particles, same classes).
subroutine GAZPART_GPU_PUT
  use iso_c_binding
  use gazpart_gpu
  use gazpart_gpu_iface_state
  implicit none
  type(c_ptr) :: pc(13)
  call pack_part()
  call col_ptrs(pc)
  call gp_check(gp_put_state(gp, ntot, pc, 0_c_int32_t), 'GAZPART_GPU_PUT')
end subroutine GAZPART_GPU_PUT


! The field arrays have new values (DNS mode, after ADV_FLUID): reload them.
subroutine GAZPART_GPU_FIELDS_CHANGED
  use iso_c_binding
  use gazpart_gpu
  use gazpart_gpu_iface_state
  use FLUID_VARIABLE, only: UFLU, VFLU, WFLU
  implicit none
  ! the velocity slots only: the vorticity arrays keep their values in DNS mode
  field_src(1:3) = c_null_ptr
  call load_field(0, UFLU)
  call load_field(1, VFLU)
  call load_field(2, WFLU)
end subroutine GAZPART_GPU_FIELDS_CHANGED
