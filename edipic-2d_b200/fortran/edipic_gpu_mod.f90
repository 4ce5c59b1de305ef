!------------------------------------------------------------------------------------------------------------
! ISO_C_BINDING interface of libedipic_b200.so (include/edipic_gpu.h) for the EDIPIC-2D Fortran host.
!
! The host keeps its decks, its set-up and its diagnostics; the per-step particle cycle is replaced by the
! calls below, made from MainProg (src/pic2d_MainProgram.f90:151-309) in place of the subroutines named beside
! each one. edp_ctx is an opaque C pointer held in a module variable. No Fortran compiler is available where
! this file was written; it follows the Fortran 2003 C-interoperability rules and the C header field by field.
!------------------------------------------------------------------------------------------------------------
module edipic_gpu
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: EDP_ABI_VERSION = 2
  integer(c_int), parameter :: EDP_MAX_ION_SPECIES = 4, EDP_MAX_INNER = 4, EDP_MAX_COLPROC = 8, EDP_MAX_SEGMENTS = 32
  integer(c_int), parameter :: EDP_PREC_MIXED = 0, EDP_PREC_FP64 = 1, EDP_SOLVER_FFTX = 0, EDP_SOLVER_CG = 1
  integer(c_int), parameter :: EDP_ELECTRONS = 0, EDP_IONS = 1
  integer(c_int), parameter :: EDP_WARM_ZERO = 0, EDP_WARM_PREVIOUS = 1, EDP_WARM_LEARNED = 3
  integer(c_int), parameter :: EDP_PRECOND_NONE = 0, EDP_PRECOND_MG = 1

  type, bind(C) :: edp_params
     integer(c_int32_t) :: abi_version, ncx, ncy, periodic_x, n_subcycles, n_of_particles_cell
     real(c_double) :: delta_t_s, delta_x_m, v_scale_ms, e_scale_vm, b_scale_t, f_scale_v
     real(c_double) :: bx, by, bz, ez
     integer(c_int32_t) :: ions_sense_b, ions_sense_ez, n_ion_species
     integer(c_int32_t) :: ion_charge(EDP_MAX_ION_SPECIES)
     real(c_double) :: ion_mass_me(EDP_MAX_ION_SPECIES)
     real(c_double) :: wall_phi_const(4), wall_phi_var(4), wall_omega(4), wall_phase(4)
     integer(c_int32_t) :: n_inner
     integer(c_int32_t) :: inner_ileft(EDP_MAX_INNER), inner_jbottom(EDP_MAX_INNER)
     integer(c_int32_t) :: inner_iright(EDP_MAX_INNER), inner_jtop(EDP_MAX_INNER)
     real(c_double) :: inner_phi(EDP_MAX_INNER)
     integer(c_int64_t) :: seed
     integer(c_int32_t) :: precision, solver, sort_every, fuse_collisions
     integer(c_int64_t) :: capacity(1 + EDP_MAX_ION_SPECIES)
     real(c_double) :: inner_eps(EDP_MAX_INNER)      ! 0 metal, > 0 dielectric permittivity
  end type edp_params

  type, bind(C) :: edp_tables
     integer(c_int32_t) :: en_on, n_act, n_seg, n_values
     real(c_double) :: seg_value(EDP_MAX_SEGMENTS + 1), seg_step(EDP_MAX_SEGMENTS)
     integer(c_int32_t) :: seg_index(EDP_MAX_SEGMENTS + 1)
     type(c_ptr) :: energy_eV, prob            ! collision_e_neutral(1)%energy_eV, %prob_colproc_energy
     real(c_double) :: max_colliding_fraction
     integer(c_int32_t) :: colproc_type(EDP_MAX_COLPROC)
     real(c_double) :: threshold_eV(EDP_MAX_COLPROC)
     integer(c_int32_t) :: ion_species_produced(EDP_MAX_COLPROC)
     real(c_double) :: ion_velocity_factor(EDP_MAX_COLPROC)
     real(c_double) :: neutral_mass_amu, energy_factor_eV
     integer(c_int32_t) :: rcx_on(EDP_MAX_ION_SPECIES)
     real(c_double) :: rcx_prob_factor, rcx_sigma_1eV, rcx_alpha
     real(c_double) :: rcx_probab_thermal(EDP_MAX_ION_SPECIES), rcx_vfactor(EDP_MAX_ION_SPECIES)
     integer(c_int32_t) :: maxwell_rmax
     type(c_ptr) :: maxwell_v                  ! MaxwellVelocity%v(0:R_max)
  end type edp_tables

  type, bind(C) :: edp_counters
     integer(c_int64_t) :: n_particles(1 + EDP_MAX_ION_SPECIES)
     integer(c_int64_t) :: electron_hits(4 + EDP_MAX_INNER), ion_hits(4 + EDP_MAX_INNER)
     integer(c_int64_t) :: en_collisions(EDP_MAX_COLPROC), rcx_collisions(EDP_MAX_ION_SPECIES)
     integer(c_int64_t) :: step
     integer(c_int32_t) :: cg_iterations
     real(c_double) :: cg_relres
     integer(c_int32_t) :: error_flags
     integer(c_int64_t) :: kernel_launches
  end type edp_counters

  interface
     integer(c_int) function edp_init(p, t, ctx) bind(C, name="edp_init")
       import :: edp_params, edp_tables, c_ptr, c_int
       type(edp_params), intent(in) :: p
       type(edp_tables), intent(in) :: t
       type(c_ptr), intent(out) :: ctx
     end function edp_init
     integer(c_int) function edp_destroy(ctx) bind(C, name="edp_destroy")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
     end function edp_destroy
     integer(c_int) function edp_upload_particles(ctx, species, n, x, y, vx, vy, vz, tag, id) &
          bind(C, name="edp_upload_particles")
       import :: c_ptr, c_int, c_int64_t, c_double, c_int32_t
       type(c_ptr), value :: ctx
       integer(c_int), value :: species
       integer(c_int64_t), value :: n
       real(c_double), intent(in) :: x(*), y(*), vx(*), vy(*), vz(*)
       integer(c_int32_t), intent(in) :: tag(*)
       type(c_ptr), value :: id
     end function edp_upload_particles
     integer(c_int) function edp_download_particles(ctx, species, cap, n_out, x, y, vx, vy, vz, tag, id) &
          bind(C, name="edp_download_particles")
       import :: c_ptr, c_int, c_int64_t, c_double, c_int32_t
       type(c_ptr), value :: ctx
       integer(c_int), value :: species
       integer(c_int64_t), value :: cap
       integer(c_int64_t), intent(out) :: n_out
       real(c_double), intent(out) :: x(*), y(*), vx(*), vy(*), vz(*)
       integer(c_int32_t), intent(out) :: tag(*)
       type(c_ptr), value :: id
     end function edp_download_particles
     integer(c_int) function edp_gather_charge_density(ctx, species, rho_out) bind(C, name="edp_gather_charge_density")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       integer(c_int), value :: species
       type(c_ptr), value :: rho_out
     end function edp_gather_charge_density
     integer(c_int) function edp_update_wall_potentials(ctx, t_cntr) bind(C, name="edp_update_wall_potentials")
       import :: c_ptr, c_int, c_int64_t
       type(c_ptr), value :: ctx
       integer(c_int64_t), value :: t_cntr
     end function edp_update_wall_potentials
     integer(c_int) function edp_field_fftx(ctx, phi_out) bind(C, name="edp_field_fftx")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx, phi_out
     end function edp_field_fftx
     integer(c_int) function edp_field_cg(ctx, rtol, max_it, warm_start, iters_out) bind(C, name="edp_field_cg")
       import :: c_ptr, c_int, c_double, c_int32_t
       type(c_ptr), value :: ctx
       real(c_double), value :: rtol
       integer(c_int32_t), value :: max_it, warm_start
       integer(c_int32_t), intent(out) :: iters_out
     end function edp_field_cg
     integer(c_int) function edp_advance_electrons(ctx) bind(C, name="edp_advance_electrons")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
     end function edp_advance_electrons
     integer(c_int) function edp_advance_ions(ctx) bind(C, name="edp_advance_ions")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
     end function edp_advance_ions
     integer(c_int) function edp_collide_en(ctx, counters_out) bind(C, name="edp_collide_en")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx, counters_out
     end function edp_collide_en
     integer(c_int) function edp_collide_rcx(ctx, count_out) bind(C, name="edp_collide_rcx")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx, count_out
     end function edp_collide_rcx
     integer(c_int) function edp_end_ion_cycle(ctx) bind(C, name="edp_end_ion_cycle")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
     end function edp_end_ion_cycle
     integer(c_int) function edp_set_cg_preconditioner(ctx, kind) bind(C, name="edp_set_cg_preconditioner")
       import :: c_ptr, c_int, c_int32_t
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: kind
     end function edp_set_cg_preconditioner
     ! PREPARE_WALL_MATERIALS (pic2d_Materials.f90:150-188) passes each wall's ion-induced emission here
     integer(c_int) function edp_set_ion_emission(ctx, wall, ion_species, yield, emin_ev, emax_ev, t_emit_ev) &
          bind(C, name="edp_set_ion_emission")
       import :: c_ptr, c_int, c_int32_t, c_double
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: wall, ion_species
       real(c_double), value :: yield, emin_ev, emax_ev, t_emit_ev
     end function edp_set_ion_emission
     integer(c_int) function edp_query_emission(ctx, counts) bind(C, name="edp_query_emission")
       import :: c_ptr, c_int, c_int64_t
       type(c_ptr), value :: ctx
       integer(c_int64_t), intent(out) :: counts(*)
     end function edp_query_emission
     ! READ_A_CHECKPOINT: the continued run's next step is Start_T_cntr
     integer(c_int) function edp_set_step(ctx, t_cntr) bind(C, name="edp_set_step")
       import :: c_ptr, c_int, c_int64_t
       type(c_ptr), value :: ctx
       integer(c_int64_t), value :: t_cntr
     end function edp_set_step
     ! electron-induced emission of a wall: see = edp_see_params filled from the material file (eV)
     integer(c_int) function edp_set_electron_emission(ctx, wall, see) bind(C, name="edp_set_electron_emission")
       import :: c_ptr, c_int, c_int32_t
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: wall
       type(c_ptr), value :: see              ! c_loc of an interoperable copy of edp_see_params, or c_null_ptr
     end function edp_set_electron_emission
     ! PERFORM_ELECTRON_EMISSION_SETUP of a wall (init_bo_NN.dat lines 11-20)
     integer(c_int) function edp_set_wall_injection(ctx, wall, n_per_step, model, t_normal_ev, t_parallel_ev, &
          beam_energy_ev) bind(C, name="edp_set_wall_injection")
       import :: c_ptr, c_int, c_int32_t, c_double
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: wall, model
       real(c_double), value :: n_per_step, t_normal_ev, t_parallel_ev, beam_energy_ev
     end function edp_set_wall_injection
     ! ion-material model 1 (specular reflection) of a wall
     integer(c_int) function edp_set_ion_reflection(ctx, wall, on) bind(C, name="edp_set_ion_reflection")
       import :: c_ptr, c_int, c_int32_t
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: wall, on
     end function edp_set_ion_reflection
     ! CALCULATE_ELECTRON_VDF / CALCULATE_ION_VDF: evdf1d(bins, box, 3) in Fortran order, evxvydf(vx, vy, box)
     integer(c_int) function edp_calculate_vdf(ctx, species, n_max_vel, nbox_x, nbox_y, n_max_vel_s, n_vbins, &
          vdf1d, vdf2d, skipped) bind(C, name="edp_calculate_vdf")
       import :: c_ptr, c_int, c_int32_t, c_int64_t
       type(c_ptr), value :: ctx
       integer(c_int), value :: species
       integer(c_int32_t), value :: n_max_vel, nbox_x, nbox_y, n_max_vel_s, n_vbins
       integer(c_int32_t), intent(out) :: vdf1d(*)
       type(c_ptr), value :: vdf2d            ! c_loc(evxvydf) or c_null_ptr
       integer(c_int64_t), intent(out) :: skipped
     end function edp_calculate_vdf
     integer(c_int) function edp_warmstart_load(ctx, blob, n) bind(C, name="edp_warmstart_load")
       import :: c_ptr, c_int, c_int64_t, c_float
       type(c_ptr), value :: ctx
       real(c_float), intent(in) :: blob(*)
       integer(c_int64_t), value :: n
     end function edp_warmstart_load
     integer(c_int) function edp_collect_moments(ctx, species, out) bind(C, name="edp_collect_moments")
       import :: c_ptr, c_int, c_float
       type(c_ptr), value :: ctx
       integer(c_int), value :: species
       real(c_float), intent(out) :: out(*)
     end function edp_collect_moments
     ! re-sort the particles by tile now (restarts the sort period); results do not depend on it
     integer(c_int) function edp_sort_particles(ctx) bind(C, name="edp_sort_particles")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
     end function edp_sort_particles
     ! ids of the particles this context creates stay in [base, end): ranks of one cluster take disjoint ranges
     integer(c_int) function edp_set_id_range(ctx, base, end) bind(C, name="edp_set_id_range")
       import :: c_ptr, c_int, c_int64_t
       type(c_ptr), value :: ctx
       integer(c_int64_t), value :: base, end
     end function edp_set_id_range
     ! x strips of a periodic domain (one cluster per strip along x, pic2d_ParticleExchange.f90); the record and
     ! density buffers are device memory the host allocates (cudaMalloc through its CUDA Fortran or C layer)
     integer(c_int) function edp_set_strip(ctx, ghost_left, ghost_right, x_first, ncx_global, periodic) &
          bind(C, name="edp_set_strip")
       import :: c_ptr, c_int, c_int32_t
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: ghost_left, ghost_right, x_first, ncx_global, periodic
     end function edp_set_strip
     integer(c_int) function edp_strip_take(ctx, species, left, cap_left, right, cap_right, n_left, n_right) &
          bind(C, name="edp_strip_take")
       import :: c_ptr, c_int, c_int32_t, c_int64_t
       type(c_ptr), value :: ctx, left, right
       integer(c_int32_t), value :: species
       integer(c_int64_t), value :: cap_left, cap_right
       integer(c_int64_t), intent(out) :: n_left, n_right
     end function edp_strip_take
     integer(c_int) function edp_strip_put(ctx, species, records, n, x_shift) bind(C, name="edp_strip_put")
       import :: c_ptr, c_int, c_int32_t, c_int64_t, c_double
       type(c_ptr), value :: ctx, records
       integer(c_int32_t), value :: species
       integer(c_int64_t), value :: n
       real(c_double), value :: x_shift
     end function edp_strip_put
     integer(c_int) function edp_strip_add_density(ctx, species, global_dev, nx_global, x_first) &
          bind(C, name="edp_strip_add_density")
       import :: c_ptr, c_int, c_int32_t
       type(c_ptr), value :: ctx, global_dev
       integer(c_int32_t), value :: species, nx_global, x_first
     end function edp_strip_add_density
     integer(c_int) function edp_strip_set_field(ctx, e_global, acc_global, nx_global, x_first) &
          bind(C, name="edp_strip_set_field")
       import :: c_ptr, c_int, c_int32_t
       type(c_ptr), value :: ctx, e_global, acc_global
       integer(c_int32_t), value :: nx_global, x_first
     end function edp_strip_set_field
     integer(c_int) function edp_device_buffer(ctx, which, species, ptr, count) bind(C, name="edp_device_buffer")
       import :: c_ptr, c_int, c_int32_t, c_int64_t
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: which, species
       type(c_ptr), intent(out) :: ptr
       integer(c_int64_t), intent(out) :: count
     end function edp_device_buffer
     integer(c_int) function edp_query_counters(ctx, c) bind(C, name="edp_query_counters")
       import :: c_ptr, c_int, edp_counters
       type(c_ptr), value :: ctx
       type(edp_counters), intent(out) :: c
     end function edp_query_counters
  end interface

  type(c_ptr), save :: edp_context = c_null_ptr

contains

  ! Argument-less wrappers with the names of the subroutines they stand in for, so MainProg's calls keep their
  ! shape. The deposit is fused into the pushes, so the two GATHER_* calls only refresh the host copies when a
  ! diagnostic needs them.
  subroutine GPU_GATHER_ELECTRON_CHARGE_DENSITY
    integer(c_int) :: rc
    rc = edp_gather_charge_density(edp_context, EDP_ELECTRONS, c_null_ptr)
    call edp_check(rc, 'GATHER_ELECTRON_CHARGE_DENSITY')
  end subroutine GPU_GATHER_ELECTRON_CHARGE_DENSITY

  subroutine GPU_SOLVE_POISSON_FFTX_LINSYSY
    integer(c_int) :: rc
    rc = edp_field_fftx(edp_context, c_null_ptr)
    call edp_check(rc, 'SOLVE_POISSON_FFTX_LINSYSY')
  end subroutine GPU_SOLVE_POISSON_FFTX_LINSYSY

  subroutine GPU_ADVANCE_ELECTRONS
    call edp_check(edp_advance_electrons(edp_context), 'ADVANCE_ELECTRONS')
  end subroutine GPU_ADVANCE_ELECTRONS

  subroutine GPU_ADVANCE_IONS
    call edp_check(edp_advance_ions(edp_context), 'ADVANCE_IONS')
  end subroutine GPU_ADVANCE_IONS

  subroutine GPU_PERFORM_ELECTRON_NEUTRAL_COLLISIONS
    call edp_check(edp_collide_en(edp_context, c_null_ptr), 'PERFORM_ELECTRON_NEUTRAL_COLLISIONS')
  end subroutine GPU_PERFORM_ELECTRON_NEUTRAL_COLLISIONS

  subroutine GPU_PERFORM_RESONANT_CHARGE_EXCHANGE
    call edp_check(edp_collide_rcx(edp_context, c_null_ptr), 'PERFORM_RESONANT_CHARGE_EXCHANGE')
  end subroutine GPU_PERFORM_RESONANT_CHARGE_EXCHANGE

  ! COLLECT_ELECTRON_MOMENTS (and the moments branch of ADVANCE_ELECTRONS_PLUS, called before the push on a
  ! snapshot step): the 13 grids cs_N, cs_VX, ... cs_QZ, each (c_indx_x_min:c_indx_x_max, c_indx_y_min:c_indx_y_max)
  subroutine GPU_COLLECT_ELECTRON_MOMENTS(moments)
    real(c_float), intent(out) :: moments(:,:,:)   ! (nodes x, nodes y, 13)
    call edp_check(edp_collect_moments(edp_context, EDP_ELECTRONS, moments), 'COLLECT_ELECTRON_MOMENTS')
  end subroutine GPU_COLLECT_ELECTRON_MOMENTS

  ! called at the end of every time step: on ion steps it is PROCESS_ADDED_IONS + CLEAR_ACCUMULATED_FIELDS,
  ! on every step it moves the ionisation add list and advances T_cntr
  subroutine GPU_END_OF_STEP
    call edp_check(edp_end_ion_cycle(edp_context), 'END_OF_STEP')
  end subroutine GPU_END_OF_STEP

  subroutine edp_check(rc, where)
    integer(c_int), intent(in) :: rc
    character(*), intent(in) :: where
    if (rc /= 0) then
       print '("edipic_gpu: ",A," returned ",i4)', where, rc
       stop 1
    end if
  end subroutine edp_check

end module edipic_gpu
