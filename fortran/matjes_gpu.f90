! Fortran 2008 binding (iso_c_binding) of include/matjes_gpu.h, the C ABI of
! the B200 spin-dynamics library libmatjes_b200.so.
!
! The module a Matjes maintainer adds to the Fortran tree to reach the library,
! in the style of the reference's own CUDA bindings
! (src/Hamiltonian_type/cuda_H_interface.f90:5-87,
! src/Hamiltonian_type/cuda_fft_interface.f90:5-88): derived types with
! bind(c) mirror the C structs field by field, opaque handles are type(c_ptr),
! scalars are passed by value, arrays by reference.  Host spin arrays keep the
! reference layout modes_v(3, N) (AoS, component fastest); device arrays are
! type(c_ptr) to SoA blocks of 3N doubles.  Every function returns an
! mj_status (0 = MJ_OK); mj_error_message() gives the text of the last failure.
!
! Build: gfortran -c matjes_gpu.f90, link with -L<dir> -lmatjes_b200.
module m_matjes_gpu
  use, intrinsic :: iso_c_binding
  implicit none
  private :: c_strlen

  ! ---- status codes and enumerations (matjes_gpu.h) ----
  integer(c_int32_t), parameter :: MJ_OK = 0, MJ_ERR_ARG = 1, MJ_ERR_OOM = 2, MJ_ERR_CUDA = 3, &
                                   MJ_ERR_TIMEOUT = 4, MJ_ERR_NAN = 5, MJ_ERR_UNSUPPORTED = 6, &
                                   MJ_ERR_GEOMETRY = 7
  integer(c_int32_t), parameter :: MJ_EULER = 1, MJ_HEUN_MATJES = 2, MJ_SIB = 3
  integer(c_int32_t), parameter :: MJ_NOISE_OFF = 0, MJ_NOISE_PHILOX = 1, MJ_NOISE_INJECT = 2
  integer(c_int32_t), parameter :: MJ_ENERGY_AFTER = 0, MJ_ENERGY_BEFORE = 1
  integer(c_int32_t), parameter :: MJ_MAX_ATOMS = 16
  integer(c_int32_t), parameter :: MJ_MC_CONE = 0, MJ_MC_ISING = 1, MJ_MC_UNDERRELAX = 2, MJ_MC_OVERRELAX = 3
  integer(c_int32_t), parameter :: MJ_OPT_TMA = 0, MJ_OPT_FUSED = 1, MJ_OPT_PDL = 2, MJ_OPT_STORE_DRAW = 3, &
                                   MJ_OPT_HOST_STRIPES = 4, MJ_OPT_BLOCKS_PER_SM = 5, MJ_OPT_DIP_ZCONV = 6, &
                                   MJ_OPT_HOST_ZEROCOPY = 7

  ! ---- descriptors ----
  ! Nsize, Periodic_log, lattice (areal(:, j) = lattice vector j in nm, alat
  ! applied), atoms (fractional positions, type, moment in mu_B)
  type, bind(c) :: mj_lattice_desc
    integer(c_int32_t) :: L(3), periodic(3)
    real(c_double)     :: areal(3, 3)
    integer(c_int32_t) :: natom
    real(c_double)     :: frac(3, MJ_MAX_ATOMS)
    integer(c_int32_t) :: attype(MJ_MAX_ATOMS)
    real(c_double)     :: moment(MJ_MAX_ATOMS)
  end type
  ! magnetic_J t1 t2 shell J
  type, bind(c) :: mj_exchange_term
    integer(c_int32_t) :: t1, t2, shell
    real(c_double)     :: value
  end type
  ! magnetic_D t1 t2 mediator shell D
  type, bind(c) :: mj_dmi_term
    integer(c_int32_t) :: t1, t2, tmed, shell
    real(c_double)     :: value
  end type
  ! magnetic_anisotropy type ex ey ez K (an easy axis is a negative K)
  type, bind(c) :: mj_aniso_term
    integer(c_int32_t) :: type
    real(c_double)     :: axis(3), value
  end type
  ! J, D, K point at arrays of the term types above (c_loc of a target array)
  type, bind(c) :: mj_hamiltonian_desc
    integer(c_int32_t) :: nJ
    type(c_ptr)        :: J = c_null_ptr
    integer(c_int32_t) :: nD
    type(c_ptr)        :: D = c_null_ptr
    integer(c_int32_t) :: nK
    type(c_ptr)        :: K = c_null_ptr
    real(c_double)     :: c_H_J = -1.0_c_double, c_H_D = -1.0_c_double, c_H_ani = 1.0_c_double, &
                          c_zeeman = -1.0_c_double
    real(c_double)     :: B_ext(3) = 0.0_c_double
    integer(c_int32_t) :: zeeman_on = 0, dip_on = 0
    integer(c_int32_t) :: dip_period_cut(3) = 1
  end type
  ! one time-step call; seed, stream_id and step0 are unsigned in C
  type, bind(c) :: mj_dyn_params
    integer(c_int32_t) :: integrator = MJ_SIB
    real(c_double)     :: timestep = 0.1_c_double, alpha = 0.1_c_double, temperature = 0.0_c_double
    integer(c_int32_t) :: noise = MJ_NOISE_OFF
    integer(c_int64_t) :: seed = 0
    integer(c_int32_t) :: stream_id = 0, step0 = 0
    type(c_ptr)        :: inject = c_null_ptr
    integer(c_int32_t) :: inject_nbuf = 0, energy_mode = MJ_ENERGY_AFTER
  end type
  ! minimize_run / minimize_infdamp_run (masse, timestep, convergence_criteria)
  type, bind(c) :: mj_min_params
    real(c_double)     :: timestep, mass, conv_torque
    integer(c_int32_t) :: check_every
  end type
  ! MC_input + track_val; seed / stream_id / sweep0 unsigned in C
  type, bind(c) :: mj_mc_params
    real(c_double)     :: temperature, cone
    integer(c_int32_t) :: proposal, adapt_cone
    integer(c_int64_t) :: seed
    integer(c_int32_t) :: stream_id, sweep0
    integer(c_int64_t) :: accepted_total, proposed_total
    integer(c_int32_t) :: round0, track_totals
  end type

  interface
    ! ---- errors ----
    type(c_ptr) function mj_last_error() bind(c, name="mj_last_error")
      import
    end function
    ! ---- plans ----
    integer(c_int32_t) function mj_plan_create(lat, ham, device, plan) bind(c, name="mj_plan_create")
      import
      type(mj_lattice_desc), intent(in) :: lat
      type(mj_hamiltonian_desc), intent(in) :: ham
      integer(c_int32_t), value :: device
      type(c_ptr), intent(out) :: plan
    end function
    integer(c_int32_t) function mj_plan_from_coo(nsites, nnz, rows, cols, vals, base, zeeman, b_cell, device, plan) &
        bind(c, name="mj_plan_from_coo")
      import
      integer(c_int64_t), value :: nsites, nnz
      integer(c_int64_t), intent(in) :: rows(*), cols(*)
      real(c_double), intent(in) :: vals(*), zeeman(*), b_cell(*)
      integer(c_int32_t), value :: base, device
      type(c_ptr), intent(out) :: plan
    end function
    integer(c_int32_t) function mj_plan_destroy(plan) bind(c, name="mj_plan_destroy")
      import
      type(c_ptr), value :: plan
    end function
    integer(c_int32_t) function mj_plan_nsites(plan, n) bind(c, name="mj_plan_nsites")
      import
      type(c_ptr), value :: plan
      integer(c_int64_t), intent(out) :: n
    end function
    integer(c_int32_t) function mj_plan_check_status(plan) bind(c, name="mj_plan_check_status")
      import
      type(c_ptr), value :: plan
    end function
    integer(c_int32_t) function mj_plan_set_option(plan, option, value) bind(c, name="mj_plan_set_option")
      import
      type(c_ptr), value :: plan
      integer(c_int32_t), value :: option, value
    end function
    integer(c_int32_t) function mj_plan_set_bfield(plan, b_cell) bind(c, name="mj_plan_set_bfield")
      import
      type(c_ptr), value :: plan
      real(c_double), intent(in) :: b_cell(3, *)
    end function
    integer(c_int32_t) function mj_plan_autotune(plan, m_dev, p, steps, best, best_tma, ms_per_step) &
        bind(c, name="mj_plan_autotune")
      import
      type(c_ptr), value :: plan, m_dev, ms_per_step
      type(mj_dyn_params), intent(in) :: p
      integer(c_int32_t), value :: steps
      integer(c_int32_t), intent(out) :: best, best_tma
    end function
    ! ---- device-resident spins ----
    integer(c_int32_t) function mj_state_create(plan, st) bind(c, name="mj_state_create")
      import
      type(c_ptr), value :: plan
      type(c_ptr), intent(out) :: st
    end function
    integer(c_int32_t) function mj_state_destroy(st) bind(c, name="mj_state_destroy")
      import
      type(c_ptr), value :: st
    end function
    integer(c_int32_t) function mj_state_upload(st, m, stream) bind(c, name="mj_state_upload")
      import
      type(c_ptr), value :: st, stream
      real(c_double), intent(in) :: m(3, *)
    end function
    integer(c_int32_t) function mj_state_download(st, m, stream) bind(c, name="mj_state_download")
      import
      type(c_ptr), value :: st, stream
      real(c_double), intent(out) :: m(3, *)
    end function
    integer(c_int32_t) function mj_state_device_ptr(st, m_dev) bind(c, name="mj_state_device_ptr")
      import
      type(c_ptr), value :: st
      type(c_ptr), intent(out) :: m_dev
    end function
    ! ---- field and energy (get_eff_field, H%energy, energy_distrib) ----
    integer(c_int32_t) function mj_field_host(plan, m, B, e_site) bind(c, name="mj_field_host")
      import
      type(c_ptr), value :: plan
      real(c_double), intent(in) :: m(3, *)
      real(c_double), intent(out) :: B(3, *), e_site(*)
    end function
    integer(c_int32_t) function mj_field(plan, st, B_dev, e_site_dev, stream) bind(c, name="mj_field")
      import
      type(c_ptr), value :: plan, st, B_dev, e_site_dev, stream
    end function
    integer(c_int32_t) function mj_energy(plan, st, E) bind(c, name="mj_energy")
      import
      type(c_ptr), value :: plan, st
      real(c_double), intent(out) :: E
    end function
    ! ---- time steps (the stage loop of spindynamics_run) ----
    integer(c_int32_t) function mj_step(plan, st, p, nsteps, E_dev, stream) bind(c, name="mj_step")
      import
      type(c_ptr), value :: plan, st, E_dev, stream
      type(mj_dyn_params), intent(in) :: p
      integer(c_int32_t), value :: nsteps
    end function
    integer(c_int32_t) function mj_step_host(plan, m, p, nsteps, E) bind(c, name="mj_step_host")
      import
      type(c_ptr), value :: plan
      real(c_double), intent(inout) :: m(3, *)
      type(mj_dyn_params), intent(in) :: p
      integer(c_int32_t), value :: nsteps
      real(c_double), intent(out) :: E(*)
    end function
    integer(c_int32_t) function mj_graph_run(plan, st, p, nsteps, nreplay, E_dev, stream) bind(c, name="mj_graph_run")
      import
      type(c_ptr), value :: plan, st, E_dev, stream
      type(mj_dyn_params), intent(in) :: p
      integer(c_int32_t), value :: nsteps, nreplay
    end function
    integer(c_int32_t) function mj_measure_temperature(plan, st, T) bind(c, name="mj_measure_temperature")
      import
      type(c_ptr), value :: plan, st
      real(c_double), intent(out) :: T
    end function
    ! ---- minimisation (minimize_run, minimize_infdamp_run) ----
    integer(c_int32_t) function mj_minimize(plan, m_dev, p, max_iter, iterations, max_torque, stream) &
        bind(c, name="mj_minimize")
      import
      type(c_ptr), value :: plan, m_dev, stream
      type(mj_min_params), intent(in) :: p
      integer(c_int64_t), value :: max_iter
      integer(c_int64_t), intent(out) :: iterations
      real(c_double), intent(out) :: max_torque
    end function
    ! ---- Monte Carlo (montecarlo_run's sweeps) ----
    integer(c_int32_t) function mj_mc_sweeps(plan, m_dev, p, nsweeps, E_dev, M_dev, accepted, colors, stream) &
        bind(c, name="mj_mc_sweeps")
      import
      type(c_ptr), value :: plan, m_dev, E_dev, M_dev, stream
      type(mj_mc_params), intent(inout) :: p
      integer(c_int32_t), value :: nsweeps
      integer(c_int64_t), intent(out) :: accepted
      integer(c_int32_t), intent(out) :: colors(4)
    end function
    ! ---- replica batches (parallel tempering ladders, field sweeps, GNEB images) ----
    integer(c_int32_t) function mj_batch_create(cell, ham, nrep, L, B_ext, T, device, b) bind(c, name="mj_batch_create")
      import
      type(mj_lattice_desc), intent(in) :: cell
      type(mj_hamiltonian_desc), intent(in) :: ham
      integer(c_int32_t), value :: nrep, device
      integer(c_int32_t), intent(in) :: L(2, *)
      real(c_double), intent(in) :: B_ext(3, *), T(*)
      type(c_ptr), intent(out) :: b
    end function
    integer(c_int32_t) function mj_batch_destroy(b) bind(c, name="mj_batch_destroy")
      import
      type(c_ptr), value :: b
    end function
    integer(c_int32_t) function mj_batch_upload(b, m, stream) bind(c, name="mj_batch_upload")
      import
      type(c_ptr), value :: b, stream
      real(c_double), intent(in) :: m(3, *)
    end function
    integer(c_int32_t) function mj_batch_download(b, m, stream) bind(c, name="mj_batch_download")
      import
      type(c_ptr), value :: b, stream
      real(c_double), intent(out) :: m(3, *)
    end function
    integer(c_int32_t) function mj_batch_step(b, p, nsteps, swap_every, E_dev, stream) bind(c, name="mj_batch_step")
      import
      type(c_ptr), value :: b, E_dev, stream
      type(mj_dyn_params), intent(in) :: p
      integer(c_int32_t), value :: nsteps, swap_every
    end function
    integer(c_int32_t) function mj_batch_graph_run(b, p, steps_per_graph, nreplay, swap_every, E_dev, stream) &
        bind(c, name="mj_batch_graph_run")
      import
      type(c_ptr), value :: b, E_dev, stream
      type(mj_dyn_params), intent(in) :: p
      integer(c_int32_t), value :: steps_per_graph, nreplay, swap_every
    end function
    integer(c_int32_t) function mj_batch_energies(b, E) bind(c, name="mj_batch_energies")
      import
      type(c_ptr), value :: b
      real(c_double), intent(out) :: E(*)
    end function
    integer(c_int32_t) function mj_batch_temperatures(b, T, accepted) bind(c, name="mj_batch_temperatures")
      import
      type(c_ptr), value :: b
      real(c_double), intent(out) :: T(*)
      integer(c_int32_t), intent(out) :: accepted(*)
    end function
    integer(c_int32_t) function mj_batch_mc(b, p, nrounds, sweeps_per_round, swap, E_dev, M_dev, slot_dev, colors, &
        stream) bind(c, name="mj_batch_mc")
      import
      type(c_ptr), value :: b, E_dev, M_dev, slot_dev, stream
      type(mj_mc_params), intent(inout) :: p
      integer(c_int32_t), value :: nrounds, sweeps_per_round, swap
      integer(c_int32_t), intent(out) :: colors(4)
    end function
    ! ---- reverse mode of the SIB trajectory ----
    integer(c_int32_t) function mj_adjoint_create(plan, nsteps, every, a) bind(c, name="mj_adjoint_create")
      import
      type(c_ptr), value :: plan
      integer(c_int32_t), value :: nsteps, every
      type(c_ptr), intent(out) :: a
    end function
    integer(c_int32_t) function mj_adjoint_destroy(a) bind(c, name="mj_adjoint_destroy")
      import
      type(c_ptr), value :: a
    end function
    integer(c_int32_t) function mj_adjoint_forward(a, p, m0_dev, mT_dev, stream) bind(c, name="mj_adjoint_forward")
      import
      type(c_ptr), value :: a, m0_dev, mT_dev, stream
      type(mj_dyn_params), intent(in) :: p
    end function
    integer(c_int32_t) function mj_adjoint_backward(a, gT_dev, g0_dev, g_terms_dev, g_b_dev, stream) &
        bind(c, name="mj_adjoint_backward")
      import
      type(c_ptr), value :: a, gT_dev, g0_dev, g_terms_dev, g_b_dev, stream
    end function
  end interface

  interface
    integer(c_size_t) function c_strlen(s) bind(c, name="strlen")
      import
      type(c_ptr), value :: s
    end function
  end interface

contains

  ! Text of the last failing call on this thread.
  function mj_error_message() result(msg)
    character(len=:), allocatable :: msg
    type(c_ptr) :: p
    character(kind=c_char), pointer :: chars(:)
    integer(c_size_t) :: n, i
    p = mj_last_error()
    n = c_strlen(p)
    call c_f_pointer(p, chars, [n])
    allocate(character(len=n) :: msg)
    do i = 1, n
      msg(i:i) = chars(i)
    end do
  end function

end module m_matjes_gpu
