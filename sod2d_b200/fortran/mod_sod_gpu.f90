! mod_sod_gpu -- Fortran binding of the B200 spectral-element library
! (include/sod2d_gpu.h, libsod2d_gpu.so).
!
! One interface per C entry point, bound with iso_c_binding in the pattern
! src/lib_sod2d/sources/mod_nvtx.f90:27-45 of the reference uses for NVTX.
! Argument conventions follow the C header:
!   - device arrays are `type(c_ptr), value`: pass `c_loc(x)` of an OpenACC
!     array inside `!$acc host_data use_device(x)`, as
!     src/lib_sod2d/sources/mod_comms.f90:1083-1092 does for NCCL;
!   - sod_gpu_init takes the mesh as HOST addresses (c_loc of the host
!     arrays) in sod_mesh_t and returns the context in a type(c_ptr);
!   - host outputs (iteration counts, residuals, time steps, analysis
!     integrals, preconditioner parameters) are plain Fortran variables passed
!     by reference; those the C side accepts as NULL are `optional`;
!   - scalars go by value.
! Every function returns SOD_GPU_OK (0) or a negative SOD_GPU_E* code;
! sod_gpu_check turns a non-zero status into an error stop with the
! library's message.
module mod_sod_gpu
   use iso_c_binding
   implicit none
   private :: c_strlen

   integer(c_int), parameter :: SOD_GPU_OK = 0
   integer(c_int), parameter :: SOD_GPU_EINVAL = -1      ! bad argument or unsupported size
   integer(c_int), parameter :: SOD_GPU_ECUDA = -2       ! a CUDA runtime call failed
   integer(c_int), parameter :: SOD_GPU_ENOMEM = -3      ! device allocation failed
   integer(c_int), parameter :: SOD_GPU_ENONFINITE = -4  ! a reduction returned NaN/Inf
   integer(c_int), parameter :: SOD_GPU_ESTAGNATE = -5   ! an iterative solve stopped making progress
   integer(c_int), parameter :: SOD_NOALLOC_MAX_ELEM = 1048576
   integer(c_int), parameter :: SOD_REDUCE_MIN_F32 = 0      ! kinds of sod_allreduce_fn
   integer(c_int), parameter :: SOD_REDUCE_MAX_F32 = 1
   integer(c_int), parameter :: SOD_REDUCE_SUM_F64 = 2

   ! Mesh and geometry (HOST addresses, reference layout), read by sod_gpu_init.
   type, bind(C) :: sod_mesh_t
      integer(c_int) :: porder, nelem, npoin, npoin_w
      type(c_ptr)    :: connec, lpoin_w, invAtoIJK, gmshAtoI, gmshAtoJ, gmshAtoK
      type(c_ptr)    :: dlxigp_ip, He, gpvol, Ml, invMl, helem, helem_l, lelpn, Ngp
   end type

   ! Physical and stabilisation constants of the compressible RHS.
   type, bind(C) :: sod_phys_t
      real(c_float) :: gamma_gas, Rgas, Cp, Prt
      real(c_float) :: c_lps, c_rho, c_ener, ce, cmax, cglob
      real(c_float) :: ducros_min_val, c_species_stab, p_inf, rho_inf
   end type

   ! Options of the certified FP64 pressure solve.
   type, bind(C) :: sod_solve_opts_t
      integer(c_int) :: max_iter
      real(c_double) :: tol
      integer(c_int) :: precond            ! 0 Jacobi, 1 learned, 2 reference FP32 CG, 3 Jacobi + extrapolated guess
      integer(c_int) :: stagnation_window
      integer(c_int) :: harvest
   end type

   ! Outcome of a pressure solve.
   type, bind(C) :: sod_solve_stats_t
      integer(c_int) :: iterations
      integer(c_int) :: fallback
      real(c_double) :: res_rel
      real(c_double) :: seconds
   end type

   ! Time integrator of the library-owned compressible state.
   type, bind(C) :: sod_rk_cfg_t
      integer(c_int) :: stages              ! 3, 4 or 5
      integer(c_int) :: rk_n                ! SSP53_2N variant when stages == 5
      integer(c_int) :: fp64_state
      real(c_float)  :: mu_factor
   end type

   ! The halo exchange a rank hands to sod_gpu_set_halo (c_funloc of a
   ! bind(C) function of this shape): for every neighbour i, send the floats
   ! [(commsMemPosInLoc(i)-1)*width, +commsMemSize(i)*width) of send_buf to
   ! ranksToComm(i) and receive the same range of recv_buf from it, as
   ! mpi_base_comms_real_ncclSendRcv(width) does; return 0 on success.
   !
   ! The global reduction a rank hands to sod_gpu_set_allreduce: reduce
   ! `count` values of the device buffer `buf` in place over all ranks
   ! (MPI_Allreduce with MPI_MIN / MPI_MAX on reals, MPI_SUM on real(8), by
   ! `kind`); return 0 on success.
   abstract interface
      integer(c_int) function sod_halo_exchange_fn(user, send_buf, recv_buf, width, stream) bind(C)
         import :: c_int, c_ptr
         type(c_ptr), value :: user, send_buf, recv_buf, stream
         integer(c_int), value :: width
      end function
      integer(c_int) function sod_allreduce_fn(user, buf, count, kind, stream) bind(C)
         import :: c_int, c_ptr
         type(c_ptr), value :: user, buf, stream
         integer(c_int), value :: count, kind
      end function
   end interface

   interface
      integer(c_int) function sod_gpu_init(mesh, phys, out) bind(C, name='sod_gpu_init')
         import :: c_int, c_ptr, sod_mesh_t, sod_phys_t
         type(sod_mesh_t), intent(in) :: mesh
         type(sod_phys_t), intent(in) :: phys
         type(c_ptr), intent(out) :: out
      end function
      integer(c_int) function sod_gpu_finalize(ctx) bind(C, name='sod_gpu_finalize')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function sod_gpu_set_stream(ctx, cuda_stream) bind(C, name='sod_gpu_set_stream')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, cuda_stream
      end function
      integer(c_int) function sod_gpu_set_async(ctx, async_enabled) bind(C, name='sod_gpu_set_async')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: async_enabled
      end function
      integer(c_int) function sod_gpu_synchronize(ctx) bind(C, name='sod_gpu_synchronize')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function
      type(c_ptr) function sod_gpu_last_error() bind(C, name='sod_gpu_last_error')
         import :: c_ptr
      end function
      integer(c_size_t) function sod_gpu_device_bytes(ctx) bind(C, name='sod_gpu_device_bytes')
         import :: c_int, c_ptr, c_size_t
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function sod_gpu_set_halo(ctx, rank, numRanksWithComms, ranksToComm, commsMemPosInLoc, &
         commsMemSize, nodesToComm, send_buf, recv_buf, exchange, user) bind(C, name='sod_gpu_set_halo')
         import :: c_funptr, c_int, c_ptr
         type(c_ptr), value :: ctx, send_buf, recv_buf, user
         integer(c_int), value :: rank, numRanksWithComms
         integer(c_int), intent(in) :: ranksToComm(*), commsMemPosInLoc(*), commsMemSize(*), nodesToComm(*)
         type(c_funptr), value :: exchange
      end function
      integer(c_int) function sod_gpu_halo_update(ctx, field, ncomp) bind(C, name='sod_gpu_halo_update')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, field
         integer(c_int), value :: ncomp
      end function
      integer(c_int) function sod_gpu_set_allreduce(ctx, allreduce, user) bind(C, name='sod_gpu_set_allreduce')
         import :: c_funptr, c_int, c_ptr
         type(c_ptr), value :: ctx, user
         type(c_funptr), value :: allreduce
      end function
      integer(c_int) function sod_gpu_full_convec_ijk(ctx, u, q, rho, pr, E, Rmass, Rmom, Rener, &
         initialze, fact) bind(C, name='sod_gpu_full_convec_ijk')
         import :: c_float, c_int, c_ptr
         type(c_ptr), value :: ctx, u, q, rho, pr, E, Rmass, Rmom, Rener
         integer(c_int), value :: initialze
         real(c_float), value :: fact
      end function
      integer(c_int) function sod_gpu_full_proj_ijk(ctx, rho, u, Tem, ProjMass, ProjEner, ProjMX, ProjMY, &
         ProjMZ) bind(C, name='sod_gpu_full_proj_ijk')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, rho, u, Tem, ProjMass, ProjEner, ProjMX, ProjMY, ProjMZ
      end function
      integer(c_int) function sod_gpu_full_diff_stab_ijk(ctx, Cp, Pr, rho_n, rho, u, Tem, mu_fluid, mu_e, &
         mu_sgs, ProjMass, ProjEner, ProjMX, ProjMY, ProjMZ, tau_stab, Rmass, Rmom, Rener, initialze, &
         fact) bind(C, name='sod_gpu_full_diff_stab_ijk')
         import :: c_float, c_int, c_ptr
         type(c_ptr), value :: ctx, rho_n, rho, u, Tem, mu_fluid, mu_e, mu_sgs, ProjMass, ProjEner, &
            ProjMX, ProjMY, ProjMZ, tau_stab, Rmass, Rmom, Rener
         real(c_float), value :: Cp, Pr, fact
         integer(c_int), value :: initialze
      end function
      integer(c_int) function sod_gpu_full_diffusion_ijk(ctx, Cp, Pr, rho_n, rho, u, Tem, mu_fluid, mu_e, &
         mu_sgs, Rmass, Rmom, Rener, initialze, fact) bind(C, name='sod_gpu_full_diffusion_ijk')
         import :: c_float, c_int, c_ptr
         type(c_ptr), value :: ctx, rho_n, rho, u, Tem, mu_fluid, mu_e, mu_sgs, Rmass, Rmom, Rener
         real(c_float), value :: Cp, Pr, fact
         integer(c_int), value :: initialze
      end function
      integer(c_int) function sod_gpu_lumped_solver(ctx, R, ncomp) bind(C, name='sod_gpu_lumped_solver')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, R
         integer(c_int), value :: ncomp
      end function
      integer(c_int) function sod_gpu_set_mu_e(ctx, mu_e) bind(C, name='sod_gpu_set_mu_e')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, mu_e
      end function
      integer(c_int) function sod_gpu_updateF(ctx, rho, q, E, mu_e, mu_factor, tau_stab, Rmass, Rmom, &
         Rener, u_out, pr_out, Tem_out, mu_fluid_out) bind(C, name='sod_gpu_updateF')
         import :: c_float, c_int, c_ptr
         type(c_ptr), value :: ctx, rho, q, E, mu_e, tau_stab, Rmass, Rmom, Rener, u_out, pr_out, &
            Tem_out, mu_fluid_out
         real(c_float), value :: mu_factor
      end function
      integer(c_int) function sod_gpu_comp_tau(ctx, csound, u, tau) bind(C, name='sod_gpu_comp_tau')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, csound, u, tau
      end function
      integer(c_int) function sod_gpu_eval_laplacian_mult(ctx, p, ResP) bind(C, &
         name='sod_gpu_eval_laplacian_mult')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, p, ResP
      end function
      integer(c_int) function sod_gpu_eval_laplacian_mult64(ctx, p, ResP) bind(C, &
         name='sod_gpu_eval_laplacian_mult64')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, p, ResP
      end function
      integer(c_int) function sod_gpu_eval_laplacian_diag(ctx, d) bind(C, &
         name='sod_gpu_eval_laplacian_diag')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, d
      end function
      integer(c_int) function sod_gpu_eval_gradient(ctx, x, gradX) bind(C, name='sod_gpu_eval_gradient')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, x, gradX
      end function
      integer(c_int) function sod_gpu_eval_divergence(ctx, u, divU) bind(C, &
         name='sod_gpu_eval_divergence')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, u, divU
      end function
      integer(c_int) function sod_gpu_full_convec_ijk_incomp(ctx, u, q, Rmom) bind(C, &
         name='sod_gpu_full_convec_ijk_incomp')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, u, q, Rmom
      end function
      integer(c_int) function sod_gpu_conjgrad_pressure(ctx, Rp0, R, maxIter, tol, iters, res_rel) bind(C, &
         name='sod_gpu_conjgrad_pressure')
         import :: c_double, c_int, c_ptr
         type(c_ptr), value :: ctx, Rp0, R
         integer(c_int), value :: maxIter
         real(c_double), value :: tol
         integer(c_int), intent(out), optional :: iters
         real(c_double), intent(out), optional :: res_rel
      end function
      integer(c_int) function sod_gpu_pressure_solve(ctx, b, x, opts, stats) bind(C, &
         name='sod_gpu_pressure_solve')
         import :: c_int, c_ptr, sod_solve_opts_t, sod_solve_stats_t
         type(c_ptr), value :: ctx, b, x
         type(sod_solve_opts_t), intent(in) :: opts
         type(sod_solve_stats_t), intent(out) :: stats
      end function
      integer(c_int) function sod_gpu_precond_num_params(ctx) bind(C, name='sod_gpu_precond_num_params')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function sod_gpu_precond_init(ctx, seed, harvest_capacity) bind(C, &
         name='sod_gpu_precond_init')
         import :: c_int, c_int64_t, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int64_t), value :: seed
         integer(c_int), value :: harvest_capacity
      end function
      integer(c_int) function sod_gpu_precond_set_params(ctx, host_params, n) bind(C, &
         name='sod_gpu_precond_set_params')
         import :: c_float, c_int, c_ptr
         type(c_ptr), value :: ctx
         real(c_float), intent(in) :: host_params(*)
         integer(c_int), value :: n
      end function
      integer(c_int) function sod_gpu_precond_get_params(ctx, host_params, n) bind(C, &
         name='sod_gpu_precond_get_params')
         import :: c_float, c_int, c_ptr
         type(c_ptr), value :: ctx
         real(c_float), intent(out) :: host_params(*)
         integer(c_int), value :: n
      end function
      integer(c_int) function sod_gpu_precond_apply(ctx, r, z) bind(C, name='sod_gpu_precond_apply')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, r, z
      end function
      integer(c_int) function sod_gpu_precond_loss_grad(ctx, r, e, loss, grad_host) bind(C, &
         name='sod_gpu_precond_loss_grad')
         import :: c_double, c_float, c_int, c_ptr
         type(c_ptr), value :: ctx, r, e
         real(c_double), intent(out) :: loss
         real(c_float), intent(out), optional :: grad_host(*)
      end function
      integer(c_int) function sod_gpu_precond_harvest_count(ctx) bind(C, &
         name='sod_gpu_precond_harvest_count')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function sod_gpu_precond_restart_harvest(ctx) bind(C, &
         name='sod_gpu_precond_restart_harvest')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function sod_gpu_precond_train(ctx, steps, batch, lr, seed, final_loss) bind(C, &
         name='sod_gpu_precond_train')
         import :: c_float, c_int, c_int64_t, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: steps, batch
         real(c_float), value :: lr
         integer(c_int64_t), value :: seed
         real(c_float), intent(out) :: final_loss
      end function
      integer(c_int) function sod_gpu_species_tau(ctx, u, tau) bind(C, name='sod_gpu_species_tau')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, u, tau
      end function
      integer(c_int) function sod_gpu_eval_tau_veloc(ctx, u, GradX, GradY, GradZ) bind(C, &
         name='sod_gpu_eval_tau_veloc')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, u, GradX, GradY, GradZ
      end function
      integer(c_int) function sod_gpu_full_diff_stab_incomp(ctx, u, mu_fluid, mu_sgs, TauPX, TauPY, TauPZ, &
         tau_stab, Rmom) bind(C, name='sod_gpu_full_diff_stab_incomp')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, u, mu_fluid, mu_sgs, TauPX, TauPY, TauPZ, tau_stab, Rmom
      end function
      integer(c_int) function sod_gpu_conjgrad_veloc(ctx, fact, dt, mu_fluid, mu_sgs, Rp0, R, maxIter, &
         tol, iters, res_rel) bind(C, name='sod_gpu_conjgrad_veloc')
         import :: c_double, c_float, c_int, c_ptr
         type(c_ptr), value :: ctx, mu_fluid, mu_sgs, Rp0, R
         real(c_float), value :: fact, dt
         integer(c_int), value :: maxIter
         real(c_double), value :: tol
         integer(c_int), intent(out), optional :: iters
         real(c_double), intent(out), optional :: res_rel
      end function
      integer(c_int) function sod_gpu_incomp_init(ctx, u, nu) bind(C, name='sod_gpu_incomp_init')
         import :: c_double, c_int, c_ptr
         type(c_ptr), value :: ctx, u
         real(c_double), value :: nu
      end function
      integer(c_int) function sod_gpu_incomp_step(ctx, dt, opts, stats) bind(C, &
         name='sod_gpu_incomp_step')
         import :: c_float, c_int, c_ptr, sod_solve_opts_t, sod_solve_stats_t
         type(c_ptr), value :: ctx
         real(c_float), value :: dt
         type(sod_solve_opts_t), intent(in) :: opts
         type(sod_solve_stats_t), intent(out) :: stats
      end function
      integer(c_int) function sod_gpu_incomp_set_veloc_solver(ctx, maxIter, tol) bind(C, &
         name='sod_gpu_incomp_set_veloc_solver')
         import :: c_double, c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: maxIter
         real(c_double), value :: tol
      end function
      integer(c_int) function sod_gpu_incomp_veloc_stats(ctx, iters, res_rel) bind(C, &
         name='sod_gpu_incomp_veloc_stats')
         import :: c_double, c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), intent(out) :: iters
         real(c_double), intent(out) :: res_rel
      end function
      integer(c_int) function sod_gpu_incomp_get(ctx, u, p) bind(C, name='sod_gpu_incomp_get')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, u, p
      end function
      integer(c_int) function sod_gpu_incomp_set_pressure(ctx, p) bind(C, &
         name='sod_gpu_incomp_set_pressure')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, p
      end function
      integer(c_int) function sod_gpu_incomp_adapt_dt(ctx, cfl_conv, dt) bind(C, &
         name='sod_gpu_incomp_adapt_dt')
         import :: c_float, c_int, c_ptr
         type(c_ptr), value :: ctx
         real(c_float), value :: cfl_conv
         real(c_float), intent(out) :: dt
      end function
      integer(c_int) function sod_gpu_incomp_analysis(ctx, out) bind(C, name='sod_gpu_incomp_analysis')
         import :: c_double, c_int, c_ptr
         type(c_ptr), value :: ctx
         real(c_double), intent(out) :: out(*)
      end function
      integer(c_int) function sod_gpu_generic_scalar_convec_ijk(ctx, q, eta, u, R, initialze, fact) &
         bind(C, name='sod_gpu_generic_scalar_convec_ijk')
         import :: c_float, c_int, c_ptr
         type(c_ptr), value :: ctx, q, eta, u, R
         integer(c_int), value :: initialze
         real(c_float), value :: fact
      end function
      integer(c_int) function sod_gpu_smart_visc_spectral_imex(ctx, Reta, rho, u, csound, mu_e) bind(C, &
         name='sod_gpu_smart_visc_spectral_imex')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, Reta, rho, u, csound, mu_e
      end function
      integer(c_int) function sod_gpu_ducros_visc_limit(ctx, rho, u, divU, vorti, csound, mu_e) bind(C, &
         name='sod_gpu_ducros_visc_limit')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, rho, u, divU, vorti, csound, mu_e
      end function
      integer(c_int) function sod_gpu_rk_ls_stage(ctx, first, lam1, lami, gam, dt, rho1, q1, E1, rho2, q2, &
         E2, Rmass, Rmom, Rener) bind(C, name='sod_gpu_rk_ls_stage')
         import :: c_float, c_int, c_ptr
         type(c_ptr), value :: ctx, rho1, q1, E1, rho2, q2, E2, Rmass, Rmom, Rener
         integer(c_int), value :: first
         real(c_float), value :: lam1, lami, gam, dt
      end function
      integer(c_int) function sod_gpu_comp_init_state(ctx, cfg, rho, u, q, pr, E, Tem, csound, machno, &
         eta) bind(C, name='sod_gpu_comp_init_state')
         import :: c_int, c_ptr, sod_rk_cfg_t
         type(c_ptr), value :: ctx, rho, u, q, pr, E, Tem, csound, machno, eta
         type(sod_rk_cfg_t), intent(in) :: cfg
      end function
      integer(c_int) function sod_gpu_comp_rk_ls_step(ctx, dt) bind(C, name='sod_gpu_comp_rk_ls_step')
         import :: c_float, c_int, c_ptr
         type(c_ptr), value :: ctx
         real(c_float), value :: dt
      end function
      integer(c_int) function sod_gpu_comp_imex_step(ctx, dt, maxIter, tol) bind(C, &
         name='sod_gpu_comp_imex_step')
         import :: c_double, c_float, c_int, c_ptr
         type(c_ptr), value :: ctx
         real(c_float), value :: dt
         integer(c_int), value :: maxIter
         real(c_double), value :: tol
      end function
      integer(c_int) function sod_gpu_comp_imex_stats(ctx, cg_iters, cg_res) bind(C, &
         name='sod_gpu_comp_imex_stats')
         import :: c_double, c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), intent(out) :: cg_iters
         real(c_double), intent(out) :: cg_res
      end function
      integer(c_int) function sod_gpu_comp_adapt_dt(ctx, cfl_conv, cfl_diff, dt) bind(C, &
         name='sod_gpu_comp_adapt_dt')
         import :: c_float, c_int, c_ptr
         type(c_ptr), value :: ctx
         real(c_float), value :: cfl_conv, cfl_diff
         real(c_float), intent(out) :: dt
      end function
      integer(c_int) function sod_gpu_comp_analysis(ctx, rho0, out) bind(C, name='sod_gpu_comp_analysis')
         import :: c_double, c_float, c_int, c_ptr
         type(c_ptr), value :: ctx
         real(c_float), value :: rho0
         real(c_double), intent(out) :: out(*)
      end function
      integer(c_int) function sod_gpu_comp_get_state(ctx, rho, q, E, mu_e) bind(C, &
         name='sod_gpu_comp_get_state')
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, rho, q, E, mu_e
      end function
      integer(c_int) function sod_gpu_analysis_noalloc(porder, nelem, npoin, npoin_w, connec, lpoin_w, &
         invAtoIJK, gmshAtoI, gmshAtoJ, gmshAtoK, dlxigp_ip, He, gpvol, Ngp, rho, u, mu_fluid, mu_e, &
         machno, rho0, volT, stream, out) bind(C, name='sod_gpu_analysis_noalloc')
         import :: c_double, c_float, c_int, c_ptr
         integer(c_int), value :: porder, nelem, npoin, npoin_w
         type(c_ptr), value :: connec, lpoin_w, invAtoIJK, gmshAtoI, gmshAtoJ, gmshAtoK, dlxigp_ip, He, &
            gpvol, Ngp, rho, u, mu_fluid, mu_e, machno, stream
         real(c_float), value :: rho0, volT
         real(c_double), intent(out) :: out(*)
      end function
   end interface

   interface
      integer(c_size_t) function c_strlen(s) bind(C, name='strlen')
         import :: c_ptr, c_size_t
         type(c_ptr), value :: s
      end function
   end interface

contains

   ! The library's description of the calling thread's last failure.
   function sod_gpu_error_message() result(msg)
      character(len=:), allocatable :: msg
      type(c_ptr) :: p
      character(kind=c_char), pointer :: chars(:)
      integer :: i, n
      p = sod_gpu_last_error()
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
   end function

   ! Stop with the library's message when a call did not return SOD_GPU_OK.
   subroutine sod_gpu_check(status, where)
      integer(c_int), intent(in) :: status
      character(len=*), intent(in) :: where
      if (status /= SOD_GPU_OK) then
         write(*, '(a, a, a, i0, a, a)') 'sod_gpu: ', where, ' returned ', status, ': ', sod_gpu_error_message()
         error stop 1
      end if
   end subroutine

end module mod_sod_gpu
