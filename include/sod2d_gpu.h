/*
 * sod2d_gpu.h -- C-ABI of the B200 (sm_100a) spectral-element RHS library.
 *
 * Drop-in for the hot-path subroutines of the SOD2D Fortran solver.  A
 * Fortran caller binds each function with `interface ... bind(C, name=...)`
 * (the pattern of src/lib_sod2d/sources/mod_nvtx.f90:27-45) and passes
 * device addresses with `!$acc host_data use_device(...)`, as
 * src/lib_sod2d/sources/mod_comms.f90:1083-1092 already does for NCCL.
 *
 * Conventions
 *  - Arrays keep the reference's Fortran layout: column-major, so a field
 *    X(npoin,3) is three contiguous blocks of npoin values; connectivity
 *    holds 1-based node ids.  Paths are relative to the reference project.
 *  - sod_gpu_init() takes HOST pointers and builds the library's own
 *    device-resident mirrors (element-major connectivity in tensor order,
 *    packed J^-1 + Gauss weights per element, node->slot CSR for the
 *    assembly).  Every other call takes DEVICE pointers.
 *  - All calls are complete on return (the reference's OpenACC regions are
 *    synchronous), unless sod_gpu_set_stream() selected a stream and
 *    sod_gpu_set_async(ctx, 1) was called, in which case work is only
 *    enqueued on that stream.  Kernels that wait on their own bulk copies
 *    bound every wait; a wait that gave up (never expected) is reported as
 *    SOD_GPU_ECUDA by the next call that synchronises (every call when not
 *    asynchronous, sod_gpu_synchronize() otherwise).
 *  - Functions return 0 on success and a negative SOD_GPU_E* code on error;
 *    sod_gpu_last_error() describes the last failure of the calling thread.
 *    The Fortran shim turns a non-zero status into `stop 1`.
 *  - Assembly is deterministic: each element writes its contributions to its
 *    own slots and a node-centric pass sums them in a fixed order with
 *    Kahan compensation (no floating-point atomics), so two runs give
 *    bit-identical results.
 */
#ifndef SOD2D_GPU_H
#define SOD2D_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SOD_GPU_OK 0
#define SOD_GPU_EINVAL -1    /* bad argument or unsupported size          */
#define SOD_GPU_ECUDA -2     /* a CUDA runtime call failed                */
#define SOD_GPU_ENOMEM -3    /* device allocation failed                  */
#define SOD_GPU_ENONFINITE -4 /* a reduction returned NaN/Inf              */
#define SOD_GPU_ESTAGNATE -5 /* an iterative solve stopped making progress */

typedef struct sod_gpu_ctx sod_gpu_ctx;

/* Mesh and geometry, HOST pointers, reference layout.  Mirrors the arrays
 * the solver classes hold after CFDSolverBase_evalJacobians / evalMass
 * (src/lib_mainBaseClass/sources/CFDSolverBase.f90:1638-1795). */
typedef struct {
  int porder;            /* element order; 3 and 4 are built             */
  int nelem, npoin, npoin_w;
  const int *connec;     /* connecParWork(nelem,nnode), 1-based          */
  const int *lpoin_w;    /* workingNodesPar(npoin_w), 1-based            */
  const int *invAtoIJK;  /* invAtoIJK(P+1,P+1,P+1)                       */
  const int *gmshAtoI, *gmshAtoJ, *gmshAtoK; /* (nnode)                  */
  const float *dlxigp_ip; /* dlxigp_ip(ngaus,3,P+1)                      */
  const float *He;       /* He(3,3,ngaus,nelem)                          */
  const float *gpvol;    /* gpvol(1,ngaus,nelem)                         */
  const float *Ml;       /* Ml(npoin)                                    */
  const float *invMl;    /* invMl(npoin)                                 */
  const float *helem;    /* helem(nelem)       (may be NULL)             */
  const float *helem_l;  /* helem_l(nelem,nnode) (may be NULL)           */
  const int *lelpn;      /* lelpn(npoin)       (may be NULL)             */
  const float *Ngp;      /* Ngp(ngaus,nnode)   (may be NULL: Kronecker)  */
} sod_mesh_t;

/* Gas and stabilisation constants of the compressible path
 * (src/lib_sod2d/sources/mod_numerical_params.f90:27-52, TGVCompSolver.f90:128-146). */
typedef struct {
  float gamma_gas, Rgas, Cp, Prt;
  float c_lps;          /* c_lps_comp = 0.1                                */
  float c_rho, c_ener;  /* 1, 1                                            */
  float ce, cmax, cglob;/* ce_comp = 1 (high-Mach path), 0.5, 1            */
  float ducros_min_val; /* 0.1                                             */
  float c_species_stab; /* tau scale of comp_tau, 0.5                      */
  float p_inf, rho_inf; /* nscbc_p_inf, nscbc_rho_inf (entropy scaling)    */
} sod_phys_t;

/* ---- context --------------------------------------------------------- */
int sod_gpu_init(const sod_mesh_t *mesh, const sod_phys_t *phys, sod_gpu_ctx **out);
int sod_gpu_finalize(sod_gpu_ctx *ctx);
int sod_gpu_set_stream(sod_gpu_ctx *ctx, void *cuda_stream);
int sod_gpu_set_async(sod_gpu_ctx *ctx, int async_enabled);
int sod_gpu_synchronize(sod_gpu_ctx *ctx);
const char *sod_gpu_last_error(void);
/* Device bytes held by the context (mirrors + scratch). */
size_t sod_gpu_device_bytes(const sod_gpu_ctx *ctx);

/* ---- partitioned meshes: halo sums over ranks -------------------------
 * A rank that holds part of the mesh (its elements, every node they touch,
 * Ml / invMl of the whole mesh) sums assembled nodal fields with the ranks
 * that share its nodes, where the reference calls
 * mpi_halo_atomic_update_real_arrays / _massEnerMom
 * (src/lib_sod2d/sources/mod_comms.f90:776-877 with the NCCL transport of
 * :1049-1102): inside sod_gpu_full_proj_ijk (elem_stab.f90:563-571) and
 * inside sod_gpu_updateF on the projections and on the residuals
 * (time_integ_ls.f90:663-667).  The plan has the reference's comms arrays
 * (HOST, 1-based): ranksToComm(numRanksWithComms), commsMemPosInLoc and
 * commsMemSize per neighbour, nodesToComm(sum of commsMemSize) as local
 * node ids, each neighbour's range listing the shared nodes in the same
 * order on both sides.  send_buf and recv_buf are DEVICE buffers of
 * 12 * numNodesToComm floats owned by the caller (the reference's
 * aux_realField_s / aux_realField_r).
 *
 * A width-W exchange packs node j of nodesToComm, component k, at
 * send_buf[j*W + k] on the context's stream, then calls
 * exchange(user, send_buf, recv_buf, W, stream), which sends, for every
 * neighbour i, the floats [(commsMemPosInLoc(i)-1)*W, +commsMemSize(i)*W)
 * of send_buf to rank ranksToComm(i) and receives the same range of
 * recv_buf from it (mpi_base_comms_real_ncclSendRcv(numArrays)); when it
 * returns, the transfers are complete or enqueued on `stream`, and a
 * non-zero return fails the calling entry point.  Each shared node is then
 * summed over its ranks in ascending rank order, so all ranks hold
 * bit-identical values (the reference's per-neighbour atomic adds do not
 * guarantee that for nodes on three or more ranks).  numRanksWithComms = 0
 * removes the plan. */
typedef int (*sod_halo_exchange_fn)(void *user, float *send_buf, float *recv_buf, int width, void *stream);
int sod_gpu_set_halo(sod_gpu_ctx *ctx, int rank, int numRanksWithComms, const int *ranksToComm,
                     const int *commsMemPosInLoc, const int *commsMemSize, const int *nodesToComm,
                     float *send_buf, float *recv_buf, sod_halo_exchange_fn exchange, void *user);
/* mpi_halo_atomic_update_real_arrays(ncomp, field): field(npoin,ncomp)
 * (device, reference layout) summed over the ranks that share each node. */
int sod_gpu_halo_update(sod_gpu_ctx *ctx, float *field, int ncomp);
/* Global reductions of a partitioned mesh, the reference's MPI_Allreduce
 * calls of the explicit step: min rho of the entropy viscosity
 * (mod_entropy_viscosity.f90:161), the CFL time step (mod_time_ops.f90:59)
 * and the analysis integrals (mod_analysis.f90:39, 134-135, 166).
 * allreduce(user, buf, count, kind, stream) reduces `count` values of the
 * DEVICE buffer `buf` in place over all ranks: kind SOD_REDUCE_MIN_F32 /
 * SOD_REDUCE_MAX_F32 (float) or SOD_REDUCE_SUM_F64 (double); when it
 * returns the result is in `buf` or enqueued on `stream`.  Every rank of the
 * plan makes the same calls in the same order.  Setting it (a collective
 * call) also sums the mesh volume of the analysis over the ranks.  With a
 * halo plan, sod_gpu_comp_rk_ls_step, sod_gpu_comp_imex_step,
 * sod_gpu_comp_adapt_dt and sod_gpu_comp_analysis do the halo sums and
 * reductions of rk_4_ls_main and imex_main; the IMEX solve's dot products
 * run over the working nodes this rank owns (a shared node belongs to the
 * lowest rank holding it; the reference's lpoin_o) and are summed over the
 * ranks.  The incompressible operators (Laplacian, its diagonal, gradient,
 * divergence, velocity projection) sum over the ranks inside, as the
 * reference's mod_operators.f90 does; sod_gpu_conjgrad_pressure and
 * sod_gpu_conjgrad_veloc sum their operators and reduce their dot products
 * over the owned nodes; sod_gpu_incomp_step (with precond 2, the reference's
 * FP32 pressure solve), sod_gpu_incomp_adapt_dt and sod_gpu_incomp_analysis
 * run a partitioned mesh.  sod_gpu_pressure_solve with precond 0 runs a
 * host-driven FP64 Jacobi-PCG on a partitioned mesh (FP64 values travel as
 * two floats each through the exchange, so send_buf and recv_buf must be
 * 8-byte aligned), certified on the true residual like the single-rank
 * solve; the learned preconditioner (precond 1), whose patches cross the
 * part boundaries, returns SOD_GPU_EINVAL on a context with a halo plan. */
#define SOD_REDUCE_MIN_F32 0
#define SOD_REDUCE_MAX_F32 1
#define SOD_REDUCE_SUM_F64 2
typedef int (*sod_allreduce_fn)(void *user, void *buf, int count, int kind, void *stream);
int sod_gpu_set_allreduce(sod_gpu_ctx *ctx, sod_allreduce_fn allreduce, void *user);

/* ---- element operators (device pointers, FP32, reference layout) ------ */

/* Split-form convective residual.  Replaces full_convec_ijk,
 * src/lib_sod2d/sources/elem_convec.f90:227-470 (E is the energy-like
 * variable the caller convects; updateF passes the enthalpy aux_h). */
int sod_gpu_full_convec_ijk(sod_gpu_ctx *ctx, const float *u, const float *q, const float *rho,
                            const float *pr, const float *E, float *Rmass, float *Rmom,
                            float *Rener, int initialze, float fact);

/* Assembled, lumped-mass-inverted LPS projections.  Replaces full_proj_ijk,
 * src/lib_sod2d/sources/elem_stab.f90:441-586.  Each Proj* is (npoin,3). */
int sod_gpu_full_proj_ijk(sod_gpu_ctx *ctx, const float *rho, const float *u, const float *Tem,
                          float *ProjMass, float *ProjEner, float *ProjMX, float *ProjMY,
                          float *ProjMZ);

/* Viscous + heat + artificial diffusion with LPS stabilisation.  Replaces
 * full_diff_stab_ijk, src/lib_sod2d/sources/elem_stab.f90:207-438.
 * mu_e, mu_sgs are (nelem,ngaus); mu_sgs may be NULL (zero). */
int sod_gpu_full_diff_stab_ijk(sod_gpu_ctx *ctx, float Cp, float Pr, const float *rho_n,
                               const float *rho, const float *u, const float *Tem,
                               const float *mu_fluid, const float *mu_e, const float *mu_sgs,
                               const float *ProjMass, const float *ProjEner, const float *ProjMX,
                               const float *ProjMY, const float *ProjMZ, const float *tau_stab,
                               float *Rmass, float *Rmom, float *Rener, int initialze, float fact);

/* Plain (not LPS-stabilised) diffusion residual; replaces
 * full_diffusion_ijk, src/lib_sod2d/sources/elem_diffu.f90:12-223 (the
 * path of flag_lps_stab = .false.).  Same argument meaning as
 * sod_gpu_full_diff_stab_ijk without the projections and tau_stab;
 * mu_e, mu_sgs are (nelem,ngaus); mu_sgs may be NULL (zero). */
int sod_gpu_full_diffusion_ijk(sod_gpu_ctx *ctx, float Cp, float Pr, const float *rho_n, const float *rho,
                               const float *u, const float *Tem, const float *mu_fluid, const float *mu_e,
                               const float *mu_sgs, float *Rmass, float *Rmom, float *Rener, int initialze,
                               float fact);

/* R(lpoin_w,:) *= invMl for ncomp components of an (npoin,ncomp) array.
 * Replaces lumped_solver_scal_opt / lumped_solver_vect_opt,
 * src/lib_sod2d/sources/mod_solver.f90:41-104. */
int sod_gpu_lumped_solver(sod_gpu_ctx *ctx, float *R, int ncomp);

/* Store the element viscosity mu_e(nelem,ngaus) in the context (converted
 * once to the library's element layout).  sod_gpu_updateF called with
 * mu_e == NULL then uses this copy: the reference keeps mu_e fixed across
 * the stages of a time step (it is updated once per step, after the
 * stages, time_integ_ls.f90:455-463). */
int sod_gpu_set_mu_e(sod_gpu_ctx *ctx, const float *mu_e);

/* One full RHS evaluation from the conserved state (level "pos" arrays):
 * equation of state, Sutherland viscosity (mu = mu_factor*1.458e-6*
 * T^1.5/(T+110.4)), convection with E := h, LPS projection, stabilised
 * diffusion and lumped inversion, fused.  Replaces the body of updateF,
 * src/lib_sod2d/sources/time_integ_ls.f90:489-691 (periodic, no LES, no
 * sources).  tau_stab(nelem) comes from sod_gpu_comp_tau; mu_e may be NULL
 * to use the copy stored by sod_gpu_set_mu_e.  Optional
 * outputs (NULL to skip): u(npoin,3), pr, Tem, mu_fluid at working nodes. */
int sod_gpu_updateF(sod_gpu_ctx *ctx, const float *rho, const float *q, const float *E,
                    const float *mu_e, float mu_factor, const float *tau_stab, float *Rmass,
                    float *Rmom, float *Rener, float *u_out, float *pr_out, float *Tem_out,
                    float *mu_fluid_out);

/* tau(nelem) = max_node h_e*(c_species_stab/P)*(c+|u|).  Replaces comp_tau,
 * src/lib_sod2d/sources/elem_stab.f90:589-616. */
int sod_gpu_comp_tau(sod_gpu_ctx *ctx, const float *csound, const float *u, float *tau);

/* ---- incompressible operators (device pointers, FP32, reference layout) */

/* ResP = sum_e int grad N . grad p (assembled, no mass inversion).
 * Replaces eval_laplacian_mult, src/lib_sod2d_incomp/sources/mod_operators.f90:16-112. */
int sod_gpu_eval_laplacian_mult(sod_gpu_ctx *ctx, const float *p, float *ResP);
/* The same operator in FP64 arithmetic on FP64 vectors (FP32 geometry). */
int sod_gpu_eval_laplacian_mult64(sod_gpu_ctx *ctx, const double *p, double *ResP);
/* d = sum gpvol |grad N_a|^2.  Replaces eval_laplacian_diag, mod_operators.f90:638-682. */
int sod_gpu_eval_laplacian_diag(sod_gpu_ctx *ctx, float *d);
/* Lumped gradient gradX(npoin,3).  Replaces eval_gradient(..., lump=.true.),
 * mod_operators.f90:212-288. */
int sod_gpu_eval_gradient(sod_gpu_ctx *ctx, const float *x, float *gradX);
/* Assembled int N div u.  Replaces eval_divergence, mod_operators.f90:485-570. */
int sod_gpu_eval_divergence(sod_gpu_ctx *ctx, const float *u, float *divU);
/* Skew-symmetric momentum convection.  Replaces full_convec_ijk_incomp,
 * src/lib_sod2d_incomp/sources/elem_convec_incomp.f90:19-125 (Rmom zeroed). */
int sod_gpu_full_convec_ijk_incomp(sod_gpu_ctx *ctx, const float *u, const float *q, float *Rmom);

/* Jacobi-preconditioned CG for the pressure Poisson problem in the
 * reference's arithmetic: FP32 vectors, FP64 dot products and norms,
 * alpha and beta rounded to FP32, Polak-Ribiere beta, x0 = Rp0, stop when
 * ||r|| < tol ||b|| or after maxIter.  On return R = x0 + x.  Replaces
 * conjGrad_pressure_incomp, src/lib_sod2d_incomp/sources/mod_solver_incomp.f90:253-506.
 * *iters and *res_rel (host, may be NULL) receive the iteration count and
 * ||r||/||b||. */
int sod_gpu_conjgrad_pressure(sod_gpu_ctx *ctx, const float *Rp0, float *R, int maxIter, double tol,
                              int *iters, double *res_rel);

/* Pressure solve to an FP64-certified tolerance: flexible (Polak-Ribiere)
 * preconditioned CG, the reference's form, on FP64 vectors with the FP64
 * Laplacian.  Preconditioner 0 = Jacobi; 1 = the learned element-patch
 * preconditioner (sod_gpu_precond_*), falling back to Jacobi when the
 * residual stagnates.  The iteration scalars stay on the device and the
 * host reads them once per batch of iterations.  b is made mean-free over
 * working nodes (the periodic Laplacian's null space).  Convergence is
 * declared only when the true residual ||b - A x|| / ||b||, recomputed in
 * FP64, is below tol. */
typedef struct {
  int max_iter;
  double tol;
  int precond;         /* 0 Jacobi, 1 learned; 2 (sod_gpu_incomp_step only):
                          the reference's conjGrad_pressure_incomp in FP32
                          with max_iter / tol, uncertified; 3
                          (sod_gpu_incomp_step only): Jacobi from the
                          learned path's initial guess 2 p^n - p^(n-1)    */
  int stagnation_window; /* iterations without a 2x residual drop -> fallback */
  int harvest;         /* 1: record (residual, error) pairs of this solve for
                          training the learned preconditioner             */
} sod_solve_opts_t;
typedef struct {
  int iterations;
  int fallback;        /* 1 if the learned preconditioner was abandoned       */
  double res_rel;      /* true FP64 relative residual at exit                 */
  double seconds;      /* device time of the solve                            */
} sod_solve_stats_t;
int sod_gpu_pressure_solve(sod_gpu_ctx *ctx, const double *b, double *x, const sod_solve_opts_t *opts,
                           sod_solve_stats_t *stats);

/* ---- learned element-patch preconditioner (no counterpart in the reference)
 * Per element: the Jacobi-scaled residual on its nodes and the element means
 * of its 6 face neighbours, scaled to unit RMS, pass through a 32-32 tanh
 * MLP whose output corrects the Jacobi step on the element's nodes; element
 * outputs are averaged at shared nodes.  With a zero output layer (the
 * initial state) it is exactly Jacobi.  Trained on the GPU by this library's
 * own forward, backward and Adam kernels to minimise the energy norm
 * ||e - M(r)||_A^2 / ||e||_A^2 over (residual, error) pairs harvested from
 * the library's Jacobi pressure solves. */
int sod_gpu_precond_num_params(sod_gpu_ctx *ctx);
/* Allocates the network and a harvest ring of `harvest_capacity` pairs and
 * sets seeded initial parameters. */
int sod_gpu_precond_init(sod_gpu_ctx *ctx, uint64_t seed, int harvest_capacity);
int sod_gpu_precond_set_params(sod_gpu_ctx *ctx, const float *host_params, int n);
int sod_gpu_precond_get_params(sod_gpu_ctx *ctx, float *host_params, int n);
/* z = M(r) on working nodes (device FP64 vectors). */
int sod_gpu_precond_apply(sod_gpu_ctx *ctx, const double *r, double *z);
/* Loss ||e - M(r)||_A^2/||e||_A^2 (host *loss) and its parameter gradient
 * (host grad, nparam floats, may be NULL) for one pair; no update. */
int sod_gpu_precond_loss_grad(sod_gpu_ctx *ctx, const double *r, const double *e, double *loss,
                              float *grad_host);
/* Number of harvested pairs available for training. */
int sod_gpu_precond_harvest_count(sod_gpu_ctx *ctx);
/* Start a new harvest and training phase: drop the harvested pairs and the
 * Adam moments, keep the parameters.  Solves with precond = 1 and
 * harvest = 1 then record pairs from the learned map's own iterations,
 * and sod_gpu_precond_train fine-tunes on them. */
int sod_gpu_precond_restart_harvest(sod_gpu_ctx *ctx);
/* Adam: `steps` updates over mini-batches of `batch` (<= 16) harvested
 * pairs; *final_loss (host) = mean loss of the last batch. */
int sod_gpu_precond_train(sod_gpu_ctx *ctx, int steps, int batch, float lr, uint64_t seed, float *final_loss);

/* ---- implicit velocity solve of the incompressible step -----------------
 * species_tau, src/lib_species/sources/elem_stab_species.f90:122-148:
 * tau(nelem) = max over element nodes of helem (c_species_stab/p) |u|. */
int sod_gpu_species_tau(sod_gpu_ctx *ctx, const float *u, float *tau);
/* eval_tau_veloc, src/lib_sod2d_incomp/sources/mod_operators.f90:373-483:
 * GradX/Y/Z(npoin,3) = assembled gpvol (grad u + grad u^T) rows / Ml. */
int sod_gpu_eval_tau_veloc(sod_gpu_ctx *ctx, const float *u, float *GradX, float *GradY, float *GradZ);
/* full_diff_stab_incomp, src/lib_sod2d_incomp/sources/elem_stab_incomp.f90:
 * 12-153: Rmom(npoin,3) (overwritten) = assembled weak divergence of
 * (mu_fluid + mu_sgs + tau)(grad u + grad u^T) - tau TauP; mu_sgs is
 * (nelem,ngaus) and may be NULL (zero). */
int sod_gpu_full_diff_stab_incomp(sod_gpu_ctx *ctx, const float *u, const float *mu_fluid, const float *mu_sgs,
                                  const float *TauPX, const float *TauPY, const float *TauPZ,
                                  const float *tau_stab, float *Rmom);
/* conjGrad_veloc_incomp (LPS path, periodic mesh),
 * src/lib_sod2d_incomp/sources/mod_solver_incomp.f90:27-251: preconditioned
 * CG on Ml x + fact dt D(x) = R, D = full_diff_stab_incomp with the LPS
 * projection of its argument, preconditioner Ml/dt, x0 = Rp0, tau from
 * species_tau(Rp0); FP32 vectors, FP64 dots, the reference's arithmetic.
 * R (npoin,3): in the right-hand side, out the solution. */
int sod_gpu_conjgrad_veloc(sod_gpu_ctx *ctx, float fact, float dt, const float *mu_fluid, const float *mu_sgs,
                           const float *Rp0, float *R, int maxIter, double tol, int *iters, double *res_rel);

/* ---- incompressible time step (library-owned state) ---------------------
 * bdfext3_main_incomp on a periodic mesh without wall model, source term or
 * LES, src/lib_sod2d_incomp/sources/time_integ_incomp.f90:88-433, rho = 1,
 * mu_fluid = nu, with BDF coefficients (g0, a) and extrapolation
 * coefficients (b) of order 1, 2 and 3 on the first, second and later steps:
 *   Rmom2 = full_convec_ijk_incomp(u1, u1, 1)
 *   u2 = (-dt (b1 Rmom2 + b2 Rmom1 + b3 Rmom3) / Ml + a1 u1 + a2 u3 + a3 u4) / g0
 *   A p = -g0 eval_divergence(u2) / dt   solved by sod_gpu_pressure_solve
 *   u2 = (u2 - dt eval_gradient(p) / g0) Ml
 *   u2 = sod_gpu_conjgrad_veloc(fact 1/g0, dt, mu_fluid, x0 = u1, R = u2)
 * then the levels rotate (u4 = u3, u3 = u1, u1 = u2; CFDSolverBase.f90:
 * 1953-2015).  The pressure solve starts from the previous pressure
 * (Jacobi, the reference's pr(:,1)) or from 2 p^n - p^(n-1) (learned).
 * init needs helem (species_tau of the velocity solve) and sets every level
 * to u. */
int sod_gpu_incomp_init(sod_gpu_ctx *ctx, const float *u, double nu);
int sod_gpu_incomp_step(sod_gpu_ctx *ctx, float dt, const sod_solve_opts_t *opts, sod_solve_stats_t *stats);
/* maxIter and tol of the velocity solve (defaults 20 and 1e-4,
 * mod_numerical_params.f90:50-51). */
int sod_gpu_incomp_set_veloc_solver(sod_gpu_ctx *ctx, int maxIter, double tol);
/* Iterations and ||r||/||r0|| of the last step's velocity solve (host). */
int sod_gpu_incomp_veloc_stats(sod_gpu_ctx *ctx, int *iters, double *res_rel);
/* Copies of the current velocity u(npoin,3) (FP32) and pressure (FP64); NULL skips. */
int sod_gpu_incomp_get(sod_gpu_ctx *ctx, float *u, double *p);
/* Pressure of the initial state (FP64, device), the first step's pr(:,1). */
int sod_gpu_incomp_set_pressure(sod_gpu_ctx *ctx, const double *p);
/* Convective CFL time step of the current velocity (host *dt):
 * adapt_dt_cfl with zero sound speed, as CFDSolverPeriodicIncomp_evalDt
 * (src/lib_mainBaseClass/sources/CFDSolverPeriodicIncomp.f90:119-128). */
int sod_gpu_incomp_adapt_dt(sod_gpu_ctx *ctx, float cfl_conv, float *dt);
/* volAvg_EK and visc_dissipationRate of the current velocity (rho = 1,
 * mu_fluid = nu, no entropy viscosity): out (host) = EK, eps_S, eps_D,
 * eps_T (src/lib_sod2d/sources/mod_analysis.f90:10-144). */
int sod_gpu_incomp_analysis(sod_gpu_ctx *ctx, double *out);

/* ---- entropy viscosity, individually (device pointers, reference layout) */
/* generic_scalar_convec_ijk, src/lib_sod2d/sources/elem_convec.f90:472-594:
 * assembled split-form residual of a scalar eta with flux q(npoin,3) and
 * velocity u(npoin,3) into R(npoin) (zeroed first when initialze != 0),
 * scaled by fact; not mass-inverted. */
int sod_gpu_generic_scalar_convec_ijk(sod_gpu_ctx *ctx, const float *q, const float *eta, const float *u, float *R,
                                      int initialze, float fact);
/* smart_visc_spectral_imex, src/lib_sod2d/sources/mod_entropy_viscosity.f90:
 * 113-227 (high-Mach path): mu_e(nelem,ngaus) from the entropy residual
 * Reta(npoin), rho, u, csound; needs helem at init. */
int sod_gpu_smart_visc_spectral_imex(sod_gpu_ctx *ctx, const float *Reta, const float *rho, const float *u,
                                     const float *csound, float *mu_e);
/* ducros_visc_limit, src/lib_sod2d/sources/mod_entropy_viscosity.f90:277-314:
 * mu_e(nelem,ngaus) (in/out) scaled by the Ducros sensor of divU (assembled,
 * eval_divergence), vorti(npoin,3) (compute_vorticity) and |u| / helem_l;
 * rho and csound only feed a quantity the reference discards.  Needs helem_l
 * at init. */
int sod_gpu_ducros_visc_limit(sod_gpu_ctx *ctx, const float *rho, const float *u, const float *divU,
                              const float *vorti, const float *csound, float *mu_e);

/* The stage update of rk_4_ls_main on the caller's FP32 arrays (working
 * nodes): first != 0: U2 += (gam dt) R (time_integ_ls.f90:325-329, U1 may be
 * NULL); otherwise U2 = lam1 U1 + lami U2 + (gam dt) R (:352-356), with
 * lam1 = lambda_ij(istep+1,1), lami = lambda_ij(istep+1,istep), gam =
 * gamma_ij(istep+1,istep).  Fields rho, q(npoin,3), E; R* mass-inverted. */
int sod_gpu_rk_ls_stage(sod_gpu_ctx *ctx, int first, float lam1, float lami, float gam, float dt, const float *rho1,
                        const float *q1, const float *E1, float *rho2, float *q2, float *E2, const float *Rmass,
                        const float *Rmom, const float *Rener);

/* ---- compressible time integration with library-owned state ----------
 * The conserved state lives on the device in FP64 (fp64_state = 1) or in
 * FP32 (fp64_state = 0, the reference's USE_RP=4 arithmetic); the element
 * kernels always read an FP32 copy.  The step restates rk_4_ls_main,
 * src/lib_sod2d/sources/time_integ_ls.f90:202-487, for periodic meshes:
 * first-step entropy viscosity, the low-storage stages (stage 1 reuses the
 * residual left by the previous step), end-of-step equation of state,
 * thermodynamic entropy, entropy residual, smart_visc_spectral_imex with
 * the Ducros limiter, Sutherland viscosity. */
typedef struct {
  int stages;      /* 3, 4 (SSPRK(4,3)) or 5 (SSP53_2N)                    */
  int rk_n;        /* SSP53_2N variant (1..4) when stages == 5             */
  int fp64_state;  /* 1: FP64 conserved state, 0: FP32                      */
  float mu_factor; /* Sutherland scale flag_mu_factor                      */
} sod_rk_cfg_t;

/* Level-2 initial state (device pointers, reference layout): rho, u(N,3),
 * q(N,3), pr, E, Tem, csound, machno, eta.  mu_e starts at zero. */
int sod_gpu_comp_init_state(sod_gpu_ctx *ctx, const sod_rk_cfg_t *cfg, const float *rho, const float *u,
                            const float *q, const float *pr, const float *E, const float *Tem,
                            const float *csound, const float *machno, const float *eta);
/* One time step of size dt. */
int sod_gpu_comp_rk_ls_step(sod_gpu_ctx *ctx, float dt);
/* One step of the IMEX integrator instead of the RK step: imex_main,
 * src/lib_sod2d/sources/time_integ_imex.f90:181-525, for a periodic case
 * (no wall model, source terms or LES): explicit convection, implicit
 * diffusion with the LPS stabilisation of the step's initial state, the
 * ARK tables of init_imex_solver (time_integ_imex.f90:42-158) for 3 or 4
 * stages (sod_rk_cfg_t.stages), and per implicit stage conjGrad_imex
 * (src/lib_sod2d/sources/mod_solver_imex.f90:25-342) with maxIter and tol
 * (the reference's defaults 200 and 1e-3, TGVCompSolver.f90:90-93); then
 * the entropy viscosity and Sutherland update of the RK step.  Needs
 * fp64_state = 0 (the reference's FP32 state). */
int sod_gpu_comp_imex_step(sod_gpu_ctx *ctx, float dt, int maxIter, double tol);
/* CG iterations summed over the last IMEX step's stages and the last
 * stage's ||r||/||r0|| (host). */
int sod_gpu_comp_imex_stats(sod_gpu_ctx *ctx, int *cg_iters, double *cg_res);
/* CFL time step (adapt_dt_cfl, src/lib_sod2d/sources/mod_time_ops.f90:11-62),
 * written to *dt (host). */
int sod_gpu_comp_adapt_dt(sod_gpu_ctx *ctx, float cfl_conv, float cfl_diff, float *dt);
/* Analysis integrals (mod_analysis.f90:10-168): out[0..4] (host) = EK,
 * eps_S, eps_D, eps_T, max Mach; FP64 accumulation across elements. */
int sod_gpu_comp_analysis(sod_gpu_ctx *ctx, float rho0, double *out);
/* Copies of the current state (device pointers, reference layout; any may
 * be NULL): rho, q(N,3), E and mu_e(nelem,ngaus). */
int sod_gpu_comp_get_state(sod_gpu_ctx *ctx, float *rho, float *q, float *E, float *mu_e);

/* ---- allocation-free analysis integrals ---------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory (a solver whose device memory belongs to its own pool or is
 * capped, callers that must not let cudaMalloc synchronise the device
 * inside the time loop), this
 * computes the same integrals as sod_gpu_comp_analysis without a context:
 * every input is a device pointer in the reference layout (connec, lpoin_w
 * 1-based; He(3,3,ngaus,nelem), gpvol, dlxigp_ip, Ngp (may be NULL), rho,
 * u(npoin,3), mu_fluid, mu_e(nelem,ngaus), machno) and out[0..4] (host)
 * receives EK, eps_S, eps_D, eps_T, max Mach.  volT is the domain volume.
 * It allocates nothing: its scratch is a fixed __device__ array of
 * SOD_NOALLOC_MAX_ELEM x 3 floats (12 MiB) that each GPU loading the
 * library keeps until the process exits; larger meshes are rejected with
 * SOD_GPU_EINVAL.  Every call looks up the array's device address in the
 * current context (cudaGetSymbolAddress; the first call in a context also
 * loads the library's device code there).  All calls share the array, so
 * calls that overlap on the GPU race; serialise them.  Work is enqueued on
 * `stream` (NULL = default); the call copies the results into the host
 * array out and waits on `stream` for them before it returns. */
#define SOD_NOALLOC_MAX_ELEM (1 << 20)
int sod_gpu_analysis_noalloc(int porder, int nelem, int npoin, int npoin_w, const int *connec,
                             const int *lpoin_w, const int *invAtoIJK, const int *gmshAtoI,
                             const int *gmshAtoJ, const int *gmshAtoK, const float *dlxigp_ip,
                             const float *He, const float *gpvol, const float *Ngp, const float *rho,
                             const float *u, const float *mu_fluid, const float *mu_e,
                             const float *machno, float rho0, float volT, void *stream, double *out);

#ifdef __cplusplus
}
#endif
#endif
