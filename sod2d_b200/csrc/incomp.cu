// C-ABI entry points of the incompressible path: Laplacian, gradient,
// divergence and convection operators, the reference-arithmetic and the
// FP64-certified pressure CG, the implicit velocity solve and the
// BDF3/EXT3 step (declarations: include/sod2d_gpu.h).
#include "cg_common.cuh"

extern "C" {

int sod_gpu_eval_laplacian_mult(sod_gpu_ctx *c, const float *p, float *ResP) {
  if (!c || !p || !ResP) return fail(SOD_GPU_EINVAL, "bad argument");
  CUDA_TRY(cudaMemsetAsync(ResP, 0, (size_t)c->npoin * 4, c->stream));
  lap<float>(c, p, ResP);
  int rc = halo_sum(c, halo_soa_view(c, ResP, 1));  // mod_operators.f90:102
  return rc ? rc : c->finish();
}

int sod_gpu_eval_laplacian_mult64(sod_gpu_ctx *c, const double *p, double *ResP) {
  if (!c || !p || !ResP) return fail(SOD_GPU_EINVAL, "bad argument");
  CUDA_TRY(cudaMemsetAsync(ResP, 0, (size_t)c->npoin * 8, c->stream));
  lap<double>(c, p, ResP);
  HaloViewT<double> hv{};
  hv.width = 1;
  hv.nstride = 1;
  hv.comp[0] = ResP;
  int rc = halo_sum<double>(c, hv);  // mod_operators.f90:102
  return rc ? rc : c->finish();
}

int sod_gpu_eval_laplacian_diag(sod_gpu_ctx *c, float *d) {
  if (!c || !d) return fail(SOD_GPU_EINVAL, "bad argument");
  int rc = ensure_diag(c);
  if (rc) return rc;
  CUDA_TRY(cudaMemcpyAsync(d, c->cg.diag, (size_t)c->npoin * 4, cudaMemcpyDeviceToDevice, c->stream));
  return c->finish();
}

int sod_gpu_eval_gradient(sod_gpu_ctx *c, const float *x, float *gradX) {
  if (!c || !x || !gradX) return fail(SOD_GPU_EINVAL, "bad argument");
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    k_vec_elem<LL::P_, LL::EPB, 0><<<LL::grid(c->nelem), LL::TPB, 0, c->stream>>>(c->md(), x, nullptr, nullptr, c->slotsB);
    return 0;
  });
  OutPtrs o{};
  const long long N = c->npoin;
  o.p[0] = gradX; o.p[1] = gradX + N; o.p[2] = gradX + 2 * N;
  k_gather<4, 3, false><<<nblk(N, 256), 256, 0, c->stream>>>(c->md(), c->slotsB, nullptr, o, 0, 1);
  int rc = halo_sum(c, halo_soa_view(c, gradX, 3));  // mod_operators.f90:274
  return rc ? rc : c->finish();
}

int sod_gpu_eval_divergence(sod_gpu_ctx *c, const float *u, float *divU) {
  if (!c || !u || !divU) return fail(SOD_GPU_EINVAL, "bad argument");
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    k_vec_elem<LL::P_, LL::EPB, 1><<<LL::grid(c->nelem), LL::TPB, 0, c->stream>>>(c->md(), nullptr, u, nullptr, c->slotsB);
    return 0;
  });
  OutPtrs o{};
  o.p[0] = divU;
  k_gather<4, 1, false><<<nblk(c->npoin, 256), 256, 0, c->stream>>>(c->md(), c->slotsB, nullptr, o, 0, 0);
  int rc = halo_sum(c, halo_soa_view(c, divU, 1));  // mod_operators.f90:566
  return rc ? rc : c->finish();
}

int sod_gpu_full_convec_ijk_incomp(sod_gpu_ctx *c, const float *u, const float *q, float *Rmom) {
  if (!c || !u || !q || !Rmom) return fail(SOD_GPU_EINVAL, "bad argument");
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    k_vec_elem<LL::P_, LL::EPB, 2><<<LL::grid(c->nelem), LL::TPB, 0, c->stream>>>(c->md(), nullptr, u, q, c->slotsB);
    return 0;
  });
  OutPtrs o{};
  const long long N = c->npoin;
  o.p[0] = Rmom; o.p[1] = Rmom + N; o.p[2] = Rmom + 2 * N;
  k_gather<4, 3, false><<<nblk(N, 256), 256, 0, c->stream>>>(c->md(), c->slotsB, nullptr, o, 0, 0);
  return c->finish();
}

int sod_gpu_conjgrad_pressure(sod_gpu_ctx *c, const float *Rp0, float *R, int maxIter, double tol, int *iters,
                              double *res_rel) {
  if (!c || !Rp0 || !R || maxIter < 1) return fail(SOD_GPU_EINVAL, "bad argument");
  int rc;
  if ((rc = ensure_diag(c)) || (rc = ensure_cg32(c))) return rc;
  auto &G = c->cg;
  const size_t N = c->npoin;
  const cudaStream_t st = c->stream;
  for (float *z : {G.x32, G.r32, G.p32, G.q32, G.z032, G.z132, G.b32}) CUDA_TRY(cudaMemsetAsync(z, 0, N * 4, st));
  // b = R - A x0 ; r0 = b ; z0 = r0 / M ; p0 = z0   (mod_solver_incomp.f90:310-350)
  lap<float>(c, Rp0, G.q32);
  if ((rc = halo_sum(c, halo_soa_view(c, G.q32, 1)))) return rc;
  const int nw = c->npoin_w;
  k_axpby<float><<<nblk(nw, 256), 256, 0, st>>>(nw, c->lpoin_w, -1.f, G.q32, 0.f, G.b32);
  k_axpby<float><<<nblk(nw, 256), 256, 0, st>>>(nw, c->lpoin_w, 1.f, R, 1.f, G.b32);
  k_axpby<float><<<nblk(nw, 256), 256, 0, st>>>(nw, c->lpoin_w, 1.f, G.b32, 0.f, G.r32);
  {
    // z0 = r0 / M, p0 = z0 via one update with a = 0
    DotArgs<float, 1> A{{G.b32}, {G.b32}, {nullptr}};
    dots<float, 1>(c, A, G.dots + 6);  // ||b||^2
    if ((rc = allreduce(c, G.dots + 6, 1, SOD_REDUCE_SUM_F64))) return rc;  // mod_solver_incomp.f90:366
  }
  // z0 = r/M
  {
    const double one_zero[2] = {0.0, 1.0};
    CUDA_TRY(cudaMemcpyAsync(G.dots + 4, one_zero, 16, cudaMemcpyHostToDevice, st));
    k_cg_update1<float><<<nblk(nw, 256), 256, 0, st>>>(nw, c->lpoin_w, G.dots + 4, G.x32, G.r32, G.p32, G.q32,
                                                       G.z032, G.z132, G.diag, 1, 1);
    k_axpby<float><<<nblk(nw, 256), 256, 0, st>>>(nw, c->lpoin_w, 1.f, G.z032, 0.f, G.p32);
  }
  double hb[1];
  CUDA_TRY(cudaMemcpyAsync(hb, G.dots + 6, 8, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  const double auxB = std::sqrt(hb[0]);
  int it;
  double nrm = auxB;
  for (it = 1; it <= maxIter; ++it) {
    lap<float>(c, G.p32, G.q32);
    if ((rc = halo_sum(c, halo_soa_view(c, G.q32, 1)))) return rc;
    dots<float, 2>(c, DotArgs<float, 2>{{G.r32, G.p32}, {G.z032, G.q32}, {nullptr, nullptr}}, G.dots);  // Q1, Q2
    if ((rc = allreduce(c, G.dots, 2, SOD_REDUCE_SUM_F64))) return rc;  // mod_solver_incomp.f90:388
    k_cg_update1<float><<<nblk(nw, 256), 256, 0, st>>>(nw, c->lpoin_w, G.dots, G.x32, G.r32, G.p32, G.q32, G.z032,
                                                       G.z132, G.diag, 1, 1);
    // ||r||^2 and <r, z0 - z1>
    dots<float, 2>(c, DotArgs<float, 2>{{G.r32, G.r32}, {G.r32, G.z032}, {nullptr, G.z132}}, G.dots + 2);
    if ((rc = allreduce(c, G.dots + 2, 2, SOD_REDUCE_SUM_F64))) return rc;  // mod_solver_incomp.f90:415, 437
    double h[2];
    CUDA_TRY(cudaMemcpyAsync(h, G.dots + 2, 16, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    nrm = std::sqrt(h[0]);
    if (!std::isfinite(nrm)) return fail(SOD_GPU_ENONFINITE, "non-finite residual in pressure CG");
    if (nrm < tol * auxB) break;
    k_cg_update2<float><<<nblk(nw, 256), 256, 0, st>>>(nw, c->lpoin_w, G.dots, G.dots + 2, G.p32, G.z032);
  }
  // R = x0 + x on every node (x is zero off the working nodes)
  k_add_all<float><<<nblk(N, 256), 256, 0, st>>>((long long)N, Rp0, G.x32, R);
  if (iters) *iters = it > maxIter ? maxIter : it;
  if (res_rel) *res_rel = auxB > 0 ? nrm / auxB : 0.0;
  return c->finish();
}

}  // extern "C"

namespace {

// ---- FP64 flexible CG with certified residual ----------------------------

__global__ void k_sub_mean(int npoin_w, const int *__restrict__ lpoin_w, const double *__restrict__ sum_in,
                           double *__restrict__ b) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  b[lpoin_w[t]] -= sum_in[0] / (double)npoin_w;
}

// per-block partial sums of b over the working nodes (fixed order); the
// final sum over blocks is k_dot_final
__global__ void k_sum_partial(int npoin_w, const int *__restrict__ lpoin_w, const double *__restrict__ b,
                              double *__restrict__ part) {
  __shared__ double sh[DOT_THREADS];
  double s = 0.0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < npoin_w; t += gridDim.x * blockDim.x) s += b[lpoin_w[t]];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}


// r = b - q over working nodes
__global__ void k_resid(int npoin_w, const int *__restrict__ lpoin_w, const double *__restrict__ b,
                        const double *__restrict__ q, double *__restrict__ r) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const int i = lpoin_w[t];
  r[i] = b[i] - q[i];
}

// b -= sc[0] / sc[1] on the working nodes (sum and count of the mean)
__global__ void k_sub_ratio(int npoin_w, const int *__restrict__ lpoin_w, const double *__restrict__ sc,
                            double *__restrict__ b) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  b[lpoin_w[t]] -= sc[0] / sc[1];
}

// z = M r on the working nodes
__global__ void k_mul_w(int npoin_w, const int *__restrict__ lpoin_w, const double *__restrict__ M,
                        const double *__restrict__ r, double *__restrict__ z) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const int i = lpoin_w[t];
  z[i] = M[i] * r[i];
}

// The FP64 Jacobi-PCG of sod_gpu_pressure_solve on a partitioned mesh,
// driven from the host: the Laplacian and its diagonal are summed over the
// ranks, the mean of b and every dot product run over the owned nodes and
// are summed over the ranks (the reference's lpoin_o and MPI_Allreduce,
// mod_solver_incomp.f90:366-437), and convergence is declared on the true
// FP64 residual ||b - A x|| / ||b||, as in the single-rank solve.
int pressure_solve_parts(sod_gpu_ctx *c, const double *b_in, double *x, const sod_solve_opts_t *opts,
                         sod_solve_stats_t *stats) {
  int rc;
  if ((rc = ensure_diag(c)) || (rc = ensure_cg64(c))) return rc;
  auto &G = c->cg;
  auto &h = c->halo;
  const size_t N = c->npoin;
  const int nw = c->npoin_w;
  const cudaStream_t st = c->stream;
  const unsigned nb = nblk(nw, 256);
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));
  CUDA_TRY(cudaEventRecord(e0, st));
  k_inv_diag64<<<nblk(N, 256), 256, 0, st>>>((long long)N, G.diag, G.Minv);
  CUDA_TRY(cudaMemcpyAsync(G.b, b_in, N * 8, cudaMemcpyDeviceToDevice, st));
  // mean of b over the whole mesh: sum and count over the owned nodes
  k_sum_partial<<<DOT_BLOCKS, DOT_THREADS, 0, st>>>(h.npoin_o, h.lpoin_o, G.b, G.part);
  k_dot_final<<<1, 1024, 0, st>>>(1, G.part, G.dots + 7);
  const double cnt = (double)h.npoin_o;
  CUDA_TRY(cudaMemcpyAsync(G.dots + 8, &cnt, 8, cudaMemcpyHostToDevice, st));
  if ((rc = allreduce(c, G.dots + 7, 2, SOD_REDUCE_SUM_F64))) return rc;
  k_sub_ratio<<<nb, 256, 0, st>>>(nw, c->lpoin_w, G.dots + 7, G.b);
  auto apply = [&](const double *v, double *out) -> int {
    lap<double>(c, v, out);
    HaloViewT<double> hv{};
    hv.width = 1;
    hv.nstride = 1;
    hv.comp[0] = out;
    return halo_sum<double>(c, hv);
  };
  // a . b and c . d over the owned nodes, summed over the ranks
  auto dot2 = [&](const double *a, const double *bb, const double *cc, const double *dd, double *out2) -> int {
    dots<double, 2>(c, DotArgs<double, 2>{{a, cc}, {bb, dd}, {nullptr, nullptr}}, G.dots);
    int r2 = allreduce(c, G.dots, 2, SOD_REDUCE_SUM_F64);
    if (r2) return r2;
    CUDA_TRY(cudaMemcpyAsync(out2, G.dots, 16, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return 0;
  };
  double d2[2];
  if ((rc = dot2(G.b, G.b, G.b, G.b, d2))) return rc;
  const double bnorm = std::sqrt(d2[0]);
  int it = 0;
  double res = 0.0;
  bool converged = false;
  if (bnorm == 0.0) {
    CUDA_TRY(cudaMemsetAsync(x, 0, N * 8, st));
    converged = true;
  }
  int restarts = 0;
  while (!converged && it < opts->max_iter) {
    // (re)start from the true residual: r = b - A x, z = M r, p = z
    if ((rc = apply(x, G.q))) return rc;
    k_resid<<<nb, 256, 0, st>>>(nw, c->lpoin_w, G.b, G.q, G.r);
    k_mul_w<<<nb, 256, 0, st>>>(nw, c->lpoin_w, G.Minv, G.r, G.z0);
    k_axpby<double><<<nb, 256, 0, st>>>(nw, c->lpoin_w, 1.0, G.z0, 0.0, G.p);
    if ((rc = dot2(G.r, G.z0, G.r, G.r, d2))) return rc;
    res = std::sqrt(d2[1]) / bnorm;
    if (res < opts->tol) { converged = true; break; }
    if (++restarts > 4) return fail(SOD_GPU_ESTAGNATE, "pressure solve made no progress");
    double rz = d2[0];
    while (it < opts->max_iter) {
      if ((rc = apply(G.p, G.q))) return rc;
      if ((rc = dot2(G.p, G.q, G.p, G.q, d2))) return rc;
      if (!(d2[0] > 0.0)) break;  // loss of positivity: restart from the true residual
      const double alpha = rz / d2[0];
      k_axpby<double><<<nb, 256, 0, st>>>(nw, c->lpoin_w, alpha, G.p, 1.0, x);
      k_axpby<double><<<nb, 256, 0, st>>>(nw, c->lpoin_w, -alpha, G.q, 1.0, G.r);
      k_mul_w<<<nb, 256, 0, st>>>(nw, c->lpoin_w, G.Minv, G.r, G.z0);
      if ((rc = dot2(G.r, G.z0, G.r, G.r, d2))) return rc;
      ++it;
      if (!std::isfinite(d2[1])) return fail(SOD_GPU_ENONFINITE, "non-finite residual in pressure solve");
      if (std::sqrt(d2[1]) / bnorm < opts->tol) break;  // certify on the true residual
      const double beta = d2[0] / rz;
      rz = d2[0];
      k_axpby<double><<<nb, 256, 0, st>>>(nw, c->lpoin_w, 1.0, G.z0, beta, G.p);
    }
  }
  CUDA_TRY(cudaEventRecord(e1, st));
  CUDA_TRY(cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (stats) {
    stats->iterations = it;
    stats->fallback = 0;
    stats->res_rel = res;
    stats->seconds = ms * 1e-3;
  }
  if (!converged) return fail(SOD_GPU_ESTAGNATE, "pressure solve did not reach the tolerance");
  return c->finish();
}

}  // namespace

extern "C" {

int sod_gpu_pressure_solve(sod_gpu_ctx *c, const double *b_in, double *x, const sod_solve_opts_t *opts,
                           sod_solve_stats_t *stats) {
  if (!c || !b_in || !x || !opts || opts->max_iter < 1 || !(opts->tol > 0)) return fail(SOD_GPU_EINVAL, "bad argument");
  if (opts->precond != 0 && opts->precond != 1) return fail(SOD_GPU_EINVAL, "precond must be 0 or 1");
  if (c->halo.on) {
    if (opts->precond != 0)
      return fail(SOD_GPU_EINVAL, "the learned preconditioner is not available with a halo plan");
    return pressure_solve_parts(c, b_in, x, opts, stats);
  }
  int rc;
  if ((rc = ensure_diag(c)) || (rc = ensure_cg64(c)) || (rc = ensure_cg_loop(c))) return rc;
  auto &G = c->cg;
  const size_t N = c->npoin;
  const int nw = c->npoin_w;
  const cudaStream_t st = c->stream;
  const unsigned nb = nblk(nw, 256);
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));
  CUDA_TRY(cudaEventRecord(e0, st));
  k_inv_diag64<<<nblk(N, 256), 256, 0, st>>>((long long)N, G.diag, G.Minv);
  // b := b_in with its mean removed (range of the periodic Laplacian)
  CUDA_TRY(cudaMemcpyAsync(G.b, b_in, N * 8, cudaMemcpyDeviceToDevice, st));
  k_sum_partial<<<DOT_BLOCKS, DOT_THREADS, 0, st>>>(nw, c->lpoin_w, G.b, G.part);
  k_dot_final<<<1, 1024, 0, st>>>(1, G.part, G.dots + 7);
  k_sub_mean<<<nb, 256, 0, st>>>(nw, c->lpoin_w, G.dots + 7, G.b);
  dots<double, 1>(c, DotArgs<double, 1>{{G.b}, {G.b}, {nullptr}}, G.dots + 6);
  double hb;
  CUDA_TRY(cudaMemcpyAsync(&hb, G.dots + 6, 8, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  const double bnorm = std::sqrt(hb);
  int kind = opts->precond;
  int it = 0, fallback = 0;
  double res = 0.0;
  const int window = opts->stagnation_window > 0 ? opts->stagnation_window : 50;
  auto &NT = c->net;
  if (kind == 1) {
    if (!NT.ready) return fail(SOD_GPU_EINVAL, "learned preconditioner not set up (sod_gpu_precond_init)");
    if ((rc = ensure_gains(c))) return rc;
  }
  // harvest snapshots (x_k, r_k) after k = 0..8, 16, 32, ... iterations, from
  // Jacobi solves (first training) or from solves with the learned map
  // itself (fine-tuning on the residuals it meets)
  const bool harvest = opts->harvest && NT.ready && NT.cap > 0;
  struct Snap {
    int slot, si, iter;
    bool fresh;
  };
  std::vector<Snap> snaps;
  int next_snap = 0;
  auto enqueue_snapshot = [&](int iter_no) {
    if (!harvest || (int)snaps.size() >= 16 || iter_no != next_snap) return;
    next_snap = next_snap < 8 ? next_snap + 1 : next_snap * 2;
    // reservoir sampling over every pair offered so far (seeded, reproducible)
    int slot;
    bool fresh = false;
    if (NT.count < NT.cap) {
      slot = NT.count++;
      fresh = true;
    } else {
      NT.rs_state = NT.rs_state * 6364136223846793005ULL + 1442695040888963407ULL;
      const long long j = (long long)((NT.rs_state >> 11) % (uint64_t)(NT.offered + 1));
      slot = j < NT.cap ? (int)j : -1;
    }
    NT.offered++;
    if (slot < 0) return;
    const int si = (int)snaps.size();
    k_cg_snapshot<<<nb, 256, 0, st>>>(nw, c->lpoin_w, x, G.r, NT.xsnap + (size_t)si * N, NT.hr + (size_t)slot * N,
                                      G.S);
    snaps.push_back({slot, si, iter_no, fresh});
  };
  auto read_scalars = [&]() -> int {
    CUDA_TRY(cudaMemcpyAsync(G.S_h, G.S, sizeof(CgScal), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaMemcpyAsync(G.hist_h, G.hist, sizeof(double) * CG_HIST, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return 0;
  };
  // (re)start from the true FP64 residual: r = b - A x, z = M r, p = z
  auto restart = [&]() -> int {
    lap<double>(c, x, G.q);
    k_resid<<<nb, 256, 0, st>>>(nw, c->lpoin_w, G.b, G.q, G.r);
    int rc2 = apply_precond(c, kind, G.r, G.z0);
    if (rc2) return rc2;
    dots<double, 2>(c, DotArgs<double, 2>{{G.r, G.r}, {G.z0, G.r}, {nullptr, nullptr}}, G.dots + 2);  // r.z, r.r
    k_axpby<double><<<nb, 256, 0, st>>>(nw, c->lpoin_w, 1.0, G.z0, 0.0, G.p);
    k_cg_start<<<1, 1, 0, st>>>(G.S, G.dots + 2, bnorm * bnorm * opts->tol * opts->tol, it);
    return 0;
  };
  auto certify = [&]() -> int {
    lap<double>(c, x, G.q);
    k_resid<<<nb, 256, 0, st>>>(nw, c->lpoin_w, G.b, G.q, G.r);
    dots<double, 1>(c, DotArgs<double, 1>{{G.r}, {G.r}, {nullptr}}, G.dots + 2);
    double h1;
    CUDA_TRY(cudaMemcpyAsync(&h1, G.dots + 2, 8, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    res = std::sqrt(h1) / bnorm;
    return 0;
  };
  // one iteration, entirely on the device: p = z + beta p, q = A p, alpha,
  // x/r update, z = M r, beta
  auto iteration = [&]() {
    const MeshDev md = c->md();
    dispatch(c, [&](auto L) {
      using LL = decltype(L);
      constexpr int P = LL::P_;
      // the search direction p = z + beta p is formed inside these two
      k_lap_elem<P, LL::EPB, double, true><<<LL::grid(c->nelem), LL::TPB, 0, st>>>(
          md, G.p, (double *)c->slotsB, &G.S->status, G.z0, &G.S->beta);
      k_cg_q<true><<<cg_blocks(c->npoin, 2), CG_THREADS, 0, st>>>(md, (const double *)c->slotsB, G.p, G.q, G.S,
                                                                  G.gpart, G.ticket, G.z0);
      if (kind == 0) {
        k_cg_update<true><<<cg_blocks(nw, CG_U), CG_THREADS, 0, st>>>(nw, c->lpoin_w, G.p, G.q, G.Minv, x, G.r, G.z0,
                                                                     G.S, G.hist, CG_HIST, G.gpart, G.ticket);
      } else {
        using D = NetDims<P>;
        k_cg_update<false><<<cg_blocks(nw, CG_U), CG_THREADS, 0, st>>>(nw, c->lpoin_w, G.p, G.q, G.Minv, x, G.r,
                                                                      G.z0, G.S, G.hist, CG_HIST, G.gpart,
                                                                      G.ticket, NT.Dh, NT.uf);
        k_patch_apply_tc<P><<<tc_grid<P>(c->nelem), TC_THREADS, TcDims<P>::smem(), st>>>(
            c->nelem, NT.pt, NT.pos, NT.uf, NT.params, NT.gains, c->slotsB, &G.S->status);
        k_cg_patch_z<<<cg_blocks(c->npoin, CG_U), CG_THREADS, 0, st>>>(c->npoin, NT.pptr, c->slotsB, G.r, NT.Dh,
                                                                       NT.params, D::O_ALPHA, G.z0, G.S, G.gpart,
                                                                       G.ticket);
      }
      return 0;
    });
  };
  if (bnorm == 0.0) {
    CUDA_TRY(cudaMemsetAsync(x, 0, N * 8, st));
  } else {
    bool converged = false;
    int breakdowns = 0;
    while (!converged && it < opts->max_iter) {
      if ((rc = restart())) return rc;
      if (it == 0) enqueue_snapshot(0);
      double best = 1e300;
      int best_it = it, batch = kind == 0 ? 16 : 8;
      while (it < opts->max_iter) {
        const int it0 = it, nbat = std::min(batch, opts->max_iter - it);
        for (int k = 0; k < nbat; ++k) {
          iteration();
          enqueue_snapshot(it0 + k + 1);
        }
        if ((rc = read_scalars())) return rc;
        const CgScal &S = *G.S_h;
        it = S.iter;
        if (S.status == 3) return fail(SOD_GPU_ENONFINITE, "non-finite residual in pressure solve");
        if (S.status == 0 && it == it0) return fail(SOD_GPU_ESTAGNATE, "pressure solve made no progress");
        // convergence history of this batch: stagnation check and next batch size
        double first = -1.0, lastv = -1.0;
        for (int k = it0; k < it; ++k) {
          const double rr = G.hist_h[k % CG_HIST];
          if (first < 0) first = rr;
          lastv = rr;
          const double nrm = std::sqrt(rr) / bnorm;
          if (nrm < best * 0.5) { best = nrm; best_it = k + 1; }
        }
        if (lastv >= 0) res = std::sqrt(lastv) / bnorm;
        if (S.status == 1) {
          if ((rc = certify())) return rc;
          if (res < opts->tol) converged = true;
          break;  // certified, or restart from the true residual
        }
        if (S.status == 2) {  // p.Ap <= 0 (loss of orthogonality): restart
          if (++breakdowns > 3) return fail(SOD_GPU_ESTAGNATE, "repeated breakdown in pressure solve");
          break;
        }
        if (kind != 0 && it - best_it > window) {  // stagnation: fall back to Jacobi
          kind = 0;
          fallback = 1;
          break;
        }
        if (it - it0 >= 2 && first > 0 && lastv > 0 && lastv < first) {
          const double rate = std::log(lastv / first) / (double)(it - it0 - 1);  // log rr per iteration
          const double need = std::log(S.thr2 / lastv) / rate;
          batch = (int)std::min(64.0, std::max(4.0, std::ceil(need) + 1.0));
        }
      }
    }
  }
  // harvested pairs: keep snapshots taken before convergence; e_k = x* - x_k
  for (auto &sn : snaps) {
    if (sn.iter >= it) {
      if (sn.fresh) { NT.count--; NT.offered--; }
      continue;
    }
    double *e = NT.tmp1;
    k_axpby<double><<<nb, 256, 0, st>>>(nw, c->lpoin_w, 1.0, x, 0.0, e);
    k_axpby<double><<<nb, 256, 0, st>>>(nw, c->lpoin_w, -1.0, NT.xsnap + (size_t)sn.si * N, 1.0, e);
    k_d2f_w<<<nb, 256, 0, st>>>(nw, c->lpoin_w, e, NT.he + (size_t)sn.slot * N);
    lap<double>(c, e, NT.tmp2);
    dots<double, 1>(c, DotArgs<double, 1>{{e}, {NT.tmp2}, {nullptr}}, G.dots + 5);
    double eAe = 0.0;
    CUDA_TRY(cudaMemcpyAsync(&eAe, G.dots + 5, 8, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    NT.eAe[sn.slot] = eAe > 0 ? eAe : 1.0;
  }
  CUDA_TRY(cudaEventRecord(e1, st));
  CUDA_TRY(cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (stats) {
    stats->iterations = it;
    stats->fallback = fallback;
    stats->res_rel = res;
    stats->seconds = ms * 1e-3;
  }
  if (!(res < opts->tol) && bnorm > 0) return fail(SOD_GPU_ESTAGNATE, "pressure solve did not reach the tolerance");
  return c->finish();
}

}  // extern "C"

// ---- incompressible BDF3/EXT3 step --------------------------------------

namespace {

// BDF (gamma0, alpha) and extrapolation (beta) coefficients of the local step
// iltime (1-based), time_integ_incomp.f90:165-229
struct BdfCoef {
  float g0, a[3], b[3];
};

BdfCoef bdf_coef(int iltime) {
  if (iltime == 1) return {1.f, {1.f, 0.f, 0.f}, {1.f, 0.f, 0.f}};
  if (iltime == 2) return {1.5f, {2.f, -0.5f, 0.f}, {2.f, -1.f, 0.f}};
  return {11.f / 6.f, {3.f, -1.5f, 1.f / 3.f}, {3.f, -3.f, 1.f}};
}

// u2 = -(b1 Rm2 + b2 Rm1 + b3 Rm3); u2 = (dt u2 / Ml + a1 u1 + a2 u3 + a3 u4) / g0
// over working nodes, time_integ_incomp.f90:322-341 (terms with a zero
// coefficient are skipped, so levels not yet filled are never read)
__global__ void k_bdf_ext(int npoin_w, long long npoin, const int *__restrict__ lpoin_w, const float *__restrict__ Ml,
                          const float *__restrict__ Rm2, const float *__restrict__ Rm1, const float *__restrict__ Rm3,
                          const float *__restrict__ u1, const float *__restrict__ u3, const float *__restrict__ u4,
                          BdfCoef k, float dt, float *__restrict__ u2) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const long long i = lpoin_w[t];
  const float ml = Ml[i];
  for (int d = 0; d < 3; ++d) {
    const long long j = i + npoin * d;
    float e = k.b[0] * Rm2[j];
    if (k.b[1] != 0.f) e = e + k.b[1] * Rm1[j];
    if (k.b[2] != 0.f) e = e + k.b[2] * Rm3[j];
    float v = dt * (-e) / ml + k.a[0] * u1[j];
    if (k.a[1] != 0.f) v = v + k.a[1] * u3[j];
    if (k.a[2] != 0.f) v = v + k.a[2] * u4[j];
    u2[j] = v / k.g0;
  }
}

// b = -g0 div / dt (time_integ_incomp.f90:351-353); x0 = the previous
// pressure (nhist 1, the reference's pr(:,1)), or 2 p - pold (nhist >= 2)
__global__ void k_poisson_rhs(int npoin_w, const int *__restrict__ lpoin_w, const float *__restrict__ div, float g0,
                              float dt, const double *__restrict__ p, const double *__restrict__ pold, int nhist,
                              double *__restrict__ b, double *__restrict__ x) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const int i = lpoin_w[t];
  b[i] = -(double)g0 * (double)div[i] / (double)dt;
  x[i] = nhist >= 2 ? 2.0 * p[i] - pold[i] : (nhist == 1 ? p[i] : 0.0);
}

// FP32 b = (-g0 div) / dt, the reference's pr(:,2) (time_integ_incomp.f90:351-353)
__global__ void k_poisson_rhs32(int npoin_w, const int *__restrict__ lpoin_w, const float *__restrict__ div, float g0,
                                float dt, float *__restrict__ b) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const int i = lpoin_w[t];
  b[i] = __fdiv_rn(__fmul_rn(-g0, div[i]), dt);
}

// u2 = (u2 - dt gradP / g0) Ml, time_integ_incomp.f90:390-394 (no wall model)
__global__ void k_veloc_rhs(int npoin_w, long long npoin, const int *__restrict__ lpoin_w,
                            const float *__restrict__ Ml, const float *__restrict__ gp, float dt, float g0,
                            float *__restrict__ u2) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const long long i = lpoin_w[t];
  const float ml = Ml[i];
  for (int d = 0; d < 3; ++d) {
    const long long j = i + npoin * d;
    u2[j] = (u2[j] - dt * gp[j] / g0) * ml;
  }
}

__global__ void k_fill(long long n, float v, float *__restrict__ a) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) a[t] = v;
}

}  // namespace

extern "C" {

}  // extern "C"

// ---- implicit velocity solve (conjGrad_veloc_incomp) ----------------------

namespace {

int ensure_velo(sod_gpu_ctx *c) {
  auto &V = c->velo;
  if (V.tauP) return 0;
  const size_t N = c->npoin;
  int rc;
  if ((rc = c->alloc(&V.tauP, N * 8)) || (rc = c->alloc(&V.tau_e, (size_t)c->nelem)) ||
      (rc = c->alloc(&V.x, 3 * N)) || (rc = c->alloc(&V.r, 3 * N)) || (rc = c->alloc(&V.p, 3 * N)) ||
      (rc = c->alloc(&V.q, 3 * N)) || (rc = c->alloc(&V.z, 3 * N)) || (rc = c->alloc(&V.z1, 3 * N)) ||
      (rc = c->alloc(&V.b, 3 * N)))
    return rc;
  if (!c->cg.part && ((rc = c->alloc(&c->cg.part, 8 * DOT_BLOCKS)) || (rc = c->alloc(&c->cg.dots, 16)))) return rc;
  for (float *v : {V.x, V.r, V.p, V.q, V.z, V.z1, V.b}) CUDA_TRY(cudaMemsetAsync(v, 0, 3 * N * 4, c->stream));
  return 0;
}

// LPS projection of v into V.tauP (node-major, mass-divided)
int velo_tau(sod_gpu_ctx *c, const float *v) {
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    k_tauv_elem<LL::P_, LL::EPB><<<LL::grid(c->nelem), LL::TPB, 0, c->stream>>>(c->md(), v, c->slotsB);
    return 0;
  });
  k_gather_tauv<<<nblk(c->npoin, 256), 256, 0, c->stream>>>(c->md(), c->slotsB, c->Ml, c->velo.tauP);
  // halo sum of the six projected components (mod_operators.f90:467-469)
  HaloView hv{};
  hv.width = 6;
  hv.nstride = 8;
  for (int k = 0; k < 6; ++k) hv.comp[k] = c->velo.tauP + k;
  return halo_sum(c, hv);
}

// out (npoin,3) = full_diff_stab_incomp(v) with the projection in V.tauP
void velo_diff(sod_gpu_ctx *c, const float *v, const float *mu_fluid, const float *musgs_t, const float *tau_e,
               float *out) {
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    k_diffv_elem<LL::P_, LL::EPB><<<LL::grid(c->nelem), LL::TPB, 0, c->stream>>>(c->md(), v, mu_fluid, musgs_t,
                                                                                c->velo.tauP, tau_e, c->slotsB);
    return 0;
  });
  OutPtrs o{};
  const long long N = c->npoin;
  o.p[0] = out; o.p[1] = out + N; o.p[2] = out + 2 * N;
  k_gather<4, 3, false><<<nblk(c->npoin, 256), 256, 0, c->stream>>>(c->md(), c->slotsB, nullptr, o, 0, 0);
}

// FP64 sums of the products of two (npoin,3) vectors (two pairs at once)
int velo_dots(sod_gpu_ctx *c, const float *a0, const float *b0, const float *c0, const float *a1, const float *b1,
              double *h) {
  const long long N = c->npoin;
  DotArgs<float, 6> A{};
  for (int d = 0; d < 3; ++d) {
    A.a[d] = a0 + N * d; A.b[d] = b0 + N * d; A.c[d] = c0 ? c0 + N * d : nullptr;
    A.a[3 + d] = a1 ? a1 + N * d : a0 + N * d; A.b[3 + d] = b1 ? b1 + N * d : b0 + N * d; A.c[3 + d] = nullptr;
  }
  dots<float, 6>(c, A, c->cg.dots + 8);
  int rc = allreduce(c, c->cg.dots + 8, 6, SOD_REDUCE_SUM_F64);  // mod_solver_incomp.f90:128-229
  if (rc) return rc;
  double t[6];
  CUDA_TRY(cudaMemcpyAsync(t, c->cg.dots + 8, 48, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  h[0] = (t[0] + t[1]) + t[2];
  h[1] = (t[3] + t[4]) + t[5];
  return 0;
}

}  // namespace

extern "C" {

int sod_gpu_species_tau(sod_gpu_ctx *c, const float *u, float *tau) {
  if (!c || !u || !tau) return fail(SOD_GPU_EINVAL, "bad argument");
  if (!c->helem) return fail(SOD_GPU_EINVAL, "species_tau needs helem at init");
  k_species_tau<<<nblk(c->nelem, 8), 256, 0, c->stream>>>(c->nelem, c->N, c->conn, c->helem, u, c->npoin,
                                                          c->phys.c_species_stab / (float)c->P, tau);
  return c->finish();
}

int sod_gpu_eval_tau_veloc(sod_gpu_ctx *c, const float *u, float *GradX, float *GradY, float *GradZ) {
  if (!c || !u || !GradX || !GradY || !GradZ) return fail(SOD_GPU_EINVAL, "bad argument");
  int rc;
  if ((rc = ensure_velo(c))) return rc;
  if ((rc = velo_tau(c, u))) return rc;
  k_unpack_tauv<<<nblk(c->npoin, 256), 256, 0, c->stream>>>(c->npoin, c->velo.tauP, GradX, GradY, GradZ);
  return c->finish();
}

int sod_gpu_full_diff_stab_incomp(sod_gpu_ctx *c, const float *u, const float *mu_fluid, const float *mu_sgs,
                                  const float *TauPX, const float *TauPY, const float *TauPZ, const float *tau_stab,
                                  float *Rmom) {
  if (!c || !u || !mu_fluid || !TauPX || !TauPY || !TauPZ || !tau_stab || !Rmom)
    return fail(SOD_GPU_EINVAL, "bad argument");
  int rc;
  if ((rc = ensure_velo(c))) return rc;
  const long long EN = (long long)c->nelem * c->N;
  if (mu_sgs) {
    if (!c->musgs_t && (rc = c->alloc(&c->musgs_t, (size_t)EN))) return rc;
    k_elem_to_t<<<nblk(c->nelem, E2T_TILE), E2T_THREADS, 0, c->stream>>>(c->nelem, c->N, c->a_of_t, mu_sgs, c->musgs_t);
  }
  k_pack_tauv<<<nblk(c->npoin, 256), 256, 0, c->stream>>>(c->npoin, TauPX, TauPY, TauPZ, c->velo.tauP);
  velo_diff(c, u, mu_fluid, mu_sgs ? c->musgs_t : nullptr, tau_stab, Rmom);
  return c->finish();
}

int sod_gpu_conjgrad_veloc(sod_gpu_ctx *c, float fact, float dt, const float *mu_fluid, const float *mu_sgs,
                           const float *Rp0, float *R, int maxIter, double tol, int *iters, double *res_rel) {
  if (!c || !mu_fluid || !Rp0 || !R || maxIter < 1 || !(dt > 0.f)) return fail(SOD_GPU_EINVAL, "bad argument");
  if (!c->helem) return fail(SOD_GPU_EINVAL, "conjgrad_veloc needs helem at init");
  int rc;
  if ((rc = ensure_velo(c))) return rc;
  auto &V = c->velo;
  const long long N = c->npoin, EN = (long long)c->nelem * c->N;
  const int nw = c->npoin_w;
  const unsigned nb = nblk(nw, 256);
  const bool was_async = c->async;
  c->async = true;
  const float *musgs = nullptr;
  if (mu_sgs) {
    if (!c->musgs_t && (rc = c->alloc(&c->musgs_t, (size_t)EN))) return rc;
    k_elem_to_t<<<nblk(c->nelem, E2T_TILE), E2T_THREADS, 0, c->stream>>>(c->nelem, c->N, c->a_of_t, mu_sgs, c->musgs_t);
    musgs = c->musgs_t;
  }
  CUDA_TRY(cudaMemcpyAsync(V.x, Rp0, 3 * N * 4, cudaMemcpyDeviceToDevice, c->stream));
  CUDA_TRY(cudaMemcpyAsync(V.b, R, 3 * N * 4, cudaMemcpyDeviceToDevice, c->stream));
  k_species_tau<<<nblk(c->nelem, 8), 256, 0, c->stream>>>(c->nelem, c->N, c->conn, c->helem, V.x, N,
                                                          c->phys.c_species_stab / (float)c->P, V.tau_e);
  auto apply = [&](const float *v) {  // q = v Ml + fact dt D(v)
    int arc = velo_tau(c, v);
    if (arc) return arc;
    velo_diff(c, v, mu_fluid, musgs, V.tau_e, V.q);
    // halo sum of the operator (mod_solver_incomp.f90:94, :146)
    if ((arc = halo_sum(c, halo_soa_view(c, V.q, 3)))) return arc;
    k_veloc_op<<<nb, 256, 0, c->stream>>>(nw, N, c->lpoin_w, c->Ml, v, fact, dt, V.q);
    return 0;
  };
  if ((rc = apply(V.x))) { c->async = was_async; return rc; }
  k_veloc_vec<<<nb, 256, 0, c->stream>>>(0, nw, N, c->lpoin_w, c->Ml, dt, 0.f, 0.f, V.b, V.x, V.r, V.p, V.q, V.z,
                                         V.z1);
  double h[2];
  if ((rc = velo_dots(c, V.r, V.r, nullptr, nullptr, nullptr, h))) { c->async = was_async; return rc; }
  const double auxB = std::sqrt(h[0]);
  double nrm = auxB;
  int it;
  for (it = 1; it <= maxIter; ++it) {
    if ((rc = apply(V.p))) { c->async = was_async; return rc; }
    if ((rc = velo_dots(c, V.r, V.z, nullptr, V.p, V.q, h))) { c->async = was_async; return rc; }
    const double Q1 = h[0];
    const float alpha = (float)(h[0] / h[1]);
    k_veloc_vec<<<nb, 256, 0, c->stream>>>(1, nw, N, c->lpoin_w, c->Ml, dt, alpha, 0.f, V.b, V.x, V.r, V.p, V.q,
                                           V.z, V.z1);
    if ((rc = velo_dots(c, V.r, V.r, nullptr, V.r, V.z, h))) { c->async = was_async; return rc; }
    nrm = std::sqrt(h[0]);
    if (!std::isfinite(nrm)) { c->async = was_async; return fail(SOD_GPU_ENONFINITE, "non-finite residual in velocity CG"); }
    if (nrm < tol * auxB) break;
    // Polak-Ribiere: r.(z - z1)
    if ((rc = velo_dots(c, V.r, V.z, V.z1, V.r, V.z, h))) { c->async = was_async; return rc; }
    const float beta = (float)(h[0] / Q1);
    k_veloc_vec<<<nb, 256, 0, c->stream>>>(2, nw, N, c->lpoin_w, c->Ml, dt, 0.f, beta, V.b, V.x, V.r, V.p, V.q, V.z,
                                           V.z1);
  }
  CUDA_TRY(cudaMemcpyAsync(R, V.x, 3 * N * 4, cudaMemcpyDeviceToDevice, c->stream));
  c->async = was_async;
  if (iters) *iters = it > maxIter ? maxIter : it;
  if (res_rel) *res_rel = auxB > 0 ? nrm / auxB : 0.0;
  return c->finish();
}

int sod_gpu_incomp_init(sod_gpu_ctx *c, const float *u, double nu) {
  if (!c || !u || nu < 0) return fail(SOD_GPU_EINVAL, "bad argument");
  if (!c->helem) return fail(SOD_GPU_EINVAL, "the incompressible step needs helem at init");
  auto &I = c->inc;
  const size_t N = c->npoin;
  int rc;
  if (!I.ready) {
    for (auto &a : I.u)
      if ((rc = c->alloc(&a, 3 * N))) return rc;
    for (auto &a : I.Rm)
      if ((rc = c->alloc(&a, 3 * N))) return rc;
    if ((rc = c->alloc(&I.div, N)) || (rc = c->alloc(&I.grad, 3 * N)) || (rc = c->alloc(&I.pf, N)) ||
        (rc = c->alloc(&I.mu, N)) || (rc = c->alloc(&I.p, N)) || (rc = c->alloc(&I.pold, N)) ||
        (rc = c->alloc(&I.b, N)) || (rc = c->alloc(&I.x, N)) || (rc = c->alloc(&I.rhs32, N)) ||
        (rc = c->alloc(&I.one, N)) || (rc = c->alloc(&I.zero, N)) ||
        (rc = c->alloc(&I.zeroE, (size_t)c->nelem * c->N)) || (rc = c->alloc(&I.part, 3 * (size_t)c->nelem)) ||
        (rc = c->alloc(&I.sums, 4)) || (rc = c->alloc(&I.bits, 4)))
      return rc;
    k_fill<<<nblk((long long)N, 256), 256, 0, c->stream>>>((long long)N, 1.0f, I.one);
    CUDA_TRY(cudaMemsetAsync(I.zero, 0, N * 4, c->stream));
    CUDA_TRY(cudaMemsetAsync(I.zeroE, 0, (size_t)c->nelem * c->N * 4, c->stream));
    CUDA_TRY(cudaMemsetAsync(I.rhs32, 0, N * 4, c->stream));
    I.ready = true;
  }
  // every level starts from the initial field (CFDSolverPeriodicIncomp.f90:54-66)
  for (auto &a : I.u) CUDA_TRY(cudaMemcpyAsync(a, u, 3 * N * 4, cudaMemcpyDeviceToDevice, c->stream));
  for (auto &a : I.Rm) CUDA_TRY(cudaMemsetAsync(a, 0, 3 * N * 4, c->stream));
  CUDA_TRY(cudaMemsetAsync(I.grad, 0, 3 * N * 4, c->stream));
  for (double *z : {I.p, I.pold, I.b, I.x}) CUDA_TRY(cudaMemsetAsync(z, 0, N * 8, c->stream));
  CUDA_TRY(cudaMemsetAsync(I.div, 0, N * 4, c->stream));
  CUDA_TRY(cudaMemsetAsync(I.pf, 0, N * 4, c->stream));
  k_fill<<<nblk((long long)N, 256), 256, 0, c->stream>>>((long long)N, (float)nu, I.mu);  // constant mu_fluid (rho = 1)
  I.nu = nu;
  I.nsteps = 0;
  return c->finish();
}

int sod_gpu_incomp_set_veloc_solver(sod_gpu_ctx *c, int maxIter, double tol) {
  if (!c || maxIter < 1 || !(tol > 0.0)) return fail(SOD_GPU_EINVAL, "bad argument");
  c->inc.v_maxiter = maxIter;
  c->inc.v_tol = tol;
  return 0;
}

int sod_gpu_incomp_veloc_stats(sod_gpu_ctx *c, int *iters, double *res_rel) {
  if (!c || !c->inc.ready) return fail(SOD_GPU_EINVAL, "state not initialised");
  if (iters) *iters = c->inc.v_iters;
  if (res_rel) *res_rel = c->inc.v_res;
  return 0;
}

int sod_gpu_incomp_step(sod_gpu_ctx *c, float dt, const sod_solve_opts_t *opts, sod_solve_stats_t *stats) {
  if (!c || !c->inc.ready || !opts || !(dt > 0.f)) return fail(SOD_GPU_EINVAL, "bad argument");
  if (opts->precond < 0 || opts->precond > 3) return fail(SOD_GPU_EINVAL, "precond must be 0, 1, 2 or 3");
  // a partitioned mesh runs the reference's FP32 solve (precond 2) or the
  // FP64-certified Jacobi solve (precond 0 or 3)
  if (opts->precond == 1)
    if (int prc = no_partition(c, "sod_gpu_incomp_step with the learned preconditioner")) return prc;
  auto &I = c->inc;
  const long long N = c->npoin;
  const int nw = c->npoin_w;
  const unsigned nb = nblk(nw, 256);
  const BdfCoef k = bdf_coef(I.nsteps + 1);
  float *const u1 = I.u[0], *const u2 = I.u[1], *const u3 = I.u[2], *const u4 = I.u[3];
  const bool was_async = c->async;
  c->async = true;  // chain the operator calls; synchronise at the end
  // Rmom(:,:,2) = full_convec_ijk_incomp(u1, u1 rho, rho), rho = 1
  int rc = sod_gpu_full_convec_ijk_incomp(c, u1, u1, I.Rm[1]);
  if (!rc) rc = halo_sum(c, halo_soa_view(c, I.Rm[1], 3));  // time_integ_incomp.f90:315
  if (rc) { c->async = was_async; return rc; }
  k_bdf_ext<<<nb, 256, 0, c->stream>>>(nw, N, c->lpoin_w, c->Ml, I.Rm[1], I.Rm[0], I.Rm[2], u1, u3, u4, k, dt, u2);
  {  // Rmom(:,:,3) = Rmom(:,:,1); Rmom(:,:,1) = Rmom(:,:,2)
    float *t = I.Rm[2];
    I.Rm[2] = I.Rm[0]; I.Rm[0] = I.Rm[1]; I.Rm[1] = t;
  }
  rc = sod_gpu_eval_divergence(c, u2, I.div);
  if (rc) { c->async = was_async; return rc; }
  int solve_rc = 0;
  if (opts->precond == 2) {
    // the reference's solve: conjGrad_pressure_incomp in FP32 from the
    // previous pressure pr(:,1), max_iter / tol, no certification
    k_poisson_rhs32<<<nb, 256, 0, c->stream>>>(nw, c->lpoin_w, I.div, k.g0, dt, I.rhs32);
    c->async = was_async;
    int pit = 0;
    double pres = 0.0;
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    CUDA_TRY(cudaEventRecord(e0, c->stream));
    rc = sod_gpu_conjgrad_pressure(c, I.pf, I.rhs32, opts->max_iter, opts->tol, &pit, &pres);
    CUDA_TRY(cudaEventRecord(e1, c->stream));
    CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if (stats) { stats->iterations = pit; stats->fallback = 0; stats->res_rel = pres; stats->seconds = ms * 1e-3; }
    c->async = true;
    {  // pold = p; p = (double) solution; pf = solution
      double *t = I.pold;
      I.pold = I.p; I.p = I.x; I.x = t;
    }
    k_f2d_w<<<nb, 256, 0, c->stream>>>(nw, c->lpoin_w, I.rhs32, I.p);
    CUDA_TRY(cudaMemcpyAsync(I.pf, I.rhs32, N * 4, cudaMemcpyDeviceToDevice, c->stream));
  } else {
    // initial guess: the previous pressure for Jacobi (the reference's
    // pr(:,1), mod_solver_incomp.f90:306); extrapolated from the previous
    // two pressures for the learned path and for precond 3 (Jacobi with the
    // learned path's guess)
    const bool extrap = opts->precond == 1 || opts->precond == 3;
    const int hist = extrap ? I.nsteps : (I.nsteps > 0 ? 1 : 0);
    k_poisson_rhs<<<nb, 256, 0, c->stream>>>(nw, c->lpoin_w, I.div, k.g0, dt, I.p, I.pold, hist, I.b, I.x);
    c->async = was_async;
    sod_solve_opts_t o = *opts;
    if (o.precond == 3) o.precond = 0;
    rc = sod_gpu_pressure_solve(c, I.b, I.x, &o, stats);
    if (rc && rc != SOD_GPU_ESTAGNATE) return rc;
    solve_rc = rc;
    {  // pold = p; p = x
      double *t = I.pold;
      I.pold = I.p; I.p = I.x; I.x = t;
    }
    c->async = true;
    k_d2f_w<<<nb, 256, 0, c->stream>>>(nw, c->lpoin_w, I.p, I.pf);
  }
  rc = sod_gpu_eval_gradient(c, I.pf, I.grad);
  if (rc) { c->async = was_async; return rc; }
  k_veloc_rhs<<<nb, 256, 0, c->stream>>>(nw, N, c->lpoin_w, c->Ml, I.grad, dt, k.g0, u2);
  c->async = was_async;
  int vit = 0;
  double vres = 0.0;
  rc = sod_gpu_conjgrad_veloc(c, 1.f / k.g0, dt, I.mu, nullptr, u1, u2, I.v_maxiter, I.v_tol, &vit, &vres);
  if (rc) return rc;
  I.v_iters = vit;
  I.v_res = vres;
  // u(:,:,4) = u(:,:,3); u(:,:,3) = u(:,:,1); u(:,:,1) = u(:,:,2) (CFDSolverBase.f90:1953-2015)
  I.u[0] = u2; I.u[1] = u4; I.u[2] = u1; I.u[3] = u3;
  I.nsteps++;
  rc = c->finish();
  return rc ? rc : solve_rc;
}

int sod_gpu_incomp_set_pressure(sod_gpu_ctx *c, const double *p) {
  if (!c || !c->inc.ready || !p) return fail(SOD_GPU_EINVAL, "bad argument");
  auto &I = c->inc;
  const size_t N = c->npoin;
  CUDA_TRY(cudaMemcpyAsync(I.p, p, N * 8, cudaMemcpyDeviceToDevice, c->stream));
  CUDA_TRY(cudaMemcpyAsync(I.pold, p, N * 8, cudaMemcpyDeviceToDevice, c->stream));
  k_d2f_w<<<nblk(c->npoin_w, 256), 256, 0, c->stream>>>(c->npoin_w, c->lpoin_w, I.p, I.pf);
  return c->finish();
}

int sod_gpu_incomp_adapt_dt(sod_gpu_ctx *c, float cfl_conv, float *dt) {
  if (!c || !c->inc.ready || !dt || !(cfl_conv > 0.f)) return fail(SOD_GPU_EINVAL, "bad argument");
  auto &I = c->inc;
  const unsigned init_bits = 0x56B5E621u;  // 1e14f, the reference's initial dt_conv
  CUDA_TRY(cudaMemcpyAsync(I.bits, &init_bits, 4, cudaMemcpyHostToDevice, c->stream));
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    // zero sound speed and viscosities: only the convective limit acts
    k_dt<LL::P_><<<nblk(c->nelem, 8), 256, 0, c->stream>>>(c->md(), c->helem, I.u[0], I.zero, I.zero, I.zeroE,
                                                            I.one, cfl_conv, 1.0f, I.bits);
    return 0;
  });
  if (int rrc = allreduce(c, I.bits, 1, SOD_REDUCE_MIN_F32)) return rrc;  // mod_time_ops.f90:212
  unsigned b = 0;
  CUDA_TRY(cudaMemcpyAsync(&b, I.bits, 4, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  std::memcpy(dt, &b, 4);
  return 0;
}

int sod_gpu_incomp_analysis(sod_gpu_ctx *c, double *out) {
  if (!c || !c->inc.ready || !out) return fail(SOD_GPU_EINVAL, "bad argument");
  auto &I = c->inc;
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    k_analysis_elem<LL::P_, LL::EPB><<<LL::grid(c->nelem), LL::TPB, 0, c->stream>>>(c->md(), I.one, I.u[0], I.mu,
                                                                                   I.zeroE, c->Ngp_t, I.part);
    return 0;
  });
  k_sum_parts<<<1, 1024, 0, c->stream>>>(c->nelem, I.part, I.sums);
  if (int rrc = allreduce(c, I.sums, 3, SOD_REDUCE_SUM_F64)) return rrc;  // mod_analysis.f90:39, 134-135
  double sums[3];
  CUDA_TRY(cudaMemcpyAsync(sums, I.sums, 24, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  const float rho0 = 1.0f, twopi = 2.0f * 3.14159f;
  const double EK = sums[0] / (double)(rho0 * powf(twopi, 3.0f));
  const float alpha = 1.0f / (rho0 * c->volT);
  const double eS = sums[1] * (double)alpha, eD = (double)(4.0f / 3.0f) * sums[2] * (double)alpha;
  out[0] = (double)(float)EK;
  out[1] = (double)(float)eS;
  out[2] = (double)(float)eD;
  out[3] = (double)(float)(eS + eD);
  return 0;
}

int sod_gpu_incomp_get(sod_gpu_ctx *c, float *u, double *p) {
  if (!c || !c->inc.ready) return fail(SOD_GPU_EINVAL, "state not initialised");
  if (u) CUDA_TRY(cudaMemcpyAsync(u, c->inc.u[0], (size_t)c->npoin * 12, cudaMemcpyDeviceToDevice, c->stream));
  if (p) CUDA_TRY(cudaMemcpyAsync(p, c->inc.p, (size_t)c->npoin * 8, cudaMemcpyDeviceToDevice, c->stream));
  return c->finish();
}

}  // extern "C"
