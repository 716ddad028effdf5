// Internal header: vector kernels, the Laplacian assembly and dot-product
// helpers and the CG workspaces shared by the incompressible solves
// (incomp.cu) and the training of the learned preconditioner (precond.cu).
#pragma once
#include "ctx.cuh"

// The learned preconditioner's application (precond.cu), used by the
// pressure solve.
namespace sod_net {
int ensure_gains(sod_gpu_ctx *c);
int apply_precond(sod_gpu_ctx *c, int kind, const double *r, double *z);
}  // namespace sod_net
using sod_net::apply_precond;
using sod_net::ensure_gains;

namespace {

// x += a p ; r -= a q ; z1 = z0 ; z0 = r * Minv   (a = dots[0]/dots[1])
template <class V>
__global__ void k_cg_update1(int npoin_w, const int *__restrict__ lpoin_w, const double *__restrict__ dots,
                             V *__restrict__ x, V *__restrict__ r, const V *__restrict__ p, const V *__restrict__ q,
                             V *__restrict__ z0, V *__restrict__ z1, const V *__restrict__ M, int divide, int jacobi) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const int i = lpoin_w[t];
  const V a = (V)(dots[0] / dots[1]);
  x[i] = x[i] + a * p[i];
  const V rn = r[i] - a * q[i];
  r[i] = rn;
  if (jacobi) {
    z1[i] = z0[i];
    z0[i] = divide ? rn / M[i] : rn * M[i];
  }
}

// p = z0 + b p   (b = dots2[1] / dots1[0])
template <class V>
__global__ void k_cg_update2(int npoin_w, const int *__restrict__ lpoin_w, const double *__restrict__ dots1,
                             const double *__restrict__ dots2, V *__restrict__ p, const V *__restrict__ z0) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const int i = lpoin_w[t];
  const V b = (V)(dots2[1] / dots1[0]);
  p[i] = z0[i] + b * p[i];
}

// generic y = a*x + b*y over working nodes (a, b host scalars)
template <class V>
__global__ void k_axpby(int npoin_w, const int *__restrict__ lpoin_w, V a, const V *__restrict__ x, V b,
                        V *__restrict__ y) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const int i = lpoin_w[t];
  y[i] = a * x[i] + b * y[i];
}

template <class V>
__global__ void k_add_all(long long n, const V *__restrict__ a, const V *__restrict__ b, V *__restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i] + b[i];
}

template <class V>
inline void lap(sod_gpu_ctx *c, const V *p, V *out) {
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    k_lap_elem<LL::P_, LL::EPB, V><<<LL::grid(c->nelem), LL::TPB, 0, c->stream>>>(c->md(), p, (V *)c->slotsB);
    return 0;
  });
  k_gather1<V><<<nblk(c->npoin, 256), 256, 0, c->stream>>>(c->md(), (const V *)c->slotsB, out, 0);
}

// Dot products over the working nodes, or over the owned ones on a
// partitioned mesh (each shared node counted once over the ranks).
template <class V, int ND>
inline void dots(sod_gpu_ctx *c, DotArgs<V, ND> A, double *out) {
  const bool part = c->halo.on;
  k_dot<V, ND><<<DOT_BLOCKS, DOT_THREADS, 0, c->stream>>>(part ? c->halo.npoin_o : c->npoin_w,
                                                          part ? c->halo.lpoin_o : c->lpoin_w, A, c->cg.part,
                                                          c->cg.dticket, out);
}

inline int ensure_diag(sod_gpu_ctx *c) {
  auto &G = c->cg;
  if (G.have_diag) return 0;
  int rc;
  if (!G.diag && (rc = c->alloc(&G.diag, (size_t)c->npoin))) return rc;
  if (!G.part && ((rc = c->alloc(&G.part, 8 * DOT_BLOCKS)) || (rc = c->alloc(&G.dots, 16)))) return rc;
  const long long EN = (long long)c->nelem * c->N;
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    k_lap_diag_elem<LL::P_><<<nblk(EN, 256), 256, 0, c->stream>>>(c->md(), c->slotsB);
    return 0;
  });
  k_gather1<float><<<nblk(c->npoin, 256), 256, 0, c->stream>>>(c->md(), c->slotsB, G.diag, 0);
  if ((rc = halo_sum(c, halo_soa_view(c, G.diag, 1)))) return rc;  // mod_operators.f90:677
  G.have_diag = true;
  return 0;
}

inline int ensure_cg32(sod_gpu_ctx *c) {
  auto &G = c->cg;
  if (G.ready32) return 0;
  int rc;
  for (float **pp : {&G.x32, &G.r32, &G.p32, &G.q32, &G.z032, &G.z132, &G.b32})
    if ((rc = c->alloc(pp, (size_t)c->npoin))) return rc;
  G.ready32 = true;
  return 0;
}

inline int ensure_cg64(sod_gpu_ctx *c) {
  auto &G = c->cg;
  if (G.ready64) return 0;
  int rc;
  for (double **pp : {&G.x, &G.r, &G.p, &G.q, &G.z0, &G.z1, &G.b, &G.Minv})
    if ((rc = c->alloc(pp, (size_t)c->npoin))) return rc;
  G.ready64 = true;
  return 0;
}

constexpr int CG_HIST = 1024;


// grid of the tensor-core patch kernel: one block per SM (the block's
// registers and shared memory allow one), fewer when there are fewer
// 16-element groups than SMs
template <int P>
inline unsigned tc_grid(long long nelem) {
  const long long groups = (nelem + 15) / 16;
  return (unsigned)std::min<long long>(std::max<long long>(groups, 1), num_sms());
}
constexpr int TC_THREADS = TcDims<3>::WARPS * 32;
static_assert(TcDims<3>::WARPS == TcDims<4>::WARPS, "one block size for both orders");

inline int ensure_cg_loop(sod_gpu_ctx *c) {
  auto &G = c->cg;
  if (G.S) return 0;
  int rc;
  if ((rc = c->alloc(&G.S, 1)) || (rc = c->alloc(&G.hist, CG_HIST)) || (rc = c->alloc(&G.ticket, 1)) ||
      (rc = c->alloc(&G.gpart, (size_t)3 * cg_blocks(c->npoin, 2))))
    return rc;
  CUDA_TRY(cudaMemset(G.ticket, 0, sizeof(unsigned)));
  CUDA_TRY(cudaMemset(G.S, 0, sizeof(CgScal)));
  void *h1 = nullptr, *h2 = nullptr;
  CUDA_TRY(cudaMallocHost(&h1, sizeof(CgScal)));
  CUDA_TRY(cudaMallocHost(&h2, sizeof(double) * CG_HIST));
  G.S_h = (CgScal *)h1;
  G.hist_h = (double *)h2;
  c->host_allocs.push_back(h1);
  c->host_allocs.push_back(h2);
  return 0;
}

// start (or restart) of the device-resident CG: d = [r.z, r.r]
__global__ void k_cg_start(CgScal *S, const double *__restrict__ d, double thr2, int iter) {
  S->rz = d[0];
  S->rr = d[1];
  S->thr2 = thr2;
  S->iter = iter;
  S->alpha = S->beta = 0.0;
  S->status = !isfinite(d[1]) ? 3 : (d[1] < thr2 ? 1 : 0);
}

__global__ void k_inv_diag64(long long n, const float *__restrict__ d, double *__restrict__ minv) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) minv[i] = d[i] != 0.f ? 1.0 / (double)d[i] : 0.0;
}

template <class T>
__global__ void k_copy_cast(long long n, const T *__restrict__ a, double *__restrict__ b) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (double)a[i];
}

// z = Minv r over working nodes
__global__ void k_jacobi64(int npoin_w, const int *__restrict__ lpoin_w, const double *__restrict__ Minv,
                           const double *__restrict__ r, double *__restrict__ z) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const int i = lpoin_w[t];
  z[i] = r[i] * Minv[i];
}

// FP32 <-> FP64 copies over working nodes
__global__ void k_f2d_w(int npoin_w, const int *__restrict__ lpoin_w, const float *__restrict__ a,
                        double *__restrict__ b) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const int i = lpoin_w[t];
  b[i] = (double)a[i];
}

__global__ void k_d2f_w(int npoin_w, const int *__restrict__ lpoin_w, const double *__restrict__ a,
                        float *__restrict__ b) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const int i = lpoin_w[t];
  b[i] = (float)a[i];
}

}  // namespace
