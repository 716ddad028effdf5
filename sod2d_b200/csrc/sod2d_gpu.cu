// C-ABI entry points of the B200 spectral-element RHS library
// (declarations and contracts: include/sod2d_gpu.h).
#include "sod2d_gpu.h"
#include "rhs_kernels.cuh"

#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace sod;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

#define CUDA_TRY(call)                                                                    \
  do {                                                                                    \
    cudaError_t _e = (call);                                                              \
    if (_e != cudaSuccess)                                                                \
      return fail(SOD_GPU_ECUDA, std::string(#call) + ": " + cudaGetErrorString(_e));     \
  } while (0)

inline int nat_of(int porder, int ii) { return ii == 0 ? 0 : (ii == 1 ? porder : ii - 1); }

}  // namespace

struct sod_gpu_ctx {
  int P = 0, N1 = 0, N = 0, nelem = 0, npoin = 0, npoin_w = 0;
  cudaStream_t stream = 0;
  bool async = false;
  bool mue_set = false;
  Phys ph{};
  sod_phys_t phys{};
  // device mirrors
  int *conn = nullptr, *lpoin_w = nullptr, *slot_ptr = nullptr, *slot_idx = nullptr, *lelpn = nullptr;
  int *a_of_t = nullptr;  // tensor position -> reference local node (0-based)
  float *geo = nullptr, *Dnat = nullptr, *invMl = nullptr, *Ml = nullptr, *helem = nullptr, *helem_l_t = nullptr;
  // scratch
  float *slotsA = nullptr, *slotsB = nullptr, *proj16 = nullptr, *mue_t = nullptr, *musgs_t = nullptr;
  size_t bytes = 0;
  std::vector<void *> allocs;

  MeshDev md() const {
    MeshDev m;
    m.nelem = nelem; m.npoin = npoin; m.npoin_w = npoin_w;
    m.conn = conn; m.geo = geo; m.Dnat = Dnat; m.lpoin_w = lpoin_w; m.invMl = invMl;
    m.slot_ptr = slot_ptr; m.slot_idx = slot_idx;
    return m;
  }
  template <class T>
  int alloc(T **p, size_t count) {
    size_t b = count * sizeof(T);
    if (b == 0) b = 16;
    cudaError_t e = cudaMalloc((void **)p, b);
    if (e != cudaSuccess) return fail(SOD_GPU_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    allocs.push_back(*p);
    bytes += b;
    return 0;
  }
  template <class T>
  int upload(T **p, const T *host, size_t count) {
    int rc = alloc(p, count);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpy(*p, host, count * sizeof(T), cudaMemcpyHostToDevice));
    return 0;
  }
  int finish() {
    CUDA_TRY(cudaGetLastError());
    if (!async) CUDA_TRY(cudaStreamSynchronize(stream));
    return 0;
  }
};

namespace {

// ---- small node / element kernels ---------------------------------------

__global__ void k_lumped(int npoin_w, long long npoin, const int *__restrict__ lpoin_w,
                         const float *__restrict__ invMl, float *__restrict__ R, int ncomp) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  int p = lpoin_w[t];
  float a = invMl[p];
  for (int c = 0; c < ncomp; ++c) R[p + npoin * c] = R[p + npoin * c] * a;
}

// Reference-layout field (nelem, nnode) -> internal [e][t].
__global__ void k_elem_to_t(long long nelem, int N, const int *__restrict__ a_of_t,
                            const float *__restrict__ src, float *__restrict__ dst) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nelem * N) return;
  long long e = idx / N;
  int t = (int)(idx % N);
  dst[idx] = src[e + nelem * a_of_t[t]];
}

// Five Proj arrays (npoin,3) -> node-major [p][16].
__global__ void k_pack_proj(long long npoin, const float *PMX, const float *PMY, const float *PMZ,
                            const float *PMass, const float *PEner, float *proj16) {
  long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npoin) return;
  const float *src[5] = {PMX, PMY, PMZ, PMass, PEner};
  float r[16];
  for (int f = 0; f < 5; ++f)
    for (int d = 0; d < 3; ++d) r[f * 3 + d] = src[f][p + npoin * d];
  r[15] = 0.f;
  float4 *o = reinterpret_cast<float4 *>(proj16 + p * 16);
  for (int c = 0; c < 4; ++c) o[c] = make_float4(r[4 * c], r[4 * c + 1], r[4 * c + 2], r[4 * c + 3]);
}

// Primitive outputs of updateF at working nodes (time_integ_ls.f90:574-587).
__global__ void k_eos_out(int npoin_w, long long npoin, const int *__restrict__ lpoin_w, Phys ph, float Rgas,
                          float mu_factor, const float *rho, const float *q, const float *E, float *u,
                          float *pr, float *Tem, float *mu) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  long long p = lpoin_w[t];
  NodeQ s;
  eos(ph, Rgas, mu_factor, rho[p], q[p], q[p + npoin], q[p + 2 * npoin], E[p], s);
  if (u) { u[p] = s.u0; u[p + npoin] = s.u1; u[p + 2 * npoin] = s.u2; }
  if (pr) pr[p] = s.p;
  if (Tem) Tem[p] = s.T;
  if (mu) mu[p] = s.mu;
}

// comp_tau, elem_stab.f90:589-616: one warp per element, max over nodes.
__global__ void k_comp_tau(long long nelem, int N, const int *__restrict__ conn, const float *__restrict__ helem,
                           const float *__restrict__ csound, const float *__restrict__ u, long long npoin,
                           float c_over_p, float *__restrict__ tau) {
  long long e = (long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  int lane = threadIdx.x % 32;
  if (e >= nelem) return;
  float taul = 0.f;
  const float he = helem[e];
  for (int t = lane; t < N; t += 32) {
    int p = conn[e * N + t];
    float u0 = u[p], u1 = u[p + npoin], u2 = u[p + 2 * npoin];
    float aux1 = 1.0f * csound[p] + sqrtf(u0 * u0 + u1 * u1 + u2 * u2);
    taul = fmaxf(taul, he * c_over_p * aux1);
  }
  for (int o = 16; o > 0; o >>= 1) taul = fmaxf(taul, __shfl_xor_sync(0xffffffffu, taul, o));
  if (lane == 0) tau[e] = taul;
}

inline unsigned nblk(long long n, int b) { return (unsigned)((n + b - 1) / b); }

// ---- launch helpers templated on the element order --------------------

template <int P>
struct Launch {
  static constexpr int EPB = (Cfg<P>::NT <= 64) ? 2 : 1;
  static constexpr int TPB = EPB * Cfg<P>::NT;
  static unsigned grid(int nelem) { return nblk(nelem, EPB); }

  static void proj(sod_gpu_ctx *c, bool prim, const float *a0, const float *a1, const float *a2) {
    if (prim)
      k_proj<P, EPB, true><<<grid(c->nelem), TPB, 0, c->stream>>>(c->md(), c->ph, c->phys.Rgas, a0, a1, a2, c->slotsA);
    else
      k_proj<P, EPB, false><<<grid(c->nelem), TPB, 0, c->stream>>>(c->md(), c->ph, c->phys.Rgas, a0, a1, a2, c->slotsA);
  }
  template <int MODE, int IN>
  static void rhs(sod_gpu_ctx *c, const RhsArgs &A) {
    k_rhs<P, EPB, MODE, IN><<<grid(c->nelem), TPB, 0, c->stream>>>(c->md(), c->ph, c->phys.Rgas, A, c->slotsB);
  }
};

template <class F>
int dispatch(sod_gpu_ctx *c, F &&f) {
  if (c->P == 3) return f(Launch<3>());
  if (c->P == 4) return f(Launch<4>());
  return fail(SOD_GPU_EINVAL, "unsupported element order");
}

void gather_proj_aos(sod_gpu_ctx *c) {
  OutPtrs none{};
  k_gather<16, 15, true><<<nblk(c->npoin, 256), 256, 0, c->stream>>>(c->md(), c->slotsA, c->proj16, none, 0, 1);
}

void gather_res(sod_gpu_ctx *c, float *Rmass, float *Rmom, float *Rener, int accumulate, int invml) {
  OutPtrs o{};
  const long long N = c->npoin;
  o.p[0] = Rmass; o.p[1] = Rener; o.p[2] = Rmom; o.p[3] = Rmom + N; o.p[4] = Rmom + 2 * N;
  k_gather<8, 5, false><<<nblk(c->npoin, 256), 256, 0, c->stream>>>(c->md(), c->slotsB, nullptr, o, accumulate, invml);
}

}  // namespace

// ===================================================================
extern "C" {

const char *sod_gpu_last_error(void) { return g_err.c_str(); }

size_t sod_gpu_device_bytes(const sod_gpu_ctx *ctx) { return ctx ? ctx->bytes : 0; }

int sod_gpu_init(const sod_mesh_t *mesh, const sod_phys_t *phys, sod_gpu_ctx **out) {
  if (!mesh || !phys || !out) return fail(SOD_GPU_EINVAL, "null argument");
  *out = nullptr;
  const int P = mesh->porder;
  if (P != 3 && P != 4) return fail(SOD_GPU_EINVAL, "porder must be 3 or 4");
  if (mesh->nelem <= 0 || mesh->npoin <= 0 || mesh->npoin_w <= 0 || mesh->npoin_w > mesh->npoin)
    return fail(SOD_GPU_EINVAL, "bad mesh sizes");
  if (!mesh->connec || !mesh->lpoin_w || !mesh->gmshAtoI || !mesh->gmshAtoJ || !mesh->gmshAtoK ||
      !mesh->dlxigp_ip || !mesh->He || !mesh->gpvol || !mesh->invMl || !mesh->Ml)
    return fail(SOD_GPU_EINVAL, "missing mesh array");
  const int N1 = P + 1, N = N1 * N1 * N1;
  const long long E = mesh->nelem, NP = mesh->npoin;
  if (E * N > 2147483647LL) return fail(SOD_GPU_EINVAL, "nelem*nnode exceeds int32 slot indexing");

  // tensor position of each reference local node
  std::vector<int> t_of_a(N), a_of_t(N, -1);
  for (int a = 0; a < N; ++a) {
    int I = mesh->gmshAtoI[a] - 1, J = mesh->gmshAtoJ[a] - 1, K = mesh->gmshAtoK[a] - 1;
    if (I < 0 || I >= N1 || J < 0 || J >= N1 || K < 0 || K >= N1) return fail(SOD_GPU_EINVAL, "bad gmshAtoI/J/K");
    int t = nat_of(P, I) + N1 * (nat_of(P, J) + N1 * nat_of(P, K));
    if (a_of_t[t] != -1) return fail(SOD_GPU_EINVAL, "gmshAtoI/J/K is not a permutation");
    t_of_a[a] = t;
    a_of_t[t] = a;
  }
  // 1-D derivative matrix in natural order, from dlxigp_ip(ngaus,1,ii)
  std::vector<float> D(N1 * N1);
  for (int a = 0; a < N; ++a) {
    int mrow = nat_of(P, mesh->gmshAtoI[a] - 1);
    for (int ii = 0; ii < N1; ++ii) D[mrow * N1 + nat_of(P, ii)] = mesh->dlxigp_ip[a + (long long)N * (0 + 3 * ii)];
  }
  std::vector<int> conn((size_t)E * N);
  std::vector<float> geo((size_t)E * 10 * N);
  std::vector<int> cnt(NP + 1, 0);
  for (long long e = 0; e < E; ++e)
    for (int a = 0; a < N; ++a) {
      int p = mesh->connec[e + E * a] - 1;
      if (p < 0 || p >= NP) return fail(SOD_GPU_EINVAL, "connectivity out of range");
      int t = t_of_a[a];
      conn[e * N + t] = p;
      cnt[p + 1]++;
      const float *he = mesh->He + 9 * ((long long)a + (long long)N * e);
      for (int c = 0; c < 9; ++c) geo[(e * 10 + c) * N + t] = he[c];
      geo[(e * 10 + 9) * N + t] = mesh->gpvol[a + (long long)N * e];
    }
  for (long long p = 0; p < NP; ++p) cnt[p + 1] += cnt[p];
  std::vector<int> slot_idx((size_t)E * N), fillp(cnt.begin(), cnt.end() - 1);
  for (long long e = 0; e < E; ++e)
    for (int t = 0; t < N; ++t) slot_idx[fillp[conn[e * N + t]]++] = (int)(e * N + t);
  std::vector<int> lw(mesh->npoin_w);
  for (int t = 0; t < mesh->npoin_w; ++t) {
    lw[t] = mesh->lpoin_w[t] - 1;
    if (lw[t] < 0 || lw[t] >= NP) return fail(SOD_GPU_EINVAL, "lpoin_w out of range");
  }

  sod_gpu_ctx *c = new sod_gpu_ctx();
  c->P = P; c->N1 = N1; c->N = N; c->nelem = mesh->nelem; c->npoin = mesh->npoin; c->npoin_w = mesh->npoin_w;
  c->phys = *phys;
  c->ph.gm1 = phys->gamma_gas - 1.0f;
  c->ph.gogm1 = phys->gamma_gas / (phys->gamma_gas - 1.0f);
  c->ph.Rgas = phys->Rgas; c->ph.Cp = phys->Cp; c->ph.Prt = phys->Prt;
  c->ph.c_lps = phys->c_lps; c->ph.c_rho = phys->c_rho; c->ph.c_ener = phys->c_ener;
  c->ph.cp_pr = phys->Cp / phys->Prt;
  c->ph.twoThirds = 2.0f / 3.0f;
  int rc = 0;
  if ((rc = c->upload(&c->conn, conn.data(), conn.size())) || (rc = c->upload(&c->geo, geo.data(), geo.size())) ||
      (rc = c->upload(&c->Dnat, D.data(), D.size())) || (rc = c->upload(&c->lpoin_w, lw.data(), lw.size())) ||
      (rc = c->upload(&c->slot_ptr, cnt.data(), cnt.size())) ||
      (rc = c->upload(&c->slot_idx, slot_idx.data(), slot_idx.size())) ||
      (rc = c->upload(&c->invMl, mesh->invMl, (size_t)NP)) || (rc = c->upload(&c->Ml, mesh->Ml, (size_t)NP)) ||
      (rc = c->upload(&c->a_of_t, a_of_t.data(), a_of_t.size())) ||
      (rc = c->alloc(&c->slotsA, (size_t)E * N * 16)) || (rc = c->alloc(&c->slotsB, (size_t)E * N * 8)) ||
      (rc = c->alloc(&c->proj16, (size_t)NP * 16)) || (rc = c->alloc(&c->mue_t, (size_t)E * N))) {
    sod_gpu_finalize(c);
    return rc;
  }
  if (mesh->helem && (rc = c->upload(&c->helem, mesh->helem, (size_t)E))) { sod_gpu_finalize(c); return rc; }
  if (mesh->lelpn && (rc = c->upload(&c->lelpn, mesh->lelpn, (size_t)NP))) { sod_gpu_finalize(c); return rc; }
  if (mesh->helem_l) {
    std::vector<float> hl((size_t)E * N);
    for (long long e = 0; e < E; ++e)
      for (int a = 0; a < N; ++a) hl[e * N + t_of_a[a]] = mesh->helem_l[e + E * a];
    if ((rc = c->upload(&c->helem_l_t, hl.data(), hl.size()))) { sod_gpu_finalize(c); return rc; }
  }
  *out = c;
  return 0;
}

int sod_gpu_finalize(sod_gpu_ctx *ctx) {
  if (!ctx) return 0;
  for (void *p : ctx->allocs) cudaFree(p);
  delete ctx;
  return 0;
}

int sod_gpu_set_stream(sod_gpu_ctx *ctx, void *stream) {
  if (!ctx) return fail(SOD_GPU_EINVAL, "null context");
  ctx->stream = (cudaStream_t)stream;
  return 0;
}

int sod_gpu_set_async(sod_gpu_ctx *ctx, int enabled) {
  if (!ctx) return fail(SOD_GPU_EINVAL, "null context");
  ctx->async = enabled != 0;
  return 0;
}

int sod_gpu_synchronize(sod_gpu_ctx *ctx) {
  if (!ctx) return fail(SOD_GPU_EINVAL, "null context");
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int sod_gpu_lumped_solver(sod_gpu_ctx *c, float *R, int ncomp) {
  if (!c || !R || ncomp < 1) return fail(SOD_GPU_EINVAL, "bad argument");
  k_lumped<<<nblk(c->npoin_w, 256), 256, 0, c->stream>>>(c->npoin_w, c->npoin, c->lpoin_w, c->invMl, R, ncomp);
  return c->finish();
}

int sod_gpu_comp_tau(sod_gpu_ctx *c, const float *csound, const float *u, float *tau) {
  if (!c || !csound || !u || !tau) return fail(SOD_GPU_EINVAL, "bad argument");
  if (!c->helem) return fail(SOD_GPU_EINVAL, "comp_tau needs helem at init");
  k_comp_tau<<<nblk(c->nelem, 8), 256, 0, c->stream>>>(c->nelem, c->N, c->conn, c->helem, csound, u, c->npoin,
                                                      c->phys.c_species_stab / (float)c->P, tau);
  return c->finish();
}

int sod_gpu_full_convec_ijk(sod_gpu_ctx *c, const float *u, const float *q, const float *rho, const float *pr,
                            const float *E, float *Rmass, float *Rmom, float *Rener, int initialze, float fact) {
  if (!c || !u || !q || !rho || !pr || !E || !Rmass || !Rmom || !Rener) return fail(SOD_GPU_EINVAL, "bad argument");
  RhsArgs A{};
  A.u = u; A.q = q; A.rho = rho; A.pr = pr; A.E = E; A.fact_c = fact;
  int rc = dispatch(c, [&](auto L) {
    L.template rhs<MODE_CONV, IN_PRIM>(c, A);
    return 0;
  });
  if (rc) return rc;
  gather_res(c, Rmass, Rmom, Rener, initialze ? 0 : 1, 0);
  return c->finish();
}

int sod_gpu_full_proj_ijk(sod_gpu_ctx *c, const float *rho, const float *u, const float *Tem, float *ProjMass,
                          float *ProjEner, float *ProjMX, float *ProjMY, float *ProjMZ) {
  if (!c || !rho || !u || !Tem || !ProjMass || !ProjEner || !ProjMX || !ProjMY || !ProjMZ)
    return fail(SOD_GPU_EINVAL, "bad argument");
  int rc = dispatch(c, [&](auto L) {
    L.proj(c, true, rho, u, Tem);
    return 0;
  });
  if (rc) return rc;
  OutPtrs o{};
  const long long N = c->npoin;
  float *f5[5] = {ProjMX, ProjMY, ProjMZ, ProjMass, ProjEner};
  for (int f = 0; f < 5; ++f)
    for (int d = 0; d < 3; ++d) o.p[f * 3 + d] = f5[f] + N * d;
  k_gather<16, 15, false><<<nblk(c->npoin, 256), 256, 0, c->stream>>>(c->md(), c->slotsA, nullptr, o, 0, 1);
  return c->finish();
}

int sod_gpu_full_diff_stab_ijk(sod_gpu_ctx *c, float Cp, float Pr, const float *rho_n, const float *rho,
                               const float *u, const float *Tem, const float *mu_fluid, const float *mu_e,
                               const float *mu_sgs, const float *ProjMass, const float *ProjEner,
                               const float *ProjMX, const float *ProjMY, const float *ProjMZ,
                               const float *tau_stab, float *Rmass, float *Rmom, float *Rener, int initialze,
                               float fact) {
  if (!c || !rho_n || !rho || !u || !Tem || !mu_fluid || !mu_e || !ProjMass || !ProjEner || !ProjMX || !ProjMY ||
      !ProjMZ || !tau_stab || !Rmass || !Rmom || !Rener)
    return fail(SOD_GPU_EINVAL, "bad argument");
  if (rho_n != rho) return fail(SOD_GPU_EINVAL, "rho_n must alias rho (as every reference caller passes)");
  const long long EN = (long long)c->nelem * c->N;
  k_elem_to_t<<<nblk(EN, 256), 256, 0, c->stream>>>(c->nelem, c->N, c->a_of_t, mu_e, c->mue_t);
  if (mu_sgs) {
    if (!c->musgs_t) {
      int rc = c->alloc(&c->musgs_t, (size_t)EN);
      if (rc) return rc;
    }
    k_elem_to_t<<<nblk(EN, 256), 256, 0, c->stream>>>(c->nelem, c->N, c->a_of_t, mu_sgs, c->musgs_t);
  }
  k_pack_proj<<<nblk(c->npoin, 256), 256, 0, c->stream>>>(c->npoin, ProjMX, ProjMY, ProjMZ, ProjMass, ProjEner,
                                                          c->proj16);
  RhsArgs A{};
  A.rho = rho; A.u = u; A.Tem = Tem; A.mu_fluid = mu_fluid;
  A.mue_t = c->mue_t; A.musgs_t = mu_sgs ? c->musgs_t : nullptr; A.tau_stab = tau_stab; A.proj16 = c->proj16;
  A.fact_d = fact;
  Phys saved = c->ph;
  c->ph.Cp = Cp; c->ph.Prt = Pr;
  int rc = dispatch(c, [&](auto L) {
    L.template rhs<MODE_DIFF, IN_DIFF>(c, A);
    return 0;
  });
  c->ph = saved;
  if (rc) return rc;
  gather_res(c, Rmass, Rmom, Rener, initialze ? 0 : 1, 0);
  return c->finish();
}

int sod_gpu_set_mu_e(sod_gpu_ctx *c, const float *mu_e) {
  if (!c || !mu_e) return fail(SOD_GPU_EINVAL, "bad argument");
  const long long EN = (long long)c->nelem * c->N;
  k_elem_to_t<<<nblk(EN, 256), 256, 0, c->stream>>>(c->nelem, c->N, c->a_of_t, mu_e, c->mue_t);
  c->mue_set = true;
  return c->finish();
}

int sod_gpu_updateF(sod_gpu_ctx *c, const float *rho, const float *q, const float *E, const float *mu_e,
                    float mu_factor, const float *tau_stab, float *Rmass, float *Rmom, float *Rener, float *u_out,
                    float *pr_out, float *Tem_out, float *mu_fluid_out) {
  if (!c || !rho || !q || !E || !tau_stab || !Rmass || !Rmom || !Rener)
    return fail(SOD_GPU_EINVAL, "bad argument");
  if (!mu_e && !c->mue_set) return fail(SOD_GPU_EINVAL, "mu_e is NULL and sod_gpu_set_mu_e was not called");
  const long long EN = (long long)c->nelem * c->N;
  if (mu_e) k_elem_to_t<<<nblk(EN, 256), 256, 0, c->stream>>>(c->nelem, c->N, c->a_of_t, mu_e, c->mue_t);
  RhsArgs A{};
  A.rho = rho; A.q = q; A.E = E; A.mu_factor = mu_factor;
  A.mue_t = c->mue_t; A.tau_stab = tau_stab; A.proj16 = c->proj16;
  A.fact_c = -1.0f; A.fact_d = -1.0f;
  int rc = dispatch(c, [&](auto L) {
    L.proj(c, false, rho, q, E);
    gather_proj_aos(c);
    L.template rhs<MODE_CONV | MODE_DIFF, IN_CONS>(c, A);
    return 0;
  });
  if (rc) return rc;
  gather_res(c, Rmass, Rmom, Rener, 0, 1);
  if (u_out || pr_out || Tem_out || mu_fluid_out)
    k_eos_out<<<nblk(c->npoin_w, 256), 256, 0, c->stream>>>(c->npoin_w, c->npoin, c->lpoin_w, c->ph, c->phys.Rgas,
                                                            mu_factor, rho, q, E, u_out, pr_out, Tem_out,
                                                            mu_fluid_out);
  return c->finish();
}

}  // extern "C"
