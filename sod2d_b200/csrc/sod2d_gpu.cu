// C-ABI entry points of the B200 spectral-element RHS library: context
// set-up, halo plans, and the compressible RHS operators
// (declarations and contracts: include/sod2d_gpu.h).  The time
// integrators are in comp_step.cu, the incompressible path in incomp.cu,
// the learned preconditioner in precond.cu.
#include "ctx.cuh"

namespace {
thread_local std::string g_err;
}  // namespace

// Records an error message for sod_gpu_last_error() (every translation
// unit of the library reports through this).
int sod_detail_set_error(int code, const char *msg) {
  g_err = msg;
  return code;
}

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
  std::vector<int> slot_idx((size_t)E * N), slot_pos((size_t)E * N), fillp(cnt.begin(), cnt.end() - 1);
  for (long long e = 0; e < E; ++e)
    for (int t = 0; t < N; ++t) {
      const int s = fillp[conn[e * N + t]]++;
      slot_idx[s] = (int)(e * N + t);
      slot_pos[e * N + t] = s;
    }
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
      (rc = c->upload(&c->slot_pos, slot_pos.data(), slot_pos.size())) ||
      (rc = c->upload(&c->invMl, mesh->invMl, (size_t)NP)) || (rc = c->upload(&c->Ml, mesh->Ml, (size_t)NP)) ||
      (rc = c->upload(&c->a_of_t, a_of_t.data(), a_of_t.size())) ||
      (rc = c->alloc(&c->slotsA, (size_t)E * N * 12)) || (rc = c->alloc(&c->slotsB, (size_t)E * N * 8)) ||
      (rc = c->alloc(&c->proj12, (size_t)NP * 12)) || (rc = c->alloc(&c->mue_t, (size_t)E * N))) {
    sod_gpu_finalize(c);
    return rc;
  }
  {
    void *h = nullptr;
    if (cudaHostAlloc(&h, sizeof(int), cudaHostAllocMapped) != cudaSuccess) {
      sod_gpu_finalize(c);
      return fail(SOD_GPU_ENOMEM, "cudaHostAlloc of the wait flag failed");
    }
    c->host_allocs.push_back(h);
    c->err_h = (int *)h;
    *c->err_h = 0;
    if (cudaHostGetDevicePointer((void **)&c->err_d, h, 0) != cudaSuccess) {
      sod_gpu_finalize(c);
      return fail(SOD_GPU_ECUDA, "cudaHostGetDevicePointer of the wait flag failed");
    }
  }
  if ((rc = c->alloc(&c->cg.dticket, 1)) || (rc = c->alloc(&c->cg.part, (size_t)8 * DOT_BLOCKS)) ||
      (rc = c->alloc(&c->cg.dots, 16))) {
    sod_gpu_finalize(c);
    return rc;
  }
  if (cudaMemset(c->cg.dticket, 0, sizeof(unsigned)) != cudaSuccess) {
    sod_gpu_finalize(c);
    return fail(SOD_GPU_ECUDA, "cudaMemset of the dot ticket failed");
  }
  if (mesh->helem && (rc = c->upload(&c->helem, mesh->helem, (size_t)E))) { sod_gpu_finalize(c); return rc; }
  if (mesh->lelpn && (rc = c->upload(&c->lelpn, mesh->lelpn, (size_t)NP))) { sod_gpu_finalize(c); return rc; }
  if (mesh->helem_l) {
    std::vector<float> hl((size_t)E * N);
    for (long long e = 0; e < E; ++e)
      for (int a = 0; a < N; ++a) hl[e * N + t_of_a[a]] = mesh->helem_l[e + E * a];
    if ((rc = c->upload(&c->helem_l_t, hl.data(), hl.size()))) { sod_gpu_finalize(c); return rc; }
  }
  {
    std::vector<int> isw((size_t)NP, 0);
    for (int t = 0; t < mesh->npoin_w; ++t) isw[lw[t]] = 1;
    std::vector<float> Nt((size_t)N * N, 0.f);
    for (int g = 0; g < N; ++g)
      for (int a = 0; a < N; ++a)
        Nt[(size_t)t_of_a[g] * N + t_of_a[a]] = mesh->Ngp ? mesh->Ngp[g + (long long)N * a] : (g == a ? 1.f : 0.f);
    double vol = 0.0;
    for (long long e = 0; e < E; ++e)
      for (int a = 0; a < N; ++a) vol += (double)mesh->gpvol[a + (long long)N * e];
    c->volT = (float)vol;
    if ((rc = c->upload(&c->is_work, isw.data(), isw.size())) || (rc = c->upload(&c->Ngp_t, Nt.data(), Nt.size()))) {
      sod_gpu_finalize(c);
      return rc;
    }
  }
  *out = c;
  return 0;
}

int sod_gpu_finalize(sod_gpu_ctx *ctx) {
  if (!ctx) return 0;
  for (void *p : ctx->halo.own) cudaFree(p);
  for (void *p : ctx->allocs) cudaFree(p);
  for (void *p : ctx->host_allocs) cudaFreeHost(p);
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
  return ctx->check_waits();
}

int sod_gpu_set_halo(sod_gpu_ctx *c, int rank, int nnb, const int *ranksToComm, const int *commsMemPosInLoc,
                     const int *commsMemSize, const int *nodesToComm, float *send_buf, float *recv_buf,
                     sod_halo_exchange_fn exchange, void *user) {
  if (!c) return fail(SOD_GPU_EINVAL, "null context");
  auto &h = c->halo;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  for (void *p : h.own) cudaFree(p);
  h.own.clear();
  h.on = false;
  h.nsend = h.nuniq = 0;
  if (nnb == 0) return 0;
  if (nnb < 0 || !ranksToComm || !commsMemPosInLoc || !commsMemSize || !nodesToComm || !send_buf || !recv_buf ||
      !exchange || rank < 0)
    return fail(SOD_GPU_EINVAL, "bad halo plan argument");
  // validate the plan: contiguous neighbour ranges, distinct neighbours,
  // node ids in range, no node twice in one neighbour's range
  long long nsend = 0;
  for (int i = 0; i < nnb; ++i) {
    if (commsMemSize[i] < 0 || commsMemPosInLoc[i] != nsend + 1 || ranksToComm[i] < 0 || ranksToComm[i] == rank)
      return fail(SOD_GPU_EINVAL, "halo plan: neighbour ranges must be contiguous, 1-based, other ranks");
    for (int j = 0; j < i; ++j)
      if (ranksToComm[j] == ranksToComm[i]) return fail(SOD_GPU_EINVAL, "halo plan: neighbour listed twice");
    nsend += commsMemSize[i];
  }
  if (nsend > (1LL << 30)) return fail(SOD_GPU_EINVAL, "halo plan too large");
  std::vector<int> send_node((size_t)nsend);
  std::vector<std::vector<std::pair<int, int>>> per_node;
  std::vector<int> slot_of((size_t)c->npoin, -1);
  std::vector<int> uniq;
  for (int i = 0; i < nnb; ++i) {
    for (long long j = commsMemPosInLoc[i] - 1; j < commsMemPosInLoc[i] - 1 + commsMemSize[i]; ++j) {
      const int node = nodesToComm[j] - 1;
      if (node < 0 || node >= c->npoin) return fail(SOD_GPU_EINVAL, "halo plan: node id out of range");
      send_node[(size_t)j] = node;
      int &s = slot_of[(size_t)node];
      if (s < 0) {
        s = (int)uniq.size();
        uniq.push_back(node);
        per_node.push_back({{rank, -1}});
      }
      for (auto &pr : per_node[(size_t)s])
        if (pr.first == ranksToComm[i]) return fail(SOD_GPU_EINVAL, "halo plan: node listed twice for a neighbour");
      per_node[(size_t)s].push_back({ranksToComm[i], (int)j});
    }
  }
  std::vector<int> ptr(uniq.size() + 1, 0), src;
  for (size_t u = 0; u < uniq.size(); ++u) {
    auto &v = per_node[u];
    std::sort(v.begin(), v.end());
    for (auto &pr : v) src.push_back(pr.second);
    ptr[u + 1] = (int)src.size();
  }
  auto up = [&](int **d, const std::vector<int> &hv) -> int {
    size_t b = std::max<size_t>(hv.size(), 1) * sizeof(int);
    cudaError_t e = cudaMalloc((void **)d, b);
    if (e != cudaSuccess) return fail(SOD_GPU_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    h.own.push_back(*d);
    if (!hv.empty()) CUDA_TRY(cudaMemcpy(*d, hv.data(), hv.size() * sizeof(int), cudaMemcpyHostToDevice));
    return 0;
  };
  // owned working nodes (the reference's lpoin_o of its dot products): a
  // shared node belongs to the lowest rank that holds it
  std::vector<int> lw((size_t)c->npoin_w), owned;
  CUDA_TRY(cudaMemcpy(lw.data(), c->lpoin_w, lw.size() * sizeof(int), cudaMemcpyDeviceToHost));
  owned.reserve(lw.size());
  for (int p : lw) {
    const int s = slot_of[(size_t)p];
    if (s >= 0 && per_node[(size_t)s].front().first < rank) continue;  // sorted by rank: front is the lowest
    owned.push_back(p);
  }
  int rc;
  if ((rc = up(&h.send_node, send_node)) || (rc = up(&h.uniq_node, uniq)) || (rc = up(&h.ptr, ptr)) ||
      (rc = up(&h.src, src)) || (rc = up(&h.lpoin_o, owned))) {
    for (void *p : h.own) cudaFree(p);
    h.own.clear();
    return rc;
  }
  c->cg.have_diag = false;  // the Jacobi diagonal is assembled over the ranks from now on
  h.rank = rank;
  h.nsend = (int)nsend;
  h.nuniq = (int)uniq.size();
  h.npoin_o = (int)owned.size();
  h.send = send_buf;
  h.recv = recv_buf;
  h.fn = exchange;
  h.user = user;
  h.on = true;
  return 0;
}

int sod_gpu_halo_update(sod_gpu_ctx *c, float *field, int ncomp) {
  if (!c || !field || ncomp < 1) return fail(SOD_GPU_EINVAL, "bad argument");
  const long long N = c->npoin;
  for (int k0 = 0; k0 < ncomp; k0 += HALO_MAX_WIDTH) {
    HaloView v{};
    v.width = std::min(HALO_MAX_WIDTH, ncomp - k0);
    v.nstride = 1;
    for (int k = 0; k < v.width; ++k) v.comp[k] = field + (k0 + k) * N;
    int rc = halo_sum(c, v);
    if (rc) return rc;
  }
  return c->finish();
}

int sod_gpu_set_allreduce(sod_gpu_ctx *c, sod_allreduce_fn fn, void *user) {
  if (!c) return fail(SOD_GPU_EINVAL, "null context");
  auto &h = c->halo;
  h.reduce = fn;
  h.reduce_user = user;
  if (!fn) return 0;
  int rc;
  if (!h.vol && (rc = c->alloc(&h.vol, 1))) return rc;
  // mesh volume of the analysis (visc_dissipationRate's volT): sum over ranks
  double v = (double)c->volT;
  CUDA_TRY(cudaMemcpyAsync(h.vol, &v, 8, cudaMemcpyHostToDevice, c->stream));
  if ((rc = allreduce(c, h.vol, 1, SOD_REDUCE_SUM_F64))) return rc;
  CUDA_TRY(cudaMemcpyAsync(&v, h.vol, 8, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->volT = (float)v;
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
  // assemble into the node-major 12-wide buffer, then expand to the
  // reference's five (npoin,3) arrays
  gather_proj_aos(c);
  if ((rc = halo_sum(c, halo_proj_view(c)))) return rc;
  k_unpack_proj<<<nblk(c->npoin, 256), 256, 0, c->stream>>>(c->npoin, c->proj12, ProjMX, ProjMY, ProjMZ, ProjMass,
                                                            ProjEner);
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
  k_elem_to_t<<<nblk(c->nelem, E2T_TILE), E2T_THREADS, 0, c->stream>>>(c->nelem, c->N, c->a_of_t, mu_e, c->mue_t);
  if (mu_sgs) {
    if (!c->musgs_t) {
      int rc = c->alloc(&c->musgs_t, (size_t)c->nelem * c->N);
      if (rc) return rc;
    }
    k_elem_to_t<<<nblk(c->nelem, E2T_TILE), E2T_THREADS, 0, c->stream>>>(c->nelem, c->N, c->a_of_t, mu_sgs, c->musgs_t);
  }
  k_pack_proj<<<nblk(c->npoin, 256), 256, 0, c->stream>>>(c->npoin, ProjMX, ProjMY, ProjMZ, ProjMass, ProjEner,
                                                          c->proj12);
  RhsArgs A{};
  A.rho = rho; A.u = u; A.Tem = Tem; A.mu_fluid = mu_fluid;
  A.mue_t = c->mue_t; A.musgs_t = mu_sgs ? c->musgs_t : nullptr; A.tau_stab = tau_stab; A.proj12 = c->proj12;
  A.fact_d = fact;
  Phys saved = c->ph;
  c->ph.Cp = Cp; c->ph.Prt = Pr; c->ph.cp_pr = Cp / Pr;
  int rc = dispatch(c, [&](auto L) {
    L.template rhs<MODE_DIFF, IN_DIFF>(c, A);
    return 0;
  });
  c->ph = saved;
  if (rc) return rc;
  gather_res(c, Rmass, Rmom, Rener, initialze ? 0 : 1, 0);
  return c->finish();
}

int sod_gpu_full_diffusion_ijk(sod_gpu_ctx *c, float Cp, float Pr, const float *rho_n, const float *rho,
                               const float *u, const float *Tem, const float *mu_fluid, const float *mu_e,
                               const float *mu_sgs, float *Rmass, float *Rmom, float *Rener, int initialze,
                               float fact) {
  if (!c || !rho_n || !rho || !u || !Tem || !mu_fluid || !mu_e || !Rmass || !Rmom || !Rener)
    return fail(SOD_GPU_EINVAL, "bad argument");
  k_elem_to_t<<<nblk(c->nelem, E2T_TILE), E2T_THREADS, 0, c->stream>>>(c->nelem, c->N, c->a_of_t, mu_e, c->mue_t);
  if (mu_sgs) {
    if (!c->musgs_t) {
      int rc = c->alloc(&c->musgs_t, (size_t)c->nelem * c->N);
      if (rc) return rc;
    }
    k_elem_to_t<<<nblk(c->nelem, E2T_TILE), E2T_THREADS, 0, c->stream>>>(c->nelem, c->N, c->a_of_t, mu_sgs, c->musgs_t);
  }
  RhsArgs A{};
  A.rho = rho; A.u = u; A.Tem = Tem; A.mu_fluid = mu_fluid;
  A.rho_n = rho_n != rho ? rho_n : nullptr;
  A.mue_t = c->mue_t; A.musgs_t = mu_sgs ? c->musgs_t : nullptr;
  A.fact_d = fact;
  Phys saved = c->ph;
  c->ph.Cp = Cp; c->ph.Prt = Pr; c->ph.cp_pr = Cp / Pr;
  int rc = dispatch(c, [&](auto L) {
    L.template rhs<MODE_DIFF | MODE_NOLPS, IN_DIFF>(c, A);
    return 0;
  });
  c->ph = saved;
  if (rc) return rc;
  gather_res(c, Rmass, Rmom, Rener, initialze ? 0 : 1, 0);
  return c->finish();
}

int sod_gpu_set_mu_e(sod_gpu_ctx *c, const float *mu_e) {
  if (!c || !mu_e) return fail(SOD_GPU_EINVAL, "bad argument");
  k_elem_to_t<<<nblk(c->nelem, E2T_TILE), E2T_THREADS, 0, c->stream>>>(c->nelem, c->N, c->a_of_t, mu_e, c->mue_t);
  c->mue_set = true;
  return c->finish();
}

int sod_gpu_updateF(sod_gpu_ctx *c, const float *rho, const float *q, const float *E, const float *mu_e,
                    float mu_factor, const float *tau_stab, float *Rmass, float *Rmom, float *Rener, float *u_out,
                    float *pr_out, float *Tem_out, float *mu_fluid_out) {
  if (!c || !rho || !q || !E || !tau_stab || !Rmass || !Rmom || !Rener)
    return fail(SOD_GPU_EINVAL, "bad argument");
  if (!mu_e && !c->mue_set) return fail(SOD_GPU_EINVAL, "mu_e is NULL and sod_gpu_set_mu_e was not called");
  if (mu_e) k_elem_to_t<<<nblk(c->nelem, E2T_TILE), E2T_THREADS, 0, c->stream>>>(c->nelem, c->N, c->a_of_t, mu_e, c->mue_t);
  RhsArgs A{};
  A.rho = rho; A.q = q; A.E = E; A.mu_factor = mu_factor;
  A.mue_t = c->mue_t; A.tau_stab = tau_stab; A.proj12 = c->proj12;
  A.fact_c = -1.0f; A.fact_d = -1.0f;
  int rc = dispatch(c, [&](auto L) {
    L.proj(c, false, rho, q, E);
    gather_proj_aos(c);
    int hrc = halo_sum(c, halo_proj_view(c));
    if (hrc) return hrc;
    L.template rhs<MODE_CONV | MODE_DIFF, IN_CONS>(c, A);
    return 0;
  });
  if (rc) return rc;
  gather_res(c, Rmass, Rmom, Rener, 0, 1);
  if ((rc = halo_sum(c, halo_res_view(c, Rmass, Rmom, Rener)))) return rc;
  if (u_out || pr_out || Tem_out || mu_fluid_out)
    k_eos_out<<<nblk(c->npoin_w, 256), 256, 0, c->stream>>>(c->npoin_w, c->npoin, c->lpoin_w, c->ph, c->phys.Rgas,
                                                            mu_factor, rho, q, E, u_out, pr_out, Tem_out,
                                                            mu_fluid_out);
  return c->finish();
}

}  // extern "C"
