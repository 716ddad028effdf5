// Learned element-patch preconditioner of the pressure solve: its
// application, set-up, loss and gradient, harvest and training
// (declarations: include/sod2d_gpu.h; kernels: precond_net.cuh).
#include "cg_common.cuh"

namespace sod_net {
int net_forward_fp32(sod_gpu_ctx *c, const double *r, double *z);
}  // namespace sod_net
using sod_net::net_forward_fp32;

namespace sod_net {

int apply_precond(sod_gpu_ctx *c, int kind, const double *r, double *z) {
  if (kind == 0) {
    k_jacobi64<<<nblk(c->npoin_w, 256), 256, 0, c->stream>>>(c->npoin_w, c->lpoin_w, c->cg.Minv, r, z);
    return 0;
  }
  auto &NT = c->net;
  if (!NT.ready) return fail(SOD_GPU_EINVAL, "learned preconditioner not set up (sod_gpu_precond_init)");
  int rc;
  if ((rc = ensure_gains(c))) return rc;
  k_scale_f32<<<nblk(c->npoin_w, 256), 256, 0, c->stream>>>(c->npoin_w, c->lpoin_w, r, NT.Dh, NT.uf);
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    constexpr int P = LL::P_;
    using D = NetDims<P>;
    k_patch_apply_tc<P><<<tc_grid<P>(c->nelem), TC_THREADS, TcDims<P>::smem(), c->stream>>>(
        c->nelem, NT.pt, NT.pos, NT.uf, NT.params, NT.gains, c->slotsB, nullptr);
    k_patch_gather_perm<<<nblk(c->npoin, 256), 256, 0, c->stream>>>(c->npoin, NT.pptr, c->slotsB, r, NT.Dh,
                                                                    NT.params, D::O_ALPHA, z);
    return 0;
  });
  return 0;
}

// FP32 (CUDA-core) forward of the same map, used by training so that the
// gradients follow the FP32 parameters exactly.
int net_forward_fp32(sod_gpu_ctx *c, const double *r, double *z) {
  auto &NT = c->net;
  int rc;
  if ((rc = ensure_gains(c))) return rc;
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    constexpr int P = LL::P_;
    using D = NetDims<P>;
    k_patch_apply<P><<<4 * 148, 256, D::apply_smem(8), c->stream>>>(c->nelem, NT.pt, r, NT.Dh, NT.params, NT.gains,
                                                                    c->slotsB);
    k_patch_gather<<<nblk(c->npoin, 256), 256, 0, c->stream>>>(c->npoin, NT.pptr, NT.pslot, c->slotsB, r, NT.Dh,
                                                               NT.params, D::O_ALPHA, z);
    return 0;
  });
  return 0;
}

}  // namespace sod_net

// ---- learned preconditioner: set-up, loss/gradient, harvest, training ----

namespace {

__global__ void k_loss_grad_vec(int npoin_w, const int *__restrict__ lpoin_w, const double *__restrict__ Ad,
                                double scale, double *__restrict__ g) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const int i = lpoin_w[t];
  g[i] = scale * Ad[i];
}


__global__ void k_inv_sqrt_diag(long long n, const float *__restrict__ diag, double *__restrict__ Dh) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) Dh[i] = diag[i] > 0.f ? 1.0 / sqrt((double)diag[i]) : 0.0;
}

}  // namespace

namespace sod_net {

int ensure_gains(sod_gpu_ctx *c) {
  auto &NT = c->net;
  if (NT.gains_ok) return 0;
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    k_mlp_gains<LL::P_><<<nblk(c->nelem, 8), 256, 0, c->stream>>>(c->nelem, NT.feat, NT.params, NT.gains);
    return 0;
  });
  NT.gains_ok = true;
  return 0;
}

}  // namespace sod_net

namespace {

int ensure_train_scratch(sod_gpu_ctx *c) {
  auto &NT = c->net;
  if (NT.dS) return 0;
  return c->alloc(&NT.dS, (size_t)c->nelem * NET_K);
}

// Parameter-gradient partials of g = dL/dz at the residual r into part
// (nblk_bwd rows of nparam floats), or added to them (accumulate).
void net_backward(sod_gpu_ctx *c, const double *r, const double *g, float *part, int accumulate) {
  auto &NT = c->net;
  const long long stride = NT.nparam;
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    constexpr int P = LL::P_;
    using D = NetDims<P>;
    k_patch_bwd_dB<P><<<NT.nblk_bwd, 256, BwdDims<P>::smem(), c->stream>>>(
        c->nelem, NT.pt, r, g, NT.Dh, NT.params, NT.gains, NT.dS, part, stride, accumulate);
    k_mlp_bwd<P><<<NT.nblk_bwd, 256, 0, c->stream>>>(c->nelem, NT.feat, NT.params, NT.dS, part, stride, accumulate);
    k_alpha_part<<<NT.nblk_bwd, 256, 0, c->stream>>>(c->npoin_w, c->lpoin_w, r, g, NT.Dh, NT.params, D::O_ALPHA,
                                                     part, stride, accumulate);
    return 0;
  });
}

// loss = d^T A d / eAe with d = e - M r; the gradient partials go to part
// (or are added to it: accumulate).
int net_loss_grad(sod_gpu_ctx *c, const double *r, const double *e, double eAe, float *part, double *loss,
                  int accumulate = 0) {
  auto &NT = c->net;
  auto &G = c->cg;
  const int nw = c->npoin_w;
  const unsigned nb = nblk(nw, 256);
  int rc;
  if ((rc = ensure_train_scratch(c)) || (rc = net_forward_fp32(c, r, NT.tmp1))) return rc;  // z
  k_axpby<double><<<nb, 256, 0, c->stream>>>(nw, c->lpoin_w, 1.0, e, -1.0, NT.tmp1);        // d = e - z
  lap<double>(c, NT.tmp1, NT.tmp2);                                                         // A d
  dots<double, 1>(c, DotArgs<double, 1>{{NT.tmp1}, {NT.tmp2}, {nullptr}}, G.dots + 2);
  k_loss_grad_vec<<<nb, 256, 0, c->stream>>>(nw, c->lpoin_w, NT.tmp2, -2.0 / eAe, NT.tmp2);
  net_backward(c, r, NT.tmp2, part, accumulate);
  if (loss) {
    double h;
    CUDA_TRY(cudaMemcpyAsync(&h, G.dots + 2, 8, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    *loss = h / eAe;
  }
  return 0;
}

// Face neighbours (element itself on a boundary) and the patch table: own
// nodes in tensor order, then for each face f the first node layer of the
// neighbour across f, at the face's tangential coordinates (a, b) of this
// element's frame (-1 without a neighbour).  The neighbour's layer is found
// from the affine map between the two elements' face corners, so any
// relative orientation of conforming hexahedra is handled.
int build_patch_table(sod_gpu_ctx *c, const std::vector<int> &conn, std::vector<int> &pt) {
  const int P = c->P, N1 = c->N1, N = c->N, F2 = N1 * N1, NP = N + 6 * F2;
  const long long E = c->nelem;
  auto tid = [&](const int *ijk) { return ijk[0] + N1 * (ijk[1] + N1 * ijk[2]); };
  auto face_ijk = [&](int f, int a, int b, int *ijk) {
    const int d = f / 2, d1 = d == 0 ? 1 : 0, d2 = d == 2 ? 1 : 2;
    ijk[d] = (f % 2) ? P : 0;
    ijk[d1] = a;
    ijk[d2] = b;
  };
  struct FaceKey {
    std::array<int, 4> k;
    long long e;
    int f;
  };
  std::vector<FaceKey> keys((size_t)E * 6);
  for (long long e = 0; e < E; ++e)
    for (int f = 0; f < 6; ++f) {
      FaceKey &fk = keys[e * 6 + f];
      int q = 0, ijk[3];
      for (int a = 0; a <= P; a += P)
        for (int b = 0; b <= P; b += P) {
          face_ijk(f, a, b, ijk);
          fk.k[q++] = conn[e * N + tid(ijk)];
        }
      std::sort(fk.k.begin(), fk.k.end());
      fk.e = e;
      fk.f = f;
    }
  std::sort(keys.begin(), keys.end(), [](const FaceKey &x, const FaceKey &y) {
    return x.k != y.k ? x.k < y.k : (x.e != y.e ? x.e < y.e : x.f < y.f);
  });
  std::vector<long long> nbr((size_t)E * 6);
  for (long long i = 0; i < E * 6; ++i) nbr[i] = i / 6;
  for (size_t i = 0; i < keys.size();) {
    size_t j = i + 1;
    while (j < keys.size() && keys[j].k == keys[i].k) ++j;
    if (j - i == 2) {
      nbr[keys[i].e * 6 + keys[i].f] = keys[i + 1].e;
      nbr[keys[i + 1].e * 6 + keys[i + 1].f] = keys[i].e;
    }
    i = j;
  }
  pt.assign((size_t)E * NP, -1);
  for (long long e = 0; e < E; ++e) {
    for (int t = 0; t < N; ++t) pt[e * NP + t] = conn[e * N + t];
    for (int f = 0; f < 6; ++f) {
      const long long e2 = nbr[e * 6 + f];
      if (e2 == e) continue;
      auto locate = [&](int a, int b, int *out) {
        int ijk[3];
        face_ijk(f, a, b, ijk);
        const int g = conn[e * N + tid(ijk)];
        for (int t = 0; t < N; ++t)
          if (conn[e2 * N + t] == g) {
            out[0] = t % N1; out[1] = (t / N1) % N1; out[2] = t / F2;
            return true;
          }
        return false;
      };
      int c00[3], cP0[3], c0P[3];
      if (!locate(0, 0, c00) || !locate(P, 0, cP0) || !locate(0, P, c0P))
        return fail(SOD_GPU_EINVAL, "inconsistent face connectivity");
      int dn = -1, ncst = 0;
      for (int x = 0; x < 3; ++x)
        if (c00[x] == cP0[x] && c00[x] == c0P[x]) { dn = x; ++ncst; }
      if (ncst != 1 || (c00[dn] != 0 && c00[dn] != P)) return fail(SOD_GPU_EINVAL, "inconsistent face connectivity");
      const int step = c00[dn] == 0 ? 1 : -1;
      for (int b = 0; b <= P; ++b)
        for (int a = 0; a <= P; ++a) {
          int ijk2[3];
          for (int x = 0; x < 3; ++x) ijk2[x] = c00[x] + (cP0[x] - c00[x]) / P * a + (c0P[x] - c00[x]) / P * b;
          ijk2[dn] += step;
          pt[e * NP + N + f * F2 + a + N1 * b] = conn[e2 * N + tid(ijk2)];
        }
    }
  }
  return 0;
}

}  // namespace

extern "C" {

int sod_gpu_precond_num_params(sod_gpu_ctx *c) {
  if (!c) return fail(SOD_GPU_EINVAL, "null context");
  return c->P == 3 ? NetDims<3>::NPARAM : NetDims<4>::NPARAM;
}

int sod_gpu_precond_init(sod_gpu_ctx *c, uint64_t seed, int harvest_capacity) {
  if (!c || harvest_capacity < 0) return fail(SOD_GPU_EINVAL, "bad argument");
  int rc;
  if ((rc = ensure_diag(c)) || (rc = ensure_cg64(c))) return rc;
  auto &NT = c->net;
  const int N = c->N, P = c->P;
  const long long E = c->nelem;
  if (!NT.ready) {
    NT.nparam = sod_gpu_precond_num_params(c);
    NT.NP = P == 3 ? NetDims<3>::NP : NetDims<4>::NP;
    NT.nblk_bwd = 4 * num_sms();  // blocks (and partial rows) of the gradient reductions
    const size_t NPt = (size_t)E * NT.NP;
    if ((rc = c->alloc(&NT.params, NT.nparam)) || (rc = c->alloc(&NT.m1, NT.nparam)) ||
        (rc = c->alloc(&NT.m2, NT.nparam)) || (rc = c->alloc(&NT.grad, NT.nparam)) ||
        (rc = c->alloc(&NT.part, (size_t)NT.nblk_bwd * NT.nparam)) || (rc = c->alloc(&NT.pt, NPt)) || (rc = c->alloc(&NT.pos, NPt)) ||
        (rc = c->alloc(&NT.pptr, (size_t)c->npoin + 1)) || (rc = c->alloc(&NT.pslot, NPt)) ||
        (rc = c->alloc(&NT.feat, (size_t)E * NET_F)) || (rc = c->alloc(&NT.gains, (size_t)E * NET_K)) ||
        (rc = c->alloc(&NT.Dh, (size_t)c->npoin)) || (rc = c->alloc(&NT.uf, (size_t)c->npoin)) ||
        (rc = c->alloc(&NT.tmp1, (size_t)c->npoin)) ||
        (rc = c->alloc(&NT.tmp2, (size_t)c->npoin)))
      return rc;
    if (P == 3) {
      using D = NetDims<3>;
      CUDA_TRY(cudaFuncSetAttribute(k_patch_apply<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)D::apply_smem(8)));
      CUDA_TRY(cudaFuncSetAttribute(k_patch_bwd_dB<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)BwdDims<3>::smem()));
      CUDA_TRY(cudaFuncSetAttribute(k_patch_apply_tc<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)TcDims<3>::smem()));
    } else {
      using D = NetDims<4>;
      CUDA_TRY(cudaFuncSetAttribute(k_patch_apply<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)D::apply_smem(8)));
      CUDA_TRY(cudaFuncSetAttribute(k_patch_bwd_dB<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)BwdDims<4>::smem()));
      CUDA_TRY(cudaFuncSetAttribute(k_patch_apply_tc<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)TcDims<4>::smem()));
    }
    // patch table and its node-centric CSR (slots in increasing (e, j) order)
    std::vector<int> conn((size_t)E * N), pt;
    CUDA_TRY(cudaMemcpy(conn.data(), c->conn, conn.size() * 4, cudaMemcpyDeviceToHost));
    if ((rc = build_patch_table(c, conn, pt))) return rc;
    std::vector<int> pptr(c->npoin + 1, 0), pslot(pt.size()), pos(pt.size(), -1);
    for (int v : pt)
      if (v >= 0) pptr[v + 1]++;
    for (long long n = 0; n < c->npoin; ++n) pptr[n + 1] += pptr[n];
    std::vector<int> fill(pptr.begin(), pptr.end() - 1);
    for (size_t i = 0; i < pt.size(); ++i)
      if (pt[i] >= 0) {
        pos[i] = fill[pt[i]];
        pslot[fill[pt[i]]++] = (int)i;
      }
    CUDA_TRY(cudaMemcpy(NT.pt, pt.data(), pt.size() * 4, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(NT.pos, pos.data(), pos.size() * 4, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(NT.pptr, pptr.data(), pptr.size() * 4, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(NT.pslot, pslot.data(), (size_t)pptr[c->npoin] * 4, cudaMemcpyHostToDevice));
    // geometry features, the last two relative to their mesh mean
    dispatch(c, [&](auto L) {
      using LL = decltype(L);
      k_elem_features<LL::P_><<<nblk(E, 8), 256, 0, c->stream>>>(c->md(), NT.tmp1);
      return 0;
    });
    std::vector<double> raw((size_t)E * NET_F);
    CUDA_TRY(cudaMemcpyAsync(raw.data(), NT.tmp1, raw.size() * 8, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    double mean6 = 0.0, mean7 = 0.0;
    for (long long e = 0; e < E; ++e) { mean6 += raw[e * NET_F + 6]; mean7 += raw[e * NET_F + 7]; }
    mean6 /= (double)E;
    mean7 /= (double)E;
    std::vector<float> feat(raw.size());
    for (long long e = 0; e < E; ++e)
      for (int q = 0; q < NET_F; ++q)
        feat[e * NET_F + q] = (float)(raw[e * NET_F + q] - (q == 6 ? mean6 : (q == 7 ? mean7 : 0.0)));
    CUDA_TRY(cudaMemcpy(NT.feat, feat.data(), feat.size() * 4, cudaMemcpyHostToDevice));
    k_inv_sqrt_diag<<<nblk(c->npoin, 256), 256, 0, c->stream>>>(c->npoin, c->cg.diag, NT.Dh);
    NT.ready = true;
  }
  // seeded initial parameters: small patch modes, zero skip exponent, Xavier
  // hidden layers, zero output layer with unit gains: the map starts as Jacobi
  {
    const int NPn = NT.NP, H = NET_H, K = NET_K, Fn = NET_F;
    const int o_alpha = K * NPn, o_w1 = o_alpha + 1, o_b1 = o_w1 + Fn * H, o_w2 = o_b1 + H, o_b2 = o_w2 + H * H,
              o_w3 = o_b2 + H, o_b3 = o_w3 + H * K;
    std::vector<float> p(NT.nparam, 0.f);
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<float> U(-1.f, 1.f);
    for (int i = 0; i < K * NPn; ++i) p[i] = 1.7e-3f * U(rng);
    const float a1 = std::sqrt(6.f / (Fn + H)), a2 = std::sqrt(6.f / (H + H));
    for (int i = 0; i < Fn * H; ++i) p[o_w1 + i] = a1 * U(rng);
    for (int i = 0; i < H * H; ++i) p[o_w2 + i] = a2 * U(rng);
    for (int i = 0; i < K; ++i) p[o_b3 + i] = 0.54132485f;  // softplus^-1(1)
    CUDA_TRY(cudaMemcpy(NT.params, p.data(), p.size() * 4, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemset(NT.m1, 0, (size_t)NT.nparam * 4));
    CUDA_TRY(cudaMemset(NT.m2, 0, (size_t)NT.nparam * 4));
    NT.step = 0;
    NT.gains_ok = false;
    NT.rs_state = 0x9e3779b97f4a7c15ULL ^ seed;
  }
  if (harvest_capacity > 0 && harvest_capacity != NT.cap) {
    if ((rc = c->alloc(&NT.hr, (size_t)harvest_capacity * c->npoin)) ||
        (rc = c->alloc(&NT.he, (size_t)harvest_capacity * c->npoin)) ||
        (!NT.xsnap && (rc = c->alloc(&NT.xsnap, (size_t)16 * c->npoin))))
      return rc;
    CUDA_TRY(cudaMemset(NT.hr, 0, (size_t)harvest_capacity * c->npoin * 4));
    CUDA_TRY(cudaMemset(NT.he, 0, (size_t)harvest_capacity * c->npoin * 4));
    NT.cap = harvest_capacity;
    NT.count = 0;
    NT.offered = 0;
    NT.eAe.assign(harvest_capacity, 1.0);
  }
  return c->finish();
}

int sod_gpu_precond_set_params(sod_gpu_ctx *c, const float *host_params, int n) {
  if (!c || !c->net.ready || !host_params || n != c->net.nparam) return fail(SOD_GPU_EINVAL, "bad argument");
  CUDA_TRY(cudaMemcpy(c->net.params, host_params, (size_t)n * 4, cudaMemcpyHostToDevice));
  c->net.gains_ok = false;
  return 0;
}

int sod_gpu_precond_get_params(sod_gpu_ctx *c, float *host_params, int n) {
  if (!c || !c->net.ready || !host_params || n != c->net.nparam) return fail(SOD_GPU_EINVAL, "bad argument");
  CUDA_TRY(cudaMemcpy(host_params, c->net.params, (size_t)n * 4, cudaMemcpyDeviceToHost));
  return 0;
}

int sod_gpu_precond_apply(sod_gpu_ctx *c, const double *r, double *z) {
  if (!c || !r || !z) return fail(SOD_GPU_EINVAL, "bad argument");
  int rc;
  if ((rc = ensure_diag(c)) || (rc = ensure_cg64(c))) return rc;
  if ((rc = apply_precond(c, 1, r, z))) return rc;
  return c->finish();
}

int sod_gpu_precond_loss_grad(sod_gpu_ctx *c, const double *r, const double *e, double *loss, float *grad_host) {
  if (!c || !c->net.ready || !r || !e || !loss) return fail(SOD_GPU_EINVAL, "bad argument");
  auto &NT = c->net;
  lap<double>(c, e, NT.tmp2);
  dots<double, 1>(c, DotArgs<double, 1>{{e}, {NT.tmp2}, {nullptr}}, c->cg.dots + 5);
  double eAe;
  CUDA_TRY(cudaMemcpyAsync(&eAe, c->cg.dots + 5, 8, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (!(eAe > 0)) return fail(SOD_GPU_EINVAL, "target has zero energy norm");
  int rc = net_loss_grad(c, r, e, eAe, NT.part, loss);
  if (rc) return rc;
  k_adam<<<nblk(NT.nparam, 256), 256, 0, c->stream>>>(NT.nparam, NT.nblk_bwd, NT.part, NT.params, NT.m1, NT.m2, 0.f,
                                                      0.9f, 0.999f, 1e-8f, 1.f, 1.f, 1.f, NT.grad);
  if (grad_host) CUDA_TRY(cudaMemcpyAsync(grad_host, NT.grad, (size_t)NT.nparam * 4, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return c->finish();
}

int sod_gpu_precond_harvest_count(sod_gpu_ctx *c) { return c ? c->net.count : 0; }

// Adam on the harvested (r, e) pairs: `steps` updates of `batch` pairs each;
// *final_loss (host) = mean relative A-norm loss of the last batch.
int sod_gpu_precond_restart_harvest(sod_gpu_ctx *c) {
  if (!c || !c->net.ready) return fail(SOD_GPU_EINVAL, "learned preconditioner not set up (sod_gpu_precond_init)");
  auto &NT = c->net;
  NT.count = 0;
  NT.offered = 0;
  NT.step = 0;
  CUDA_TRY(cudaMemsetAsync(NT.m1, 0, (size_t)NT.nparam * 4, c->stream));
  CUDA_TRY(cudaMemsetAsync(NT.m2, 0, (size_t)NT.nparam * 4, c->stream));
  return c->finish();
}

int sod_gpu_precond_train(sod_gpu_ctx *c, int steps, int batch, float lr, uint64_t seed, float *final_loss) {
  if (!c || !c->net.ready || steps < 0 || batch < 1 || batch > 16) return fail(SOD_GPU_EINVAL, "bad argument");
  auto &NT = c->net;
  if (NT.count < 1) return fail(SOD_GPU_EINVAL, "no harvested pairs to train on");
  double *rd = c->cg.z1, *ed = c->cg.q;  // FP64 staging of one pair (solver scratch, idle here)
  std::mt19937_64 rng(seed);
  double last = 0.0;
  const int nw = c->npoin_w;
  const size_t N = c->npoin;
  for (int st = 0; st < steps; ++st) {
    double sum = 0.0;
    for (int b = 0; b < batch; ++b) {
      const int k = (int)(rng() % (uint64_t)NT.count);
      k_f2d_w<<<nblk(nw, 256), 256, 0, c->stream>>>(nw, c->lpoin_w, NT.hr + (size_t)k * N, rd);
      k_f2d_w<<<nblk(nw, 256), 256, 0, c->stream>>>(nw, c->lpoin_w, NT.he + (size_t)k * N, ed);
      double l = 0.0;
      // the batch's gradient partials add up in one set of block rows
      int rc = net_loss_grad(c, rd, ed, NT.eAe[k], NT.part, (st == steps - 1) ? &l : nullptr, b > 0);
      if (rc) return rc;
      sum += l;
    }
    NT.step += 1;
    const float bc1 = 1.f - std::pow(0.9f, (float)NT.step), bc2 = 1.f - std::pow(0.999f, (float)NT.step);
    k_adam<<<nblk(NT.nparam, 256), 256, 0, c->stream>>>(NT.nparam, NT.nblk_bwd, NT.part, NT.params, NT.m1,
                                                        NT.m2, lr, 0.9f, 0.999f, 1e-8f, bc1, bc2, 1.f / batch,
                                                        nullptr);
    NT.gains_ok = false;
    last = sum / batch;
  }
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (final_loss) *final_loss = (float)last;
  return c->finish();
}

}  // extern "C"
