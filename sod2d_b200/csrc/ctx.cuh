// Internal header of the B200 library: the device context shared by the
// translation units (context and compressible RHS, compressible time
// integration, incompressible operators and solves, learned
// preconditioner) and the launch helpers they all use.  Not installed: the
// public contract is include/sod2d_gpu.h.
#pragma once
#include "sod2d_gpu.h"
#include "rhs_kernels.cuh"
#include "step_kernels.cuh"
#include "incomp_kernels.cuh"
#include "precond_net.cuh"
#include "veloc_kernels.cuh"
#include "imex_kernels.cuh"
#include "halo.cuh"

#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <map>
#include <algorithm>
#include <type_traits>
#include <array>
#include <cmath>
#include <random>

using namespace sod;

// Error message storage of sod_gpu_last_error() lives in sod2d_gpu.cu.
int sod_detail_set_error(int code, const char *msg);
inline int fail(int code, const std::string &msg) { return sod_detail_set_error(code, msg.c_str()); }

#define CUDA_TRY(call)                                                                    \
  do {                                                                                    \
    cudaError_t _e = (call);                                                              \
    if (_e != cudaSuccess)                                                                \
      return fail(SOD_GPU_ECUDA, std::string(#call) + ": " + cudaGetErrorString(_e));     \
  } while (0)

inline int nat_of(int porder, int ii) { return ii == 0 ? 0 : (ii == 1 ? porder : ii - 1); }

struct sod_gpu_ctx {
  int P = 0, N1 = 0, N = 0, nelem = 0, npoin = 0, npoin_w = 0;
  cudaStream_t stream = 0;
  bool async = false;
  bool mue_set = false;
  Phys ph{};
  sod_phys_t phys{};
  // device mirrors
  int *conn = nullptr, *lpoin_w = nullptr, *slot_ptr = nullptr, *slot_idx = nullptr, *slot_pos = nullptr,
      *lelpn = nullptr;
  int *a_of_t = nullptr;  // tensor position -> reference local node (0-based)
  float *geo = nullptr, *Dnat = nullptr, *invMl = nullptr, *Ml = nullptr, *helem = nullptr, *helem_l_t = nullptr;
  // scratch
  float *slotsA = nullptr, *slotsB = nullptr, *proj12 = nullptr, *mue_t = nullptr, *musgs_t = nullptr;
  unsigned *vbits = nullptr;  // minimum density of the standalone smart_visc_spectral_imex
  int *err_h = nullptr, *err_d = nullptr;  // mapped pinned flag (host / device view) of a device wait that gave up
  size_t bytes = 0;
  std::vector<void *> allocs;
  std::vector<void *> host_allocs;  // pinned host memory
  // analysis / entropy-viscosity support
  int *is_work = nullptr;
  float *Ngp_t = nullptr;  // [g][a] tensor order
  float volT = 0.f;
  // pressure-solve workspace (lazily allocated)
  struct Cg {
    bool ready32 = false, ready64 = false, have_diag = false;
    float *diag = nullptr;                                     // Jacobi diagonal (FP32)
    float *x32, *r32, *p32, *q32, *z032, *z132, *b32;          // reference-arithmetic CG
    double *x, *r, *p, *q, *z0, *z1, *b, *Minv;                // FP64 CG
    double *part, *dots;                                        // reductions
    CgScal *S = nullptr, *S_h = nullptr;                        // device-resident CG scalars (+ pinned host copy)
    double *hist = nullptr, *hist_h = nullptr;                  // ||r||^2 per iteration (ring)
    unsigned *ticket = nullptr;                                 // grid-sum ticket
    unsigned *dticket = nullptr;                                // ticket of k_dot
    double *gpart = nullptr;                                    // grid-sum block partials
  } cg;
  // learned preconditioner
  struct Net {
    bool ready = false, gains_ok = false;
    int nparam = 0, nblk_bwd = 0, step = 0, NP = 0;
    float *params = nullptr, *m1 = nullptr, *m2 = nullptr, *part = nullptr, *grad = nullptr;
    int *pt = nullptr, *pptr = nullptr, *pslot = nullptr;   // patch table [E][NP]; node -> patch-slot CSR
    int *pos = nullptr;                                      // CSR position of each patch slot [E][NP]
    float *feat = nullptr, *gains = nullptr;                  // [E][8], [E][32]
    float *dS = nullptr;  // training scratch: dL/ds per element and mode
    double *Dh = nullptr;                                     // D^-1/2
    float *uf = nullptr;                                      // (float) D^-1/2 r for tensor-core inference
    // harvested (r, e) pairs, FP32, reservoir-sampled, and e^T A e per pair
    int cap = 0, count = 0;
    long long offered = 0;
    uint64_t rs_state = 0x9e3779b97f4a7c15ULL;
    float *hr = nullptr, *he = nullptr;
    std::vector<double> eAe;
    double *xsnap = nullptr;  // solver snapshots (FP64) while harvesting
    double *tmp1 = nullptr, *tmp2 = nullptr;
  } net;
  // incompressible BDF3/EXT3 state (time levels rotate by pointer)
  struct Inc {
    bool ready = false;
    float *u[4] = {nullptr, nullptr, nullptr, nullptr};  // u(:,:,1..4): u^n, new level, u^(n-1), u^(n-2)
    float *Rm[3] = {nullptr, nullptr, nullptr};          // Rmom(:,:,1..3)
    float *div = nullptr, *grad = nullptr, *pf = nullptr, *mu = nullptr;
    double *p = nullptr, *pold = nullptr, *b = nullptr, *x = nullptr;
    double nu = 0.0;
    int nsteps = 0;
    int v_maxiter = 20;  // mod_numerical_params.f90:50-51 defaults
    double v_tol = 1e-4;
    int v_iters = 0;     // statistics of the last velocity solve
    double v_res = 0.0;
    // reference-arithmetic pressure solve and the case's dt / analysis
    float *rhs32 = nullptr, *one = nullptr, *zero = nullptr, *zeroE = nullptr, *part = nullptr;
    double *sums = nullptr;
    unsigned *bits = nullptr;
  } inc;
  // implicit velocity solve (conjGrad_veloc_incomp)
  struct Velo {
    float *tauP = nullptr, *tau_e = nullptr;                   // [npoin][8] projection, [E] tau
    float *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr, *z = nullptr, *z1 = nullptr, *b = nullptr;  // (npoin,3)
  } velo;
  // compressible time-integration state
  struct Comp {
    bool ready = false, fp64 = true, first = true;
    int stages = 5;
    double lam[7][7], gam[7][7];
    float mu_factor = 1.f;
    void *U1[5], *U2[5];  // double or float
    float *rho32, *q32, *E32, *u1, *u2, *eint, *pr, *csound, *machno, *Tem, *eta1, *eta2, *feta, *Reta1, *Reta2,
        *aux, *divU, *vort, *mu_fluid, *tau, *Rmass, *Rmom, *Rener, *part;
    unsigned int *bits;  // [0] min rho, [1] dt, [2] max Mach
    double *sums;        // [3]
  } comp;
  // IMEX integrator scratch (five-variable blocks [mass][energy][momentum])
  struct Imex {
    float *R = nullptr, *D = nullptr;  // [4 stages][5N] explicit / implicit residuals
    float *stab = nullptr, *lvl1 = nullptr, *aux_h = nullptr;
    float *x = nullptr, *r = nullptr, *p = nullptr, *qn = nullptr, *b = nullptr, *z = nullptr, *z1 = nullptr;
    float *au = nullptr, *aT = nullptr, *zmu = nullptr, *zmue = nullptr;  // CG primitives; zero viscosities
    int cg_iters = 0;
    double cg_res = 0.0;
  } imex;
  // halo plan of a partitioned mesh (sod_gpu_set_halo)
  struct Halo {
    bool on = false;
    int rank = 0, nsend = 0, nuniq = 0;
    int *send_node = nullptr;                    // [nsend] local node (0-based) of each buffer position
    int *uniq_node = nullptr, *ptr = nullptr, *src = nullptr;  // shared nodes, rank-ordered contributions
    float *send = nullptr, *recv = nullptr;
    sod_halo_exchange_fn fn = nullptr;
    void *user = nullptr;
    std::vector<void *> own;                     // device arrays of the current plan
    int npoin_o = 0;                             // working nodes this rank owns (dot products):
    int *lpoin_o = nullptr;                      //   shared nodes belong to the lowest rank holding them
    sod_allreduce_fn reduce = nullptr;           // global reductions (sod_gpu_set_allreduce)
    void *reduce_user = nullptr;
    double *vol = nullptr;                       // scratch of the volume sum
  } halo;

  MeshDev md() const {
    MeshDev m;
    m.nelem = nelem; m.npoin = npoin; m.npoin_w = npoin_w;
    m.conn = conn; m.geo = geo; m.Dnat = Dnat; m.lpoin_w = lpoin_w; m.invMl = invMl;
    m.slot_ptr = slot_ptr; m.slot_idx = slot_idx; m.slot_pos = slot_pos;
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
    if (!async) {
      CUDA_TRY(cudaStreamSynchronize(stream));
      return check_waits();
    }
    return 0;
  }
  // A bounded wait inside a kernel that gave up (a bulk copy that never
  // completed) is reported once, at the next synchronisation.
  int check_waits() {
    if (err_h && *(volatile int *)err_h) {
      *(volatile int *)err_h = 0;
      return fail(SOD_GPU_ECUDA, "a bulk copy into shared memory did not complete");
    }
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

// Reference-layout field (nelem, nnode) -> internal [e][t], as a tiled
// transpose: a block takes 32 consecutive elements, reads each node's 32
// values as one coalesced row (the reference layout is element-fastest)
// into shared memory and writes the 32 elements' N values contiguously.
constexpr int E2T_TILE = 32;
constexpr int E2T_THREADS = 256;
__global__ void __launch_bounds__(E2T_THREADS) k_elem_to_t(long long nelem, int N, const int *__restrict__ a_of_t,
                                                           const float *__restrict__ src, float *__restrict__ dst) {
  __shared__ float tile[125][E2T_TILE + 1];  // N <= 125 (P = 4)
  const long long e0 = (long long)blockIdx.x * E2T_TILE;
  const int tx = threadIdx.x % E2T_TILE, ty = threadIdx.x / E2T_TILE;
  constexpr int ROWS = E2T_THREADS / E2T_TILE;
  const long long e = e0 + tx;
  for (int a = ty; a < N; a += ROWS) tile[a][tx] = e < nelem ? src[e + nelem * a] : 0.f;
  __syncthreads();
  const long long ne = nelem - e0 < E2T_TILE ? nelem - e0 : E2T_TILE;
  for (int f = threadIdx.x; f < ne * N; f += E2T_THREADS) {
    const int le = f / N, t = f % N;
    dst[(e0 + le) * N + t] = tile[a_of_t[t]][le];
  }
}

// Internal [e][t] -> reference-layout (nelem, nnode).
__global__ void k_t_to_elem(long long nelem, int N, const int *__restrict__ a_of_t, const float *__restrict__ src,
                            float *__restrict__ dst) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nelem * N) return;
  long long e = idx / N;
  int t = (int)(idx % N);
  dst[e + nelem * a_of_t[t]] = src[idx];
}

// Five Proj arrays (npoin,3) -> node-major [p][12] (tau00 tau01 tau02
// tau11 tau12 tau22 gradRho gradT); the symmetric stress rows ProjMY(:,1),
// ProjMZ(:,1:2) equal ProjMX(:,2:3), ProjMY(:,3).
__global__ void k_pack_proj(long long npoin, const float *PMX, const float *PMY, const float *PMZ,
                            const float *PMass, const float *PEner, float *proj12) {
  long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npoin) return;
  const float r[12] = {PMX[p], PMX[p + npoin], PMX[p + 2 * npoin], PMY[p + npoin], PMY[p + 2 * npoin],
                       PMZ[p + 2 * npoin], PMass[p], PMass[p + npoin], PMass[p + 2 * npoin],
                       PEner[p], PEner[p + npoin], PEner[p + 2 * npoin]};
  float4 *o = reinterpret_cast<float4 *>(proj12 + p * 12);
  for (int c = 0; c < 3; ++c) o[c] = make_float4(r[4 * c], r[4 * c + 1], r[4 * c + 2], r[4 * c + 3]);
}

__global__ void k_unpack_proj(long long npoin, const float *proj12, float *PMX, float *PMY, float *PMZ,
                              float *PMass, float *PEner) {
  long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npoin) return;
  const float *r = proj12 + p * 12;
  PMX[p] = r[0]; PMX[p + npoin] = r[1]; PMX[p + 2 * npoin] = r[2];
  PMY[p] = r[1]; PMY[p + npoin] = r[3]; PMY[p + 2 * npoin] = r[4];
  PMZ[p] = r[2]; PMZ[p + npoin] = r[4]; PMZ[p + 2 * npoin] = r[5];
  PMass[p] = r[6]; PMass[p + npoin] = r[7]; PMass[p + 2 * npoin] = r[8];
  PEner[p] = r[9]; PEner[p + npoin] = r[10]; PEner[p + 2 * npoin] = r[11];
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

inline int num_sms() {
  // initialised once, thread-safely (contexts may be driven from several host threads)
  static const int n = [] {
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v < 1)
      v = 148;
    return v;
  }();
  return n;
}

inline unsigned nblk(long long n, int b) { return (unsigned)((n + b - 1) / b); }

// ---- launch helpers templated on the element order --------------------

template <int P>
struct Launch {
  static constexpr int P_ = P;
  // One element per block (64 threads for P=3, 128 for P=4) for every
  // element kernel but pass A, whose latency-bound gathers do better with
  // two elements per block for P=3 (0.405 against 0.447 ms at 64^3), while
  // pass B and the Laplacian do better with one (0.94 against 1.05 ms).
  static constexpr int EPB = 1;
  static constexpr int TPB = EPB * Cfg<P>::NT;
  static constexpr int EPB_A = (Cfg<P>::NT <= 64) ? 2 : 1;
  static constexpr int TPB_A = EPB_A * Cfg<P>::NT;
  static unsigned grid(int nelem) { return nblk(nelem, EPB); }

  static void proj(sod_gpu_ctx *c, bool prim, const float *a0, const float *a1, const float *a2) {
    if (prim)
      k_proj<P, EPB_A, true><<<nblk(c->nelem, EPB_A), TPB_A, 0, c->stream>>>(c->md(), c->ph, c->phys.Rgas, a0, a1, a2,
                                                                          c->slotsA);
    else
      k_proj<P, EPB_A, false><<<nblk(c->nelem, EPB_A), TPB_A, 0, c->stream>>>(c->md(), c->ph, c->phys.Rgas, a0, a1,
                                                                           a2, c->slotsA);
  }
  // Persistent pass B: as many blocks as fit on the GPU at once (at most
  // one per element group), each walking the groups with a stride.
  template <int MODE, int IN>
  static void rhs(sod_gpu_ctx *c, const RhsArgs &A) {
    using PL = RhsPlan<P, EPB, MODE, IN>;
    static const int per_sm = [] {
      int nb = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_rhs<P, EPB, MODE, IN>, TPB, PL::BYTES) != cudaSuccess ||
          nb < 1)
        nb = 1;
      return nb;
    }();
    const long long groups = grid(c->nelem);
    const unsigned g = (unsigned)std::min<long long>(groups, (long long)per_sm * num_sms());
    RhsArgs Ae = A;
    Ae.err = c->err_d;
    k_rhs<P, EPB, MODE, IN><<<g, TPB, PL::BYTES, c->stream>>>(c->md(), c->ph, c->phys.Rgas, Ae, c->slotsB);
  }
};

template <class F>
inline int dispatch(sod_gpu_ctx *c, F &&f) {
  if (c->P == 3) return f(Launch<3>());
  if (c->P == 4) return f(Launch<4>());
  return fail(SOD_GPU_EINVAL, "unsupported element order");
}

inline void gather_proj_aos(sod_gpu_ctx *c) {
  OutPtrs none{};
  // 128-thread blocks: 1.642-1.650 ms per RHS against 1.660 with 256 (64^3 bench)
  k_gather<12, 12, true><<<nblk(c->npoin, 128), 128, 0, c->stream>>>(c->md(), c->slotsA, c->proj12, none, 0, 1);
}

// Sum the view's components over the ranks that share each node (no-op
// without a halo plan).
template <class T>
inline int halo_sum(sod_gpu_ctx *c, const HaloViewT<T> &v) {
  auto &h = c->halo;
  if (!h.on) return 0;
  static_assert(sizeof(T) % sizeof(float) == 0, "values travel as whole floats");
  if ((int)(v.width * sizeof(T) / sizeof(float)) > HALO_MAX_WIDTH)
    return fail(SOD_GPU_EINVAL, "halo exchange wider than the buffers");
  // the widths the library exchanges get their own instantiation
  auto launch = [&](auto wc, bool pack) {
    constexpr int W = decltype(wc)::value;
    if (pack)
      k_halo_pack<T, W><<<nblk(h.nsend, 256), 256, 0, c->stream>>>(h.nsend, h.send_node, v, (T *)h.send);
    else
      k_halo_sum<T, W><<<nblk(h.nuniq, 128), 128, 0, c->stream>>>(h.nuniq, h.uniq_node, h.ptr, h.src, v,
                                                                  (const T *)h.recv);
  };
  auto by_width = [&](bool pack) {
    switch (v.width) {
      case 12: launch(std::integral_constant<int, 12>{}, pack); break;
      case 6: launch(std::integral_constant<int, 6>{}, pack); break;
      case 5: launch(std::integral_constant<int, 5>{}, pack); break;
      case 3: launch(std::integral_constant<int, 3>{}, pack); break;
      case 1: launch(std::integral_constant<int, 1>{}, pack); break;
      default: launch(std::integral_constant<int, 0>{}, pack); break;
    }
  };
  if (h.nsend > 0) by_width(true);
  CUDA_TRY(cudaGetLastError());
  const int width_floats = v.width * (int)(sizeof(T) / sizeof(float));
  if (h.fn(h.user, h.send, h.recv, width_floats, (void *)c->stream) != 0)
    return fail(SOD_GPU_EINVAL, "halo exchange callback failed");
  if (h.nuniq > 0) by_width(false);
  CUDA_TRY(cudaGetLastError());
  return 0;
}

inline HaloView halo_proj_view(sod_gpu_ctx *c) {
  HaloView v{};
  v.width = 12;
  v.nstride = 12;
  for (int k = 0; k < 12; ++k) v.comp[k] = c->proj12 + k;
  return v;
}

inline HaloView halo_res_view(sod_gpu_ctx *c, float *Rmass, float *Rmom, float *Rener) {
  HaloView v{};
  const long long N = c->npoin;
  v.width = 5;
  v.nstride = 1;
  v.comp[0] = Rmass; v.comp[1] = Rener; v.comp[2] = Rmom; v.comp[3] = Rmom + N; v.comp[4] = Rmom + 2 * N;
  return v;
}

// View of ncomp reference-layout components (npoin each) of one array.
inline HaloView halo_soa_view(sod_gpu_ctx *c, float *a, int ncomp) {
  HaloView v{};
  v.width = ncomp;
  v.nstride = 1;
  for (int k = 0; k < ncomp; ++k) v.comp[k] = a + (long long)k * c->npoin;
  return v;
}

// In-place global reduction of a device buffer (no-op without a callback).
inline int allreduce(sod_gpu_ctx *c, void *buf, int count, int kind) {
  auto &h = c->halo;
  if (!h.reduce) return 0;
  CUDA_TRY(cudaGetLastError());
  if (h.reduce(h.reduce_user, buf, count, kind, (void *)c->stream) != 0)
    return fail(SOD_GPU_EINVAL, "allreduce callback failed");
  return 0;
}

// Entry points whose solves need global dot products refuse a partitioned mesh.
inline int no_partition(sod_gpu_ctx *c, const char *what) {
  if (c && c->halo.on) return fail(SOD_GPU_EINVAL, std::string(what) + " is not available with a halo plan");
  return 0;
}

inline void gather_res(sod_gpu_ctx *c, float *Rmass, float *Rmom, float *Rener, int accumulate, int invml) {
  OutPtrs o{};
  const long long N = c->npoin;
  o.p[0] = Rmass; o.p[1] = Rener; o.p[2] = Rmom; o.p[3] = Rmom + N; o.p[4] = Rmom + 2 * N;
  k_gather_sorted_res5<<<nblk(c->npoin, 128), 128, 0, c->stream>>>(c->md(), c->slotsB, (long long)c->nelem * c->N,
                                                                    o, accumulate, invml);
}

}  // namespace
