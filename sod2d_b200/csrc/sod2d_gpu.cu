// C-ABI entry points of the B200 spectral-element RHS library
// (declarations and contracts: include/sod2d_gpu.h).
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

// Records an error message for sod_gpu_last_error() from other translation
// units of the library.
int sod_detail_set_error(int code, const char *msg) { return fail(code, msg); }

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
    int nparam = 0, nblk_bwd = 148, step = 0, NP = 0;
    float *params = nullptr, *m1 = nullptr, *m2 = nullptr, *part = nullptr, *grad = nullptr;
    int *pt = nullptr, *pptr = nullptr, *pslot = nullptr;   // patch table [E][NP]; node -> patch-slot CSR
    int *pos = nullptr;                                      // CSR position of each patch slot [E][NP]
    float *feat = nullptr, *gains = nullptr;                  // [E][8], [E][32]
    float *X = nullptr, *W = nullptr, *Y = nullptr, *SA = nullptr, *dS = nullptr;  // training scratch
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

int num_sms() {
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
  static constexpr int EPB = (Cfg<P>::NT <= 64) ? 2 : 1;
  static constexpr int TPB = EPB * Cfg<P>::NT;
  static unsigned grid(int nelem) { return nblk(nelem, EPB); }

  static void proj(sod_gpu_ctx *c, bool prim, const float *a0, const float *a1, const float *a2) {
    if (prim)
      k_proj<P, EPB, true><<<grid(c->nelem), TPB, 0, c->stream>>>(c->md(), c->ph, c->phys.Rgas, a0, a1, a2, c->slotsA);
    else
      k_proj<P, EPB, false><<<grid(c->nelem), TPB, 0, c->stream>>>(c->md(), c->ph, c->phys.Rgas, a0, a1, a2, c->slotsA);
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
    k_rhs<P, EPB, MODE, IN><<<g, TPB, PL::BYTES, c->stream>>>(c->md(), c->ph, c->phys.Rgas, A, c->slotsB);
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
  k_gather<12, 12, true><<<nblk(c->npoin, 256), 256, 0, c->stream>>>(c->md(), c->slotsA, c->proj12, none, 0, 1);
}

// Sum the view's components over the ranks that share each node (no-op
// without a halo plan).
template <class T>
int halo_sum(sod_gpu_ctx *c, const HaloViewT<T> &v) {
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

HaloView halo_proj_view(sod_gpu_ctx *c) {
  HaloView v{};
  v.width = 12;
  v.nstride = 12;
  for (int k = 0; k < 12; ++k) v.comp[k] = c->proj12 + k;
  return v;
}

HaloView halo_res_view(sod_gpu_ctx *c, float *Rmass, float *Rmom, float *Rener) {
  HaloView v{};
  const long long N = c->npoin;
  v.width = 5;
  v.nstride = 1;
  v.comp[0] = Rmass; v.comp[1] = Rener; v.comp[2] = Rmom; v.comp[3] = Rmom + N; v.comp[4] = Rmom + 2 * N;
  return v;
}

// View of ncomp reference-layout components (npoin each) of one array.
HaloView halo_soa_view(sod_gpu_ctx *c, float *a, int ncomp) {
  HaloView v{};
  v.width = ncomp;
  v.nstride = 1;
  for (int k = 0; k < ncomp; ++k) v.comp[k] = a + (long long)k * c->npoin;
  return v;
}

// In-place global reduction of a device buffer (no-op without a callback).
int allreduce(sod_gpu_ctx *c, void *buf, int count, int kind) {
  auto &h = c->halo;
  if (!h.reduce) return 0;
  CUDA_TRY(cudaGetLastError());
  if (h.reduce(h.reduce_user, buf, count, kind, (void *)c->stream) != 0)
    return fail(SOD_GPU_EINVAL, "allreduce callback failed");
  return 0;
}

// Entry points whose solves need global dot products refuse a partitioned mesh.
int no_partition(sod_gpu_ctx *c, const char *what) {
  if (c && c->halo.on) return fail(SOD_GPU_EINVAL, std::string(what) + " is not available with a halo plan");
  return 0;
}

void gather_res(sod_gpu_ctx *c, float *Rmass, float *Rmom, float *Rener, int accumulate, int invml) {
  OutPtrs o{};
  const long long N = c->npoin;
  o.p[0] = Rmass; o.p[1] = Rener; o.p[2] = Rmom; o.p[3] = Rmom + N; o.p[4] = Rmom + 2 * N;
  k_gather_sorted_res5<<<nblk(c->npoin, 256), 256, 0, c->stream>>>(c->md(), c->slotsB, (long long)c->nelem * c->N,
                                                                    o, accumulate, invml);
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
  return 0;
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
  const long long EN = (long long)c->nelem * c->N;
  k_elem_to_t<<<nblk(c->nelem, E2T_TILE), E2T_THREADS, 0, c->stream>>>(c->nelem, c->N, c->a_of_t, mu_e, c->mue_t);
  if (mu_sgs) {
    if (!c->musgs_t) {
      int rc = c->alloc(&c->musgs_t, (size_t)EN);
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
  const long long EN = (long long)c->nelem * c->N;
  k_elem_to_t<<<nblk(c->nelem, E2T_TILE), E2T_THREADS, 0, c->stream>>>(c->nelem, c->N, c->a_of_t, mu_e, c->mue_t);
  if (mu_sgs) {
    if (!c->musgs_t) {
      int rc = c->alloc(&c->musgs_t, (size_t)EN);
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
  const long long EN = (long long)c->nelem * c->N;
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
  const long long EN = (long long)c->nelem * c->N;
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

// ---- incompressible operators and pressure CG ---------------------------

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
void lap(sod_gpu_ctx *c, const V *p, V *out) {
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
void dots(sod_gpu_ctx *c, DotArgs<V, ND> A, double *out) {
  const bool part = c->halo.on;
  k_dot<V, ND><<<DOT_BLOCKS, DOT_THREADS, 0, c->stream>>>(part ? c->halo.npoin_o : c->npoin_w,
                                                          part ? c->halo.lpoin_o : c->lpoin_w, A, c->cg.part,
                                                          c->cg.dticket, out);
}

int ensure_diag(sod_gpu_ctx *c) {
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

int ensure_cg32(sod_gpu_ctx *c) {
  auto &G = c->cg;
  if (G.ready32) return 0;
  int rc;
  for (float **pp : {&G.x32, &G.r32, &G.p32, &G.q32, &G.z032, &G.z132, &G.b32})
    if ((rc = c->alloc(pp, (size_t)c->npoin))) return rc;
  G.ready32 = true;
  return 0;
}

int ensure_cg64(sod_gpu_ctx *c) {
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
unsigned tc_grid(long long nelem) {
  const long long groups = (nelem + 15) / 16;
  return (unsigned)std::min<long long>(std::max<long long>(groups, 1), num_sms());
}
constexpr int TC_THREADS = TcDims<3>::WARPS * 32;
static_assert(TcDims<3>::WARPS == TcDims<4>::WARPS, "one block size for both orders");

int ensure_cg_loop(sod_gpu_ctx *c) {
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

}  // namespace

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

int apply_precond(sod_gpu_ctx *c, int kind, const double *r, double *z);  // defined with the network
int ensure_gains(sod_gpu_ctx *c);

__global__ void k_d2f_w(int npoin_w, const int *__restrict__ lpoin_w, const double *__restrict__ a,
                        float *__restrict__ b);

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

__global__ void k_jacobi64(int npoin_w, const int *__restrict__ lpoin_w, const double *__restrict__ Minv,
                           const double *__restrict__ r, double *__restrict__ z) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const int i = lpoin_w[t];
  z[i] = r[i] * Minv[i];
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

namespace {

int ensure_gains(sod_gpu_ctx *c);

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

}  // namespace

extern "C" {
}  // extern "C"

// ---- compressible time integration --------------------------------------

namespace {

int rk_coeffs(int S, int n, double lam[7][7], double gam[7][7]) {
  for (int i = 0; i < 7; ++i)
    for (int j = 0; j < 7; ++j) { lam[i][j] = 0.0; gam[i][j] = 0.0; }
  // time_integ_ls.f90:87-167, 1-based indices
  if (S == 3) {
    lam[2][1] = 1.0; lam[3][1] = 3.0 / 4.0; lam[3][2] = 1.0 / 4.0; lam[4][1] = 1.0 / 3.0; lam[4][3] = 2.0 / 3.0;
    gam[2][1] = 1.0; gam[3][2] = 0.25; gam[4][3] = 2.0 / 3.0;
  } else if (S == 4) {
    lam[2][1] = 1.0; lam[3][2] = 1.0; lam[4][1] = 2.0 / 3.0; lam[4][3] = 1.0 / 3.0; lam[5][4] = 1.0;
    gam[2][1] = 0.5; gam[3][2] = 0.5; gam[4][3] = 1.0 / 6.0; gam[5][4] = 0.5;
  } else if (S == 5) {
    lam[2][1] = lam[3][2] = lam[4][3] = lam[5][4] = lam[6][5] = 1.0;
    if (n == 1) {
      lam[5][1] = 0.571403511494104; lam[5][4] = 0.428596488505896;
      gam[2][1] = 0.443568244942995; gam[3][2] = 0.291111420073766; gam[4][3] = 0.270612601278217;
      gam[5][4] = 0.110577759392786; gam[6][5] = 0.458557505351052;
    } else if (n == 2) {
      lam[4][1] = 0.682342861037239; lam[4][3] = 0.317657138962761; lam[6][1] = 0.045230974482400;
      lam[6][5] = 0.954769025517600;
      gam[2][1] = 0.465388589249323; gam[3][2] = 0.465388589249323; gam[4][3] = 0.124745797313998;
      gam[5][4] = 0.465388589249323; gam[6][5] = 0.154263303748666;
    } else if (n == 3) {
      lam[5][1] = 0.592032910942121; lam[5][4] = 1.0 - lam[5][1];
      gam[2][1] = 0.266541020678955; gam[3][2] = 0.548560709048532; gam[4][3] = 0.289517014154401;
      gam[5][4] = 0.086408328057923; gam[6][5] = 0.462943578481813;
    } else if (n == 4) {
      lam[4][1] = 0.707858560931430; lam[4][3] = 1.0 - lam[4][1]; lam[6][1] = 0.222853615080669;
      lam[6][5] = 1.0 - lam[6][1];
      gam[2][1] = 0.292845746913355; gam[3][2] = 0.339532793976408; gam[4][3] = 0.200532330324672;
      gam[5][4] = 0.701676169006879; gam[6][5] = 0.155278812461877;
    } else {
      return -1;
    }
  } else {
    return -1;
  }
  return 0;
}

// The FP32 reference rounds its RK coefficients to real(rp): mirror that.
inline double as_rp(double v, bool fp64) { return fp64 ? v : (double)(float)v; }

template <class T>
void launch_stage(sod_gpu_ctx *c, double l1, double li, double gdt, int first) {
  auto &S = c->comp;
  State5<T> U1, U2;
  for (int f = 0; f < 5; ++f) { U1.f[f] = (T *)S.U1[f]; U2.f[f] = (T *)S.U2[f]; }
  k_stage<T><<<nblk(c->npoin_w, 256), 256, 0, c->stream>>>(c->npoin_w, c->npoin, c->lpoin_w, U1, U2, S.Rmass,
                                                           S.Rmom, S.Rener, (T)l1, (T)li, (T)gdt, first, S.rho32,
                                                           S.q32, S.E32);
}

// RHS at the current FP32 shadow state into comp.R* (updateF body).
int comp_updateF(sod_gpu_ctx *c) {
  auto &S = c->comp;
  RhsArgs A{};
  A.rho = S.rho32; A.q = S.q32; A.E = S.E32; A.mu_factor = S.mu_factor;
  A.mue_t = c->mue_t; A.tau_stab = S.tau; A.proj12 = c->proj12;
  A.fact_c = -1.0f; A.fact_d = -1.0f;
  int rc = dispatch(c, [&](auto L) {
    L.proj(c, false, S.rho32, S.q32, S.E32);
    gather_proj_aos(c);
    int hrc = halo_sum(c, halo_proj_view(c));
    if (hrc) return hrc;
    L.template rhs<MODE_CONV | MODE_DIFF, IN_CONS>(c, A);
    return 0;
  });
  if (rc) return rc;
  gather_res(c, S.Rmass, S.Rmom, S.Rener, 0, 1);
  return halo_sum(c, halo_res_view(c, S.Rmass, S.Rmom, S.Rener));
}

// Entropy residual (+ divergence and vorticity when dc) of (feta, eta1, u1[, u2]).
int comp_entropy_pass(sod_gpu_ctx *c, float *Reta_out, bool dc) {
  auto &S = c->comp;
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    constexpr int P = LL::P_;
    if (dc)
      k_entropy_elem<P, LL::EPB, true><<<LL::grid(c->nelem), LL::TPB, 0, c->stream>>>(c->md(), S.feta, S.eta1, S.u1,
                                                                                     S.u2, c->slotsB);
    else
      k_entropy_elem<P, LL::EPB, false><<<LL::grid(c->nelem), LL::TPB, 0, c->stream>>>(c->md(), S.feta, S.eta1, S.u1,
                                                                                      S.u2, c->slotsB);
    return 0;
  });
  k_gather_entropy<<<nblk(c->npoin, 256), 256, 0, c->stream>>>(c->md(), c->slotsB, c->lelpn, c->is_work, Reta_out,
                                                               S.divU, S.vort, dc ? 1 : 0);
  // halo sums of the lumped entropy residual (time_integ_ls.f90:287, :431),
  // the divergence and the vorticity (mod_operators.f90:566, :759)
  HaloView v{};
  const long long N = c->npoin;
  v.nstride = 1;
  v.width = dc ? 5 : 1;
  v.comp[0] = Reta_out;
  if (dc) { v.comp[1] = S.divU; v.comp[2] = S.vort; v.comp[3] = S.vort + N; v.comp[4] = S.vort + 2 * N; }
  return halo_sum(c, v);
}

int comp_visc(sod_gpu_ctx *c, const float *Reta, const float *rho, const float *u, bool ducros) {
  auto &S = c->comp;
  const unsigned init_bits = 0x47C35000u;  // 100000.0f
  CUDA_TRY(cudaMemcpyAsync(S.bits, &init_bits, sizeof(unsigned), cudaMemcpyHostToDevice, c->stream));
  k_min_rho<<<MINMAX_BLOCKS, 256, 0, c->stream>>>(c->npoin_w, c->lpoin_w, rho, S.bits);
  // the bits of a positive float order like the float: reduce as float
  int rc = allreduce(c, S.bits, 1, SOD_REDUCE_MIN_F32);
  if (rc) return rc;
  ViscArgs V{};
  V.Reta = Reta; V.rho = rho; V.u = u; V.csound = S.csound; V.divU = S.divU; V.vort = S.vort; V.Ml = c->Ml;
  V.helem = c->helem; V.helem_l_t = c->helem_l_t; V.min_rho_bits = S.bits;
  V.ce = c->phys.ce; V.cmax = c->phys.cmax; V.cglob = c->phys.cglob; V.ducros_min = c->phys.ducros_min_val;
  V.inv_p = 1.0f / (float)c->P; V.ducros = ducros ? 1 : 0;
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    k_visc<LL::P_><<<nblk(c->nelem, 8), 256, 0, c->stream>>>(c->md(), V, c->a_of_t, c->mue_t, nullptr);
    return 0;
  });
  return 0;
}

}  // namespace

extern "C" {

int sod_gpu_generic_scalar_convec_ijk(sod_gpu_ctx *c, const float *q, const float *eta, const float *u, float *R,
                                      int initialze, float fact) {
  if (!c || !q || !eta || !u || !R) return fail(SOD_GPU_EINVAL, "bad argument");
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    k_entropy_elem<LL::P_, LL::EPB, false><<<LL::grid(c->nelem), LL::TPB, 0, c->stream>>>(c->md(), q, eta, u,
                                                                                        nullptr, c->slotsB, fact);
    return 0;
  });
  OutPtrs o{};
  o.p[0] = R;
  k_gather<8, 1, false><<<nblk(c->npoin, 256), 256, 0, c->stream>>>(c->md(), c->slotsB, nullptr, o,
                                                                     initialze ? 0 : 1, 0);
  return c->finish();
}

int sod_gpu_smart_visc_spectral_imex(sod_gpu_ctx *c, const float *Reta, const float *rho, const float *u,
                                     const float *csound, float *mu_e) {
  if (!c || !Reta || !rho || !u || !csound || !mu_e) return fail(SOD_GPU_EINVAL, "bad argument");
  if (!c->helem) return fail(SOD_GPU_EINVAL, "smart_visc_spectral_imex needs helem at init");
  int rc;
  if (!c->vbits && (rc = c->alloc(&c->vbits, 4))) return rc;
  const unsigned init_bits = 0x47C35000u;  // 100000.0f, the reference's initial minimum
  CUDA_TRY(cudaMemcpyAsync(c->vbits, &init_bits, sizeof(unsigned), cudaMemcpyHostToDevice, c->stream));
  k_min_rho<<<MINMAX_BLOCKS, 256, 0, c->stream>>>(c->npoin_w, c->lpoin_w, rho, c->vbits);
  if ((rc = allreduce(c, c->vbits, 1, SOD_REDUCE_MIN_F32))) return rc;
  ViscArgs V{};
  V.Reta = Reta; V.rho = rho; V.u = u; V.csound = csound; V.Ml = c->Ml;
  V.helem = c->helem; V.helem_l_t = c->helem_l_t; V.min_rho_bits = c->vbits;
  V.ce = c->phys.ce; V.cmax = c->phys.cmax; V.cglob = c->phys.cglob; V.ducros_min = c->phys.ducros_min_val;
  V.inv_p = 1.0f / (float)c->P; V.ducros = 0;
  // the element-layout copy goes to scratch: the context's own mu_e is left alone
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    k_visc<LL::P_><<<nblk(c->nelem, 8), 256, 0, c->stream>>>(c->md(), V, c->a_of_t, c->slotsA, mu_e);
    return 0;
  });
  return c->finish();
}

int sod_gpu_ducros_visc_limit(sod_gpu_ctx *c, const float *rho, const float *u, const float *divU,
                              const float *vorti, const float *csound, float *mu_e) {
  if (!c || !rho || !u || !divU || !vorti || !csound || !mu_e) return fail(SOD_GPU_EINVAL, "bad argument");
  if (!c->helem_l_t) return fail(SOD_GPU_EINVAL, "ducros_visc_limit needs helem_l at init");
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    k_ducros<LL::P_><<<nblk(c->nelem, 8), 256, 0, c->stream>>>(c->md(), u, divU, vorti, c->Ml, c->helem_l_t,
                                                               c->phys.ducros_min_val, c->a_of_t, mu_e);
    return 0;
  });
  return c->finish();
}

int sod_gpu_rk_ls_stage(sod_gpu_ctx *c, int first, float lam1, float lami, float gam, float dt, const float *rho1,
                        const float *q1, const float *E1, float *rho2, float *q2, float *E2, const float *Rmass,
                        const float *Rmom, const float *Rener) {
  if (!c || !rho2 || !q2 || !E2 || !Rmass || !Rmom || !Rener || (!first && (!rho1 || !q1 || !E1)))
    return fail(SOD_GPU_EINVAL, "bad argument");
  k_ls_stage_ref<<<nblk(c->npoin_w, 256), 256, 0, c->stream>>>(c->npoin_w, c->npoin, c->lpoin_w, first ? 1 : 0, lam1,
                                                               lami, gam, dt, rho1, q1, E1, rho2, q2, E2, Rmass,
                                                               Rmom, Rener);
  return c->finish();
}

int sod_gpu_comp_init_state(sod_gpu_ctx *c, const sod_rk_cfg_t *cfg, const float *rho, const float *u,
                            const float *q, const float *pr, const float *E, const float *Tem, const float *csound,
                            const float *machno, const float *eta) {
  if (!c || !cfg || !rho || !u || !q || !pr || !E || !Tem || !csound || !machno || !eta)
    return fail(SOD_GPU_EINVAL, "bad argument");
  if (!c->helem || !c->helem_l_t || !c->lelpn) return fail(SOD_GPU_EINVAL, "time integration needs helem, helem_l and lelpn at init");
  auto &S = c->comp;
  if (rk_coeffs(cfg->stages, cfg->rk_n, S.lam, S.gam)) return fail(SOD_GPU_EINVAL, "unsupported RK scheme");
  const size_t N = c->npoin, NE = (size_t)c->nelem;
  int rc = 0;
  if (!S.ready) {
    const size_t tb = cfg->fp64_state ? sizeof(double) : sizeof(float);
    for (int f = 0; f < 5; ++f) {
      char *p1, *p2;
      if ((rc = c->alloc(&p1, N * tb)) || (rc = c->alloc(&p2, N * tb))) return rc;
      S.U1[f] = p1; S.U2[f] = p2;
    }
    float **f1[] = {&S.rho32, &S.E32, &S.eint, &S.pr, &S.csound, &S.machno, &S.Tem, &S.eta1, &S.eta2,
                    &S.Reta1, &S.Reta2, &S.aux, &S.divU, &S.mu_fluid, &S.Rmass, &S.Rener};
    for (auto pp : f1)
      if ((rc = c->alloc(pp, N))) return rc;
    float **f3[] = {&S.q32, &S.u1, &S.u2, &S.feta, &S.vort, &S.Rmom};
    for (auto pp : f3)
      if ((rc = c->alloc(pp, 3 * N))) return rc;
    if ((rc = c->alloc(&S.tau, NE)) || (rc = c->alloc(&S.part, 3 * NE)) || (rc = c->alloc(&S.bits, 4)) ||
        (rc = c->alloc(&S.sums, 4)))
      return rc;
    S.ready = true;
    S.fp64 = cfg->fp64_state != 0;
  } else if ((cfg->fp64_state != 0) != S.fp64) {
    return fail(SOD_GPU_EINVAL, "state precision cannot change after the first init");
  }
  S.stages = cfg->stages;
  S.mu_factor = cfg->mu_factor;
  S.first = true;
  const cudaStream_t st = c->stream;
  CUDA_TRY(cudaMemcpyAsync(S.rho32, rho, N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(S.q32, q, 3 * N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(S.E32, E, N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(S.u2, u, 3 * N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(S.pr, pr, N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(S.Tem, Tem, N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(S.csound, csound, N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(S.machno, machno, N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(S.eta2, eta, N * 4, cudaMemcpyDeviceToDevice, st));
  for (float *z : {S.Reta1, S.Reta2, S.Rmass, S.Rener, S.divU, S.aux})
    CUDA_TRY(cudaMemsetAsync(z, 0, N * 4, st));
  CUDA_TRY(cudaMemsetAsync(S.Rmom, 0, 3 * N * 4, st));
  CUDA_TRY(cudaMemsetAsync(S.vort, 0, 3 * N * 4, st));
  CUDA_TRY(cudaMemsetAsync(c->mue_t, 0, NE * c->N * 4, st));
  c->mue_set = true;
  // FP64 (or FP32) master state from the FP32 initial arrays
  {
    const float *src[5] = {rho, q, q + N, q + 2 * N, E};
    std::vector<float> h(N);
    for (int f = 0; f < 5; ++f) {
      CUDA_TRY(cudaMemcpyAsync(h.data(), src[f], N * 4, cudaMemcpyDeviceToHost, st));
      CUDA_TRY(cudaStreamSynchronize(st));
      if (S.fp64) {
        std::vector<double> d(h.begin(), h.end());
        CUDA_TRY(cudaMemcpy(S.U2[f], d.data(), N * 8, cudaMemcpyHostToDevice));
      } else {
        CUDA_TRY(cudaMemcpy(S.U2[f], h.data(), N * 4, cudaMemcpyHostToDevice));
      }
    }
  }
  k_sutherland<<<nblk(c->npoin_w, 256), 256, 0, st>>>(c->npoin_w, c->lpoin_w, S.mu_factor, S.Tem, S.mu_fluid);
  return c->finish();
}

int sod_gpu_comp_rk_ls_step(sod_gpu_ctx *c, float dt) {
  if (!c || !c->comp.ready) return fail(SOD_GPU_EINVAL, "state not initialised");
  if (!(dt > 0.f)) return fail(SOD_GPU_EINVAL, "dt must be positive");
  auto &S = c->comp;
  const cudaStream_t st = c->stream;
  const size_t N = c->npoin;
  const size_t tb = S.fp64 ? 8 : 4;
  // level 1 <- level 2 (CFDSolverBase.f90:1951-1960)
  for (int f = 0; f < 5; ++f) CUDA_TRY(cudaMemcpyAsync(S.U1[f], S.U2[f], N * tb, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(S.u1, S.u2, 3 * N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(S.eta1, S.eta2, N * 4, cudaMemcpyDeviceToDevice, st));
  // tau from level 2 (comp_tau)
  k_comp_tau<<<nblk(c->nelem, 8), 256, 0, st>>>(c->nelem, c->N, c->conn, c->helem, S.csound, S.u2, c->npoin,
                                                c->phys.c_species_stab / (float)c->P, S.tau);
  if (S.first) {
    S.first = false;
    k_feta<<<nblk(c->npoin_w, 256), 256, 0, st>>>(c->npoin_w, c->npoin, c->lpoin_w, S.u1, S.eta1, S.feta);
    int rc;
    if ((rc = comp_entropy_pass(c, S.Reta1, false)) || (rc = comp_visc(c, S.Reta1, S.rho32, S.u1, false)) ||
        (rc = comp_updateF(c)))
      return rc;
  }
  const double dtd = (double)dt;
  auto stage = [&](double l1, double li, double g, int first) {
    const double gdt = S.fp64 ? g * dtd : (double)((float)g * dt);
    if (S.fp64)
      launch_stage<double>(c, l1, li, gdt, first);
    else
      launch_stage<float>(c, as_rp(l1, false), as_rp(li, false), gdt, first);
  };
  stage(0.0, 0.0, as_rp(S.gam[2][1], S.fp64), 1);
  for (int i = 2; i <= S.stages; ++i) {
    int rc = comp_updateF(c);
    if (rc) return rc;
    stage(as_rp(S.lam[i + 1][1], S.fp64), as_rp(S.lam[i + 1][i], S.fp64), as_rp(S.gam[i + 1][i], S.fp64), 0);
  }
  const float gm = c->phys.gamma_gas;
  k_eos_end<<<nblk(c->npoin_w, 256), 256, 0, st>>>(c->npoin_w, c->npoin, c->lpoin_w, gm - 1.0f, gm, c->phys.Rgas,
                                                   S.rho32, S.q32, S.E32, S.u2, S.eint, S.pr, S.csound, S.machno,
                                                   S.Tem);
  k_thermo_entropy<<<nblk(c->npoin_w, 256), 256, 0, st>>>(c->npoin_w, c->npoin, c->lpoin_w, gm, c->phys.p_inf,
                                                          c->phys.rho_inf, S.rho32, S.pr, S.u1, S.eta1, S.eta2,
                                                          S.feta);
  int rc = comp_entropy_pass(c, S.Reta2, true);
  if (rc) return rc;
  k_aux_reta<<<nblk(c->npoin_w, 256), 256, 0, st>>>(c->npoin_w, c->lpoin_w, dt, S.Reta1, S.Reta2, S.eta1, S.eta2,
                                                    S.aux);
  if ((rc = comp_visc(c, S.aux, S.rho32, S.u2, true))) return rc;
  k_sutherland<<<nblk(c->npoin_w, 256), 256, 0, st>>>(c->npoin_w, c->lpoin_w, S.mu_factor, S.Tem, S.mu_fluid);
  return c->finish();
}

}  // extern "C"

// ---- IMEX time step (imex_main) ------------------------------------------

namespace {

int ensure_imex(sod_gpu_ctx *c) {
  auto &X = c->imex;
  if (X.R) return 0;
  const size_t N = c->npoin, EN = (size_t)c->nelem * c->N;
  int rc;
  if ((rc = c->alloc(&X.R, 4 * 5 * N)) || (rc = c->alloc(&X.D, 4 * 5 * N)) || (rc = c->alloc(&X.stab, 5 * N)) ||
      (rc = c->alloc(&X.lvl1, 5 * N)) || (rc = c->alloc(&X.aux_h, N)) || (rc = c->alloc(&X.x, 5 * N)) ||
      (rc = c->alloc(&X.r, 5 * N)) || (rc = c->alloc(&X.p, 5 * N)) || (rc = c->alloc(&X.qn, 5 * N)) ||
      (rc = c->alloc(&X.b, 5 * N)) || (rc = c->alloc(&X.z, 5 * N)) || (rc = c->alloc(&X.z1, 5 * N)) ||
      (rc = c->alloc(&X.au, 3 * N)) || (rc = c->alloc(&X.aT, N)) || (rc = c->alloc(&X.zmu, N)) ||
      (rc = c->alloc(&X.zmue, EN)))
    return rc;
  if (!c->cg.part && ((rc = c->alloc(&c->cg.part, 8 * DOT_BLOCKS)) || (rc = c->alloc(&c->cg.dots, 16)))) return rc;
  for (float *v : {X.R, X.D}) CUDA_TRY(cudaMemsetAsync(v, 0, 4 * 5 * N * 4, c->stream));
  for (float *v : {X.stab, X.x, X.r, X.p, X.qn, X.b, X.z, X.z1}) CUDA_TRY(cudaMemsetAsync(v, 0, 5 * N * 4, c->stream));
  CUDA_TRY(cudaMemsetAsync(X.au, 0, 3 * N * 4, c->stream));
  for (float *v : {X.aT, X.zmu, X.aux_h}) CUDA_TRY(cudaMemsetAsync(v, 0, N * 4, c->stream));
  CUDA_TRY(cudaMemsetAsync(X.zmue, 0, EN * 4, c->stream));
  return 0;
}

// Butcher tables of init_imex_solver, time_integ_imex.f90:42-158, rounded
// to FP32 as the reference's real(rp) constants
ImexCoef imex_coef(int S) {
  ImexCoef k{};
  if (S == 4) {
    const float bi1 = 4.0f / 15.0f, bi2 = 1.0f / 3.0f, bi3 = 7.0f / 30.0f, bi4 = 1.0f / 6.0f;
    const float be1 = 1.0f / 4.0f, be2 = 0.0f, be3 = 3.0f / 4.0f, be4 = 0.0f;
    k.ai[2][1] = bi1; k.ai[2][2] = bi1;
    k.ai[3][1] = bi1; k.ai[3][2] = bi2; k.ai[3][3] = 1.0f / 15.0f;
    k.ai[4][1] = bi1; k.ai[4][2] = bi2; k.ai[4][3] = bi3; k.ai[4][4] = bi4;
    k.ae[2][1] = 8.0f / 15.0f;
    k.ae[3][1] = be1; k.ae[3][2] = 5.0f / 12.0f;
    k.ae[4][1] = be1; k.ae[4][2] = be2; k.ae[4][3] = be3; k.ae[4][4] = be4;
  } else {
    k.ai[2][1] = (float)0.353842865099275; k.ai[2][2] = (float)0.353842865099275;
    k.ai[3][1] = (float)0.398930808264689; k.ai[3][2] = (float)0.345755244189622;
    k.ai[3][3] = (float)0.255313947545689;
    k.ae[2][1] = (float)0.711664700366941;
    k.ae[3][1] = (float)0.077338168947683; k.ae[3][2] = (float)0.917273367886007;
  }
  return k;
}

// explicit convection (fact +1) of a stage state into a five-variable block
// Halo sum of a five-variable block [mass][energy][mom x][mom y][mom z].
int halo_block5(sod_gpu_ctx *c, float *out) {
  HaloView v{};
  const long long N = c->npoin;
  v.width = 5;
  v.nstride = 1;
  for (int k = 0; k < 5; ++k) v.comp[k] = out + k * N;
  return halo_sum(c, v);
}

int imex_convec(sod_gpu_ctx *c, const float *rho, const float *u, const float *q, const float *pr, const float *h,
                float *out) {
  RhsArgs A{};
  A.rho = rho; A.u = u; A.q = q; A.pr = pr; A.E = h; A.fact_c = 1.0f;
  dispatch(c, [&](auto L) {
    L.template rhs<MODE_CONV, IN_PRIM>(c, A);
    return 0;
  });
  const long long N = c->npoin;
  gather_res(c, out, out + 2 * N, out + N, 0, 0);
  return halo_block5(c, out);
}

// diffusion without LPS (fact +1) into a five-variable block; rho_n null: rho
int imex_diffusion(sod_gpu_ctx *c, const float *rho_n, const float *rho, const float *u, const float *Tem,
                    float *out) {
  auto &S = c->comp;
  RhsArgs A{};
  A.rho = rho; A.rho_n = rho_n; A.u = u; A.Tem = Tem; A.mu_fluid = S.mu_fluid; A.mue_t = c->mue_t;
  A.musgs_t = nullptr; A.fact_d = 1.0f;
  dispatch(c, [&](auto L) {
    L.template rhs<MODE_DIFF | MODE_NOLPS, IN_DIFF>(c, A);
    return 0;
  });
  const long long N = c->npoin;
  gather_res(c, out, out + 2 * N, out + N, 0, 0);
  return halo_block5(c, out);  // mod_solver_imex.f90:123, :196 (operator); time_integ_imex.f90:382 (stages)
}

// FP64 sum over the working nodes and the five variables of a (b - c)
double imex_dot(sod_gpu_ctx *c, const float *a, const float *b, const float *cc, int *rc) {
  const long long N = c->npoin;
  DotArgs<float, 5> A{};
  for (int k = 0; k < 5; ++k) {
    A.a[k] = a + N * k; A.b[k] = b + N * k; A.c[k] = cc ? cc + N * k : nullptr;
  }
  dots<float, 5>(c, A, c->cg.dots + 8);
  if ((*rc = allreduce(c, c->cg.dots + 8, 5, SOD_REDUCE_SUM_F64))) return 0.0;  // mod_solver_imex.f90:181, 225
  double t[5] = {0, 0, 0, 0, 0};
  if (cudaMemcpyAsync(t, c->cg.dots + 8, 40, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess) {
    *rc = fail(SOD_GPU_ECUDA, "dot product of the IMEX solve failed");
    return 0.0;
  }
  return (((t[0] + t[1]) + t[2]) + t[3]) + t[4];
}

// conjGrad_imex, mod_solver_imex.f90:25-342 (periodic): x0 = the step's
// initial state (X.lvl1), right-hand side the stage state in (rho32, E32,
// q32), which receives the solution on the working nodes.
int imex_cg(sod_gpu_ctx *c, float fact, float dt, int maxIter, double tol) {
  auto &S = c->comp;
  auto &X = c->imex;
  const long long N = c->npoin;
  const int nw = c->npoin_w;
  const unsigned nb = nblk(nw, 256);
  const float gm1 = c->phys.gamma_gas - 1.0f;
  CUDA_TRY(cudaMemcpyAsync(X.x, X.lvl1, 5 * N * 4, cudaMemcpyDeviceToDevice, c->stream));
  CUDA_TRY(cudaMemcpyAsync(X.b, S.rho32, N * 4, cudaMemcpyDeviceToDevice, c->stream));
  CUDA_TRY(cudaMemcpyAsync(X.b + N, S.E32, N * 4, cudaMemcpyDeviceToDevice, c->stream));
  CUDA_TRY(cudaMemcpyAsync(X.b + 2 * N, S.q32, 3 * N * 4, cudaMemcpyDeviceToDevice, c->stream));
  auto apply = [&](const float *v) {  // qn = v Ml + fact dt D(v)
    k_imex_prim<<<nb, 256, 0, c->stream>>>(nw, N, c->lpoin_w, gm1, c->phys.Rgas, X.x, v, X.au, X.aT);
    int arc = imex_diffusion(c, X.x, v, X.au, X.aT, X.qn);
    k_imex_op<<<nb, 256, 0, c->stream>>>(nw, N, c->lpoin_w, c->Ml, v, fact, dt, X.qn);
    return arc;
  };
  int rc = apply(X.x);
  if (rc) return rc;
  k_imex_vec<<<nb, 256, 0, c->stream>>>(0, nw, N, c->lpoin_w, c->Ml, dt, 0.f, 0.f, X.b, X.x, X.r, X.p, X.qn, X.z,
                                        X.z1);
  const double auxB = std::sqrt(imex_dot(c, X.r, X.r, nullptr, &rc));
  if (rc) return rc;
  double nrm = auxB;
  int it;
  for (it = 1; it <= maxIter; ++it) {
    if ((rc = apply(X.p))) return rc;
    const double Q1 = imex_dot(c, X.r, X.z, nullptr, &rc);
    const double Q2 = imex_dot(c, X.p, X.qn, nullptr, &rc);
    if (rc) return rc;
    const float alpha = (float)(Q1 / Q2);
    k_imex_vec<<<nb, 256, 0, c->stream>>>(1, nw, N, c->lpoin_w, c->Ml, dt, alpha, 0.f, X.b, X.x, X.r, X.p, X.qn,
                                          X.z, X.z1);
    nrm = std::sqrt(imex_dot(c, X.r, X.r, nullptr, &rc));
    if (rc) return rc;
    if (!std::isfinite(nrm)) return fail(SOD_GPU_ENONFINITE, "non-finite residual in the IMEX solve");
    if (nrm < tol * auxB) break;
    const double T = imex_dot(c, X.r, X.z, X.z1, &rc);
    if (rc) return rc;
    const float beta = (float)(T / Q1);
    k_imex_vec<<<nb, 256, 0, c->stream>>>(2, nw, N, c->lpoin_w, c->Ml, dt, 0.f, beta, X.b, X.x, X.r, X.p, X.qn,
                                          X.z, X.z1);
  }
  k_imex_out<<<nb, 256, 0, c->stream>>>(nw, N, c->lpoin_w, X.x, S.rho32, S.E32, S.q32);
  X.cg_iters = it > maxIter ? maxIter : it;
  X.cg_res = auxB > 0 ? nrm / auxB : 0.0;
  return 0;
}

}  // namespace

extern "C" {

int sod_gpu_comp_imex_step(sod_gpu_ctx *c, float dt, int maxIter, double tol) {
  if (!c || !c->comp.ready) return fail(SOD_GPU_EINVAL, "state not initialised");
  if (!(dt > 0.f) || maxIter < 1 || !(tol > 0.0)) return fail(SOD_GPU_EINVAL, "bad argument");
  auto &S = c->comp;
  if (S.stages != 3 && S.stages != 4) return fail(SOD_GPU_EINVAL, "the IMEX integrator has 3 or 4 stages");
  if (S.fp64) return fail(SOD_GPU_EINVAL, "the IMEX integrator runs on the FP32 state (fp64_state = 0)");
  int rc;
  if ((rc = ensure_imex(c))) return rc;
  auto &X = c->imex;
  const cudaStream_t st = c->stream;
  const long long N = c->npoin;
  const int nw = c->npoin_w;
  const unsigned nb = nblk(nw, 256);
  const float gm = c->phys.gamma_gas;
  const ImexCoef K = imex_coef(S.stages);
  const bool was_async = c->async;
  c->async = true;
  // level 1 <- level 2 (CFDSolverBase.f90:1951-1960)
  CUDA_TRY(cudaMemcpyAsync(S.u1, S.u2, 3 * N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(S.eta1, S.eta2, N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(X.lvl1, S.rho32, N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(X.lvl1 + N, S.E32, N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(X.lvl1 + 2 * N, S.q32, 3 * N * 4, cudaMemcpyDeviceToDevice, st));
  const long long B = 5 * N;
  if (S.first) {  // time_integ_imex.f90:240-273
    S.first = false;
    k_feta<<<nb, 256, 0, st>>>(nw, N, c->lpoin_w, S.u1, S.eta1, S.feta);
    k_aux_h<<<nb, 256, 0, st>>>(nw, c->lpoin_w, gm / (gm - 1.0f), S.rho32, S.pr, X.aux_h);
    if ((rc = comp_entropy_pass(c, S.Reta1, false)) || (rc = comp_visc(c, S.Reta1, S.rho32, S.u1, false)) ||
        (rc = imex_convec(c, S.rho32, S.u2, S.q32, S.pr, X.aux_h, X.R)) ||
        (rc = imex_diffusion(c, nullptr, S.rho32, S.u2, S.Tem, X.D))) {
      c->async = was_async;
      return rc;
    }
  } else {  // the last stage's residuals open the step
    CUDA_TRY(cudaMemcpyAsync(X.R, X.R + (S.stages - 1) * B, B * 4, cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(X.D, X.D + (S.stages - 1) * B, B * 4, cudaMemcpyDeviceToDevice, st));
  }
  // LPS stabilisation of the step's initial state (comp_tau, full_proj_ijk,
  // full_stab_ijk with fact -1 = the LPS part of full_diff_stab_ijk with zero
  // viscosities and fact +1)
  k_comp_tau<<<nblk(c->nelem, 8), 256, 0, st>>>(c->nelem, c->N, c->conn, c->helem, S.csound, S.u2, c->npoin,
                                                c->phys.c_species_stab / (float)c->P, S.tau);
  {
    RhsArgs A{};
    A.rho = S.rho32; A.u = S.u2; A.Tem = S.Tem; A.mu_fluid = X.zmu; A.mue_t = X.zmue; A.musgs_t = nullptr;
    A.tau_stab = S.tau; A.proj12 = c->proj12; A.fact_d = 1.0f;
    rc = dispatch(c, [&](auto L) {
      L.proj(c, true, S.rho32, S.u2, S.Tem);
      gather_proj_aos(c);
      int hrc = halo_sum(c, halo_proj_view(c));
      if (hrc) return hrc;
      L.template rhs<MODE_DIFF, IN_DIFF>(c, A);
      return 0;
    });
    if (!rc) {
      gather_res(c, X.stab, X.stab + 2 * N, X.stab + N, 0, 0);
      rc = halo_block5(c, X.stab);
    }
    if (rc) {
      c->async = was_async;
      return rc;
    }
  }
  int iters = 0;
  for (int is = 2; is <= S.stages; ++is) {
    k_imex_comb<<<nblk(N, 256), 256, 0, st>>>(N, is, K, dt, c->Ml, X.R, X.D, X.stab, X.lvl1, S.rho32, S.E32, S.q32);
    if ((rc = imex_cg(c, K.ai[is][is], dt, maxIter, tol))) { c->async = was_async; return rc; }
    iters += X.cg_iters;
    k_eos_end<<<nb, 256, 0, st>>>(nw, N, c->lpoin_w, gm - 1.0f, gm, c->phys.Rgas, S.rho32, S.q32, S.E32, S.u2, S.eint,
                                  S.pr, S.csound, S.machno, S.Tem);
    k_aux_h<<<nb, 256, 0, st>>>(nw, c->lpoin_w, gm / (gm - 1.0f), S.rho32, S.pr, X.aux_h);
    if ((rc = imex_convec(c, S.rho32, S.u2, S.q32, S.pr, X.aux_h, X.R + (is - 1) * B)) ||
        (rc = imex_diffusion(c, nullptr, S.rho32, S.u2, S.Tem, X.D + (is - 1) * B))) {
      c->async = was_async;
      return rc;
    }
  }
  X.cg_iters = iters;
  // entropy viscosity of the new state (time_integ_imex.f90:454-505)
  k_thermo_entropy<<<nb, 256, 0, st>>>(nw, N, c->lpoin_w, gm, c->phys.p_inf, c->phys.rho_inf, S.rho32, S.pr, S.u1,
                                       S.eta1, S.eta2, S.feta);
  if ((rc = comp_entropy_pass(c, S.Reta2, true))) {
    c->async = was_async;
    return rc;
  }
  k_aux_reta<<<nb, 256, 0, st>>>(nw, c->lpoin_w, dt, S.Reta1, S.Reta2, S.eta1, S.eta2, S.aux);
  if ((rc = comp_visc(c, S.aux, S.rho32, S.u2, true))) {
    c->async = was_async;
    return rc;
  }
  k_sutherland<<<nb, 256, 0, st>>>(nw, c->lpoin_w, S.mu_factor, S.Tem, S.mu_fluid);
  c->async = was_async;
  return c->finish();
}

int sod_gpu_comp_imex_stats(sod_gpu_ctx *c, int *cg_iters, double *cg_res) {
  if (!c || !c->comp.ready) return fail(SOD_GPU_EINVAL, "state not initialised");
  if (cg_iters) *cg_iters = c->imex.cg_iters;
  if (cg_res) *cg_res = c->imex.cg_res;
  return 0;
}

int sod_gpu_comp_adapt_dt(sod_gpu_ctx *c, float cfl_conv, float cfl_diff, float *dt) {
  if (!c || !c->comp.ready || !dt) return fail(SOD_GPU_EINVAL, "bad argument");
  auto &S = c->comp;
  const unsigned init_bits = 0x56B5E621u;  // 1e14f
  CUDA_TRY(cudaMemcpyAsync(S.bits + 1, &init_bits, 4, cudaMemcpyHostToDevice, c->stream));
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    k_dt<LL::P_><<<nblk(c->nelem, 8), 256, 0, c->stream>>>(c->md(), c->helem, S.u2, S.csound, S.mu_fluid,
                                                            c->mue_t, S.rho32, cfl_conv, cfl_diff, S.bits + 1);
    return 0;
  });
  int rc = allreduce(c, S.bits + 1, 1, SOD_REDUCE_MIN_F32);
  if (rc) return rc;
  unsigned b = 0;
  CUDA_TRY(cudaMemcpyAsync(&b, S.bits + 1, 4, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  float v;
  std::memcpy(&v, &b, 4);
  *dt = v;
  return 0;
}

int sod_gpu_comp_analysis(sod_gpu_ctx *c, float rho0, double *out) {
  if (!c || !c->comp.ready || !out) return fail(SOD_GPU_EINVAL, "bad argument");
  auto &S = c->comp;
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    k_analysis_elem<LL::P_, LL::EPB><<<LL::grid(c->nelem), LL::TPB, 0, c->stream>>>(
        c->md(), S.rho32, S.u2, S.mu_fluid, c->mue_t, c->Ngp_t, S.part);
    return 0;
  });
  k_sum_parts<<<1, 1024, 0, c->stream>>>(c->nelem, S.part, S.sums);
  const unsigned zero = 0u;
  CUDA_TRY(cudaMemcpyAsync(S.bits + 2, &zero, 4, cudaMemcpyHostToDevice, c->stream));
  k_max_mach<<<MINMAX_BLOCKS, 256, 0, c->stream>>>(c->npoin_w, c->lpoin_w, S.machno, S.bits + 2);
  int rc;
  if ((rc = allreduce(c, S.sums, 3, SOD_REDUCE_SUM_F64)) || (rc = allreduce(c, S.bits + 2, 1, SOD_REDUCE_MAX_F32)))
    return rc;
  double sums[3];
  unsigned mb = 0;
  CUDA_TRY(cudaMemcpyAsync(sums, S.sums, 24, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaMemcpyAsync(&mb, S.bits + 2, 4, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  const float twopi = 2.0f * 3.14159f;
  double EK = sums[0] / (double)(rho0 * powf(twopi, 3.0f));
  const float alpha = 1.0f / (rho0 * c->volT);
  double eS = sums[1] * (double)alpha;
  double eD = (double)(4.0f / 3.0f) * sums[2] * (double)alpha;
  float mach;
  std::memcpy(&mach, &mb, 4);
  out[0] = (double)(float)EK;
  out[1] = (double)(float)eS;
  out[2] = (double)(float)eD;
  out[3] = (double)(float)(eS + eD);
  out[4] = (double)mach;
  return 0;
}

int sod_gpu_comp_get_state(sod_gpu_ctx *c, float *rho, float *q, float *E, float *mu_e) {
  if (!c || !c->comp.ready) return fail(SOD_GPU_EINVAL, "state not initialised");
  auto &S = c->comp;
  const size_t N = c->npoin;
  if (rho) CUDA_TRY(cudaMemcpyAsync(rho, S.rho32, N * 4, cudaMemcpyDeviceToDevice, c->stream));
  if (q) CUDA_TRY(cudaMemcpyAsync(q, S.q32, 3 * N * 4, cudaMemcpyDeviceToDevice, c->stream));
  if (E) CUDA_TRY(cudaMemcpyAsync(E, S.E32, N * 4, cudaMemcpyDeviceToDevice, c->stream));
  if (mu_e) {
    const long long EN = (long long)c->nelem * c->N;
    k_t_to_elem<<<nblk(EN, 256), 256, 0, c->stream>>>(c->nelem, c->N, c->a_of_t, c->mue_t, mu_e);
  }
  return c->finish();
}

}  // extern "C"

// ---- learned preconditioner: set-up, loss/gradient, harvest, training ----

namespace {

__global__ void k_loss_grad_vec(int npoin_w, const int *__restrict__ lpoin_w, const double *__restrict__ Ad,
                                double scale, double *__restrict__ g) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const int i = lpoin_w[t];
  g[i] = scale * Ad[i];
}

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

__global__ void k_inv_sqrt_diag(long long n, const float *__restrict__ diag, double *__restrict__ Dh) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) Dh[i] = diag[i] > 0.f ? 1.0 / sqrt((double)diag[i]) : 0.0;
}

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

int ensure_train_scratch(sod_gpu_ctx *c) {
  auto &NT = c->net;
  if (NT.X) return 0;
  const size_t E = (size_t)c->nelem;
  int rc;
  if ((rc = c->alloc(&NT.X, E * NT.NP)) || (rc = c->alloc(&NT.W, E * NT.NP)) || (rc = c->alloc(&NT.Y, E * NET_K)) ||
      (rc = c->alloc(&NT.SA, E * NET_K)) || (rc = c->alloc(&NT.dS, E * NET_K)))
    return rc;
  return 0;
}

// Parameter-gradient partials of g = dL/dz at the residual r into part
// (nblk_bwd rows of nparam floats).
void net_backward(sod_gpu_ctx *c, const double *r, const double *g, float *part) {
  auto &NT = c->net;
  const long long stride = NT.nparam;
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    constexpr int P = LL::P_;
    using D = NetDims<P>;
    k_patch_bwd_elem<P><<<4 * 148, 256, D::bwd_smem(8), c->stream>>>(c->nelem, NT.pt, r, g, NT.Dh, NT.params,
                                                                     NT.gains, NT.X, NT.W, NT.Y, NT.SA, NT.dS);
    k_patch_dB<P><<<NT.nblk_bwd, 256, 0, c->stream>>>(c->nelem, NT.X, NT.W, NT.Y, NT.SA, part, stride);
    k_mlp_bwd<P><<<NT.nblk_bwd, 256, 0, c->stream>>>(c->nelem, NT.feat, NT.params, NT.dS,
                                                                           part, stride);
    k_alpha_part<<<NT.nblk_bwd, 256, 0, c->stream>>>(c->npoin_w, c->lpoin_w, r, g, NT.Dh, NT.params, D::O_ALPHA,
                                                     part, stride);
    return 0;
  });
}

// loss = d^T A d / eAe with d = e - M r; the gradient partials go to part.
int net_loss_grad(sod_gpu_ctx *c, const double *r, const double *e, double eAe, float *part, double *loss) {
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
  net_backward(c, r, NT.tmp2, part);
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
    const size_t NPt = (size_t)E * NT.NP;
    if ((rc = c->alloc(&NT.params, NT.nparam)) || (rc = c->alloc(&NT.m1, NT.nparam)) ||
        (rc = c->alloc(&NT.m2, NT.nparam)) || (rc = c->alloc(&NT.grad, NT.nparam)) ||
        (rc = c->alloc(&NT.part, (size_t)NT.nblk_bwd * NT.nparam * 16)) || (rc = c->alloc(&NT.pt, NPt)) || (rc = c->alloc(&NT.pos, NPt)) ||
        (rc = c->alloc(&NT.pptr, (size_t)c->npoin + 1)) || (rc = c->alloc(&NT.pslot, NPt)) ||
        (rc = c->alloc(&NT.feat, (size_t)E * NET_F)) || (rc = c->alloc(&NT.gains, (size_t)E * NET_K)) ||
        (rc = c->alloc(&NT.Dh, (size_t)c->npoin)) || (rc = c->alloc(&NT.uf, (size_t)c->npoin)) ||
        (rc = c->alloc(&NT.tmp1, (size_t)c->npoin)) ||
        (rc = c->alloc(&NT.tmp2, (size_t)c->npoin)))
      return rc;
    if (P == 3) {
      using D = NetDims<3>;
      CUDA_TRY(cudaFuncSetAttribute(k_patch_apply<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)D::apply_smem(8)));
      CUDA_TRY(cudaFuncSetAttribute(k_patch_bwd_elem<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)D::bwd_smem(8)));
      CUDA_TRY(cudaFuncSetAttribute(k_patch_apply_tc<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)TcDims<3>::smem()));
    } else {
      using D = NetDims<4>;
      CUDA_TRY(cudaFuncSetAttribute(k_patch_apply<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)D::apply_smem(8)));
      CUDA_TRY(cudaFuncSetAttribute(k_patch_bwd_elem<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)D::bwd_smem(8)));
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
      int rc = net_loss_grad(c, rd, ed, NT.eAe[k], NT.part + (size_t)b * NT.nblk_bwd * NT.nparam,
                             (st == steps - 1) ? &l : nullptr);
      if (rc) return rc;
      sum += l;
    }
    NT.step += 1;
    const float bc1 = 1.f - std::pow(0.9f, (float)NT.step), bc2 = 1.f - std::pow(0.999f, (float)NT.step);
    k_adam<<<nblk(NT.nparam, 256), 256, 0, c->stream>>>(NT.nparam, NT.nblk_bwd * batch, NT.part, NT.params, NT.m1,
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
