// Allocation-free variant of the analysis integrals (EK, eps_S, eps_D,
// eps_T, max Mach) for callers that cannot allocate device memory.
//
// Who needs it: a Fortran/OpenACC solver that hands all device memory to
// its own pool (or runs with a memory cap), and embedded callers that must
// not trigger cudaMalloc's implicit device synchronisation inside the time
// loop.  The context-based sod_gpu_comp_analysis needs a sod_gpu_ctx,
// whose creation allocates; this entry point takes every array as a plain
// device pointer in the reference layout and uses a fixed scratch area in a
// file-scope __device__ array instead of allocated memory.
//
// Scratch: SOD_NOALLOC_MAX_ELEM elements x 3 FP32 partial sums (12 MiB)
// plus 3 FP64 totals and one FP32 maximum.  The array exists on every GPU
// that loads this library, for the life of the process.  All calls share
// it: each call clears what must start at zero and overwrites the rest, so
// two calls that overlap on the GPU (different streams, or different host
// threads on the same device) race and must be serialised by the caller.
#include "sod2d_gpu.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

int sod_detail_set_error(int code, const char *msg);  // sod2d_gpu.cu

namespace {

constexpr long long kMaxElem = SOD_NOALLOC_MAX_ELEM;
// layout (bytes): [0, 12*kMaxElem) per-element FP32 partials (3 per
// element); then 3 FP64 totals; then one 32-bit max-Mach cell.
constexpr size_t kPartBytes = (size_t)kMaxElem * 3 * sizeof(float);
constexpr size_t kScratchBytes = kPartBytes + 4 * sizeof(double);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of g_noalloc_scratch in the calling thread's current
// context.  Looked up on every call (a table lookup in the runtime once the
// module is loaded; the first call in a context also loads the module
// there): a cached address would go stale after cudaDeviceReset or when the
// caller switches to another context on the same device, and the kernels
// would then write through a dangling pointer.
int scratch_address(void **out) {
  void *p = nullptr;
  if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return -1;
  *out = p;
  return 0;
}

// One block per element, one thread per reference-local node a; loops
// follow volAvg_EK and visc_dissipationRate (src/lib_sod2d/sources/
// mod_analysis.f90:10-144) with sum-factorised gradients.
template <int P>
__global__ void k_noalloc_elem(int nelem, long long npoin, const int *__restrict__ connec,
                               const int *__restrict__ invA, const int *__restrict__ gI, const int *__restrict__ gJ,
                               const int *__restrict__ gK, const float *__restrict__ dl, const float *__restrict__ He,
                               const float *__restrict__ gpvol, const float *__restrict__ Ngp,
                               const float *__restrict__ rho, const float *__restrict__ u,
                               const float *__restrict__ mu_fluid, const float *__restrict__ mu_e,
                               float *__restrict__ part) {
  constexpr int N1 = P + 1, N = N1 * N1 * N1;
  __shared__ float su[3][N], ske[N];
  __shared__ float red[3][4];
  const int e = blockIdx.x, a = threadIdx.x, lane = a % 32, w = a / 32;
  const long long NE = nelem;
  int node = 0;
  if (a < N) {
    node = connec[e + NE * a] - 1;
    const float u0 = u[node], u1 = u[node + npoin], u2 = u[node + 2 * npoin];
    su[0][a] = u0; su[1][a] = u1; su[2][a] = u2;
    ske[a] = 0.5f * rho[node] * (u0 * u0 + u1 * u1 + u2 * u2);
  }
  __syncthreads();
  float r[3] = {0.f, 0.f, 0.f};
  if (a < N) {
    const int I = gI[a] - 1, J = gJ[a] - 1, K = gK[a] - 1;
    float gi[3][3] = {};
    for (int ii = 0; ii < N1; ++ii) {
      const int a0 = invA[ii + N1 * (J + N1 * K)] - 1, a1 = invA[I + N1 * (ii + N1 * K)] - 1,
                a2 = invA[I + N1 * (J + N1 * ii)] - 1;
      const float d0 = dl[a + N * (0 + 3 * ii)], d1 = dl[a + N * (1 + 3 * ii)], d2 = dl[a + N * (2 + 3 * ii)];
      for (int c = 0; c < 3; ++c) {
        gi[c][0] += d0 * su[c][a0];
        gi[c][1] += d1 * su[c][a1];
        gi[c][2] += d2 * su[c][a2];
      }
    }
    const float *h = He + 9 * ((long long)a + (long long)N * e);
    float gu[3][3];
    for (int c = 0; c < 3; ++c)
      for (int b = 0; b < 3; ++b) gu[c][b] = h[b] * gi[c][0] + h[b + 3] * gi[c][1] + h[b + 6] * gi[c][2];
    float div = gu[0][0] + gu[1][1] + gu[2][2];
    div = div * div;
    const float c0 = gu[1][2] - gu[2][1], c1 = gu[2][0] - gu[0][2], c2 = gu[0][1] - gu[1][0];
    const float curl2 = c0 * c0 + c1 * c1 + c2 * c2;
    float ek = 0.f;
    for (int b = 0; b < N; ++b) ek += (Ngp ? Ngp[a + N * b] : (a == b ? 1.f : 0.f)) * ske[b];
    const float gv = gpvol[a + (long long)N * e];
    const float mu = mu_fluid[node];
    r[0] = gv * ek;
    r[1] = gv * (mu + mu_e[e + NE * a]) * curl2;
    r[2] = gv * mu * div;
  }
  for (int q = 0; q < 3; ++q)
    for (int o = 16; o > 0; o >>= 1) r[q] += __shfl_down_sync(0xffffffffu, r[q], o);
  if (lane == 0)
    for (int q = 0; q < 3; ++q) red[q][w] = r[q];
  __syncthreads();
  if (a == 0) {
    const int nw = blockDim.x / 32;
    for (int q = 0; q < 3; ++q) {
      float sq = 0.f;
      for (int ww = 0; ww < nw; ++ww) sq += red[q][ww];
      part[(long long)e * 3 + q] = sq;
    }
  }
}

// Fixed-order FP64 totals of the partials, and the max-Mach cell reset.
__global__ void k_noalloc_sum(int nelem, const float *__restrict__ part, double *__restrict__ tot,
                              unsigned int *__restrict__ mach_bits) {
  __shared__ double sh[3][1024];
  const int t = threadIdx.x;
  double s[3] = {0.0, 0.0, 0.0};
  for (long long e = t; e < nelem; e += blockDim.x)
    for (int q = 0; q < 3; ++q) s[q] += (double)part[e * 3 + q];
  for (int q = 0; q < 3; ++q) sh[q][t] = s[q];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (t < w)
      for (int q = 0; q < 3; ++q) sh[q][t] += sh[q][t + w];
    __syncthreads();
  }
  if (t == 0) {
    for (int q = 0; q < 3; ++q) tot[q] = sh[q][0];
    *mach_bits = 0u;  // must start at zero for the max below
  }
}

__global__ void k_noalloc_mach(int npoin_w, const int *__restrict__ lpoin_w, const float *__restrict__ machno,
                               unsigned int *__restrict__ mach_bits) {
  float v = 0.f;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < npoin_w; t += gridDim.x * blockDim.x)
    v = fmaxf(v, machno[lpoin_w[t] - 1]);
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) atomicMax(mach_bits, __float_as_uint(v));  // machno >= 0
}

}  // namespace

extern "C" int sod_gpu_analysis_noalloc(int porder, int nelem, int npoin, int npoin_w, const int *connec,
                                        const int *lpoin_w, const int *invAtoIJK, const int *gmshAtoI,
                                        const int *gmshAtoJ, const int *gmshAtoK, const float *dlxigp_ip,
                                        const float *He, const float *gpvol, const float *Ngp, const float *rho,
                                        const float *u, const float *mu_fluid, const float *mu_e,
                                        const float *machno, float rho0, float volT, void *stream, double *out) {
  if ((porder != 3 && porder != 4) || nelem <= 0 || npoin <= 0 || npoin_w <= 0 || !connec || !lpoin_w ||
      !invAtoIJK || !gmshAtoI || !gmshAtoJ || !gmshAtoK || !dlxigp_ip || !He || !gpvol || !rho || !u ||
      !mu_fluid || !mu_e || !machno || !out || !(rho0 > 0.f) || !(volT > 0.f))
    return sod_detail_set_error(SOD_GPU_EINVAL, "sod_gpu_analysis_noalloc: bad argument");
  if ((long long)nelem > kMaxElem)
    return sod_detail_set_error(SOD_GPU_EINVAL, "sod_gpu_analysis_noalloc: nelem exceeds SOD_NOALLOC_MAX_ELEM "
                                                "(the fixed scratch holds 1048576 elements)");
  void *base = nullptr;
  if (scratch_address(&base))
    return sod_detail_set_error(SOD_GPU_ECUDA, "sod_gpu_analysis_noalloc: cudaGetSymbolAddress failed");
  float *part = (float *)base;
  double *tot = (double *)((unsigned char *)base + kPartBytes);
  unsigned int *mach = (unsigned int *)(tot + 3);
  cudaStream_t st = (cudaStream_t)stream;
  if (porder == 3)
    k_noalloc_elem<3><<<nelem, 64, 0, st>>>(nelem, npoin, connec, invAtoIJK, gmshAtoI, gmshAtoJ, gmshAtoK,
                                            dlxigp_ip, He, gpvol, Ngp, rho, u, mu_fluid, mu_e, part);
  else
    k_noalloc_elem<4><<<nelem, 128, 0, st>>>(nelem, npoin, connec, invAtoIJK, gmshAtoI, gmshAtoJ, gmshAtoK,
                                             dlxigp_ip, He, gpvol, Ngp, rho, u, mu_fluid, mu_e, part);
  k_noalloc_sum<<<1, 1024, 0, st>>>(nelem, part, tot, mach);
  k_noalloc_mach<<<296, 256, 0, st>>>(npoin_w, lpoin_w, machno, mach);
  double h[3];
  unsigned int mb = 0;
  if (cudaMemcpyAsync(h, tot, sizeof h, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(&mb, mach, sizeof mb, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return sod_detail_set_error(SOD_GPU_ECUDA, "sod_gpu_analysis_noalloc: CUDA copy failed");
  if (cudaGetLastError() != cudaSuccess)
    return sod_detail_set_error(SOD_GPU_ECUDA, "sod_gpu_analysis_noalloc: kernel launch failed");
  const float twopi = 2.0f * 3.14159f;
  const double EK = h[0] / (double)(rho0 * powf(twopi, 3.0f));
  const float alpha = 1.0f / (rho0 * volT);
  const double eS = h[1] * (double)alpha;
  const double eD = (double)(4.0f / 3.0f) * h[2] * (double)alpha;
  float mach_v;
  std::memcpy(&mach_v, &mb, 4);
  out[0] = (double)(float)EK;
  out[1] = (double)(float)eS;
  out[2] = (double)(float)eD;
  out[3] = (double)(float)(eS + eD);
  out[4] = (double)mach_v;
  return SOD_GPU_OK;
}
