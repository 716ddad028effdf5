// Element kernels of the compressible RHS for sm_100a.
//
// Layout (built once by sod_gpu_init):
//   conn[e][t]        0-based node id of tensor position t = i + n1*j + n1^2*k
//                     (natural 1-D GLL order, xi ascending)
//   geo[e][c][t]      c = 0..8: He(i,j) at c = i + 3j (= d xi_j / d x_i);
//                     c = 9: gpvol
//   slots             per element-node contributions of the RHS passes, at
//                     the node-sorted position slot_pos[e][t] (W floats)
// One thread owns one Gauss point (= node) of one element; an element's
// nodal fields are staged in shared memory and differentiated with the 1-D
// GLL derivative matrix D[m][n] = l'_n(xi_m) (sum factorisation).  The
// 4x4 / 5x5 contractions are too small for tensor cores; they run on the
// FP32 pipes.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#ifndef SOD_VEC_XI
#define SOD_VEC_XI 1
#endif
// Pass-B blocks resident per SM: 512 threads per SM, 128 registers each.
#ifndef SOD_RHS_THREADS_PER_SM
#define SOD_RHS_THREADS_PER_SM 512
#endif

namespace sod {

template <int P>
struct Cfg {
  static constexpr int N1 = P + 1;
  static constexpr int N = N1 * N1 * N1;
  static constexpr int NT = ((N + 31) / 32) * 32;  // threads per element
};

struct Phys {
  float gm1;      // gamma - 1
  float gogm1;    // gamma / (gamma - 1)
  float Rgas, Cp, Prt;
  float c_lps, c_rho, c_ener;
  float cp_pr;    // Cp / Pr
  float twoThirds;
};

struct MeshDev {
  int nelem, npoin, npoin_w;
  const int *conn;      // [E][N]
  const float *geo;     // [E][10][N]
  const float *Dnat;    // [N1][N1]
  const int *lpoin_w;   // 0-based
  const float *invMl;   // [npoin]
  const int *slot_ptr;  // [npoin+1]
  const int *slot_idx;  // [E*N], value e*N+t
  const int *slot_pos;  // [E*N]: node-sorted slot of element node (e, t); inverse of slot_idx
};

// 1-D summation order of the reference ([-1, +1, interior...] as natural
// indices): 0, P, 1, 2, ..., P-1.
template <int P>
__device__ __forceinline__ int ref_order(int s) {
  return s == 0 ? 0 : (s == 1 ? P : s - 1);
}

// Iso-parametric derivatives of a staged field at tensor position (i,j,k).
template <int P>
__device__ __forceinline__ void iso_grad(const float *__restrict__ f, int i, int j, int k,
                                         const float (&Di)[P + 1], const float (&Dj)[P + 1],
                                         const float (&Dk)[P + 1], float &g0, float &g1, float &g2) {
  constexpr int N1 = P + 1;
  g0 = 0.f; g1 = 0.f; g2 = 0.f;
  if constexpr (P == 3 && SOD_VEC_XI) {
    // the xi-line of a 4-node element row is one aligned 16-byte load
    const float4 v = *reinterpret_cast<const float4 *>(f + 4 * j + 16 * k);
    const float fx[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int s = 0; s < N1; ++s) {
      const int m = ref_order<P>(s);
      g0 = fmaf(Di[m], fx[m], g0);
      g1 = fmaf(Dj[m], f[i + N1 * m + N1 * N1 * k], g1);
      g2 = fmaf(Dk[m], f[i + N1 * j + N1 * N1 * m], g2);
    }
  } else {
#pragma unroll
    for (int s = 0; s < N1; ++s) {
      const int m = ref_order<P>(s);
      g0 = fmaf(Di[m], f[m + N1 * j + N1 * N1 * k], g0);
      g1 = fmaf(Dj[m], f[i + N1 * m + N1 * N1 * k], g1);
      g2 = fmaf(Dk[m], f[i + N1 * j + N1 * N1 * m], g2);
    }
  }
}

struct NodeQ {  // primitive quantities of one node
  float rho, u0, u1, u2, q0, q1, q2, p, h, T, mu;
};

// Equation of state at one node from the conserved variables, in the
// operation order of updateF (time_integ_ls.f90:574-587) and
// sutherland_viscosity (mod_fluid_viscosity.f90:21-41).
__device__ __forceinline__ void eos(const Phys &ph, float Rgas, float mu_factor, float rho,
                                    float q0, float q1, float q2, float E, NodeQ &s) {
  s.rho = rho; s.q0 = q0; s.q1 = q1; s.q2 = q2;
  s.u0 = q0 / rho; s.u1 = q1 / rho; s.u2 = q2 / rho;
  float umag = s.u0 * s.u0;
  umag = umag + s.u1 * s.u1;
  umag = umag + s.u2 * s.u2;
  const float eint = (E / rho) - 0.5f * umag;
  s.p = rho * ph.gm1 * eint;
  s.h = ph.gogm1 * s.p / rho;
  s.T = s.p / (rho * Rgas);
  s.mu = mu_factor * 1.458e-6f * powf(s.T, 1.5f) / (s.T + 110.4f);
}

// Equation of state of the element kernels: the operations of updateF
// (time_integ_ls.f90:574-587) and sutherland_viscosity
// (mod_fluid_viscosity.f90:21-41) with one reciprocal of rho in place of
// the divisions and T*sqrt(T) for T**1.5 (each within 2 ulp of the
// reference's FP32 value).
__device__ __forceinline__ void eos_fast(const Phys &ph, float invR, float mu_factor, float rho, float q0,
                                         float q1, float q2, float E, NodeQ &s) {
  const float ri = __frcp_rn(rho);
  s.rho = rho; s.q0 = q0; s.q1 = q1; s.q2 = q2;
  s.u0 = q0 * ri; s.u1 = q1 * ri; s.u2 = q2 * ri;
  float umag = s.u0 * s.u0;
  umag = umag + s.u1 * s.u1;
  umag = umag + s.u2 * s.u2;
  const float eint = E * ri - 0.5f * umag;
  s.p = rho * ph.gm1 * eint;
  s.h = ph.gogm1 * s.p * ri;
  s.T = s.p * ri * invR;
  s.mu = mu_factor * 1.458e-6f * (s.T * sqrtf(s.T)) * __frcp_rn(s.T + 110.4f);
}

// Asynchronous global -> shared copies (cp.async): the prefetch of the next
// element group holds no registers while it is in flight.
__device__ __forceinline__ void cp_async4(float *dst, const void *src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(float *dst, const void *src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Bulk (TMA) copies of contiguous per-element data into shared memory,
// completed on an mbarrier (transaction count).
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// dst (shared) and src (global) 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// Bounded wait for the phase `parity` of bar (try_wait itself suspends the
// thread for a while): false after SOD_BULK_WAIT_LIMIT polls.
#ifndef SOD_BULK_WAIT_LIMIT
#define SOD_BULK_WAIT_LIMIT (1 << 24)
#endif
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity) {
  for (int it = 0; it < SOD_BULK_WAIT_LIMIT; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// ---------------------------------------------------------------------
// Pass A: LPS projections (full_proj_ijk, elem_stab.f90:474-562).  Writes
// gpvol * {tau00, tau01, tau02, tau11, tau12, tau22, grad rho (3), grad T
// (3)} per element node into element-ordered slots of width 12 (coalesced
// stores; k_gather reads them through the node->slot CSR).  tau = grad u + grad u^T
// - 2/3 div u I is symmetric (tau_ab and tau_ba are the same FP32 sum), so
// the reference's ProjMX/MY/MZ rows are read back from its 6 entries.
// Input: conserved state (SoA, reference layout) -> EOS in registers, or
// primitive rho/u/T (prim = true).
// ---------------------------------------------------------------------
// P = 3: 16 blocks per SM (32 registers, full occupancy) hide more of the
// latency of the state gather: 1.636 against 1.643 ms per RHS at 64^3 with
// 44 registers (11 blocks); 40 registers (12 blocks) gave 1.643.
template <int P, int EPB, bool PRIM>
__global__ void __launch_bounds__(EPB *Cfg<P>::NT, P == 3 ? 16 : 1)
k_proj(MeshDev m, Phys ph, float Rgas, const float *__restrict__ a0, const float *__restrict__ a1,
       const float *__restrict__ a2, float *__restrict__ slots) {
  constexpr int N1 = Cfg<P>::N1, N = Cfg<P>::N, NT = Cfg<P>::NT, NF = 5;
  __shared__ __align__(16) float sm[EPB][NF][N];
  const int el = threadIdx.x / NT, t = threadIdx.x % NT;
  const long long e = (long long)blockIdx.x * EPB + el;
  const bool active = (e < m.nelem) && (t < N);
  const long long NP = m.npoin;
  float He[9], gv = 0.f;
  if (active) {
    const int node = m.conn[e * N + t];
    // geometry loads issued before the staging barrier (independent of it)
    const float *g = m.geo + e * 10 * N + t;
#pragma unroll
    for (int c = 0; c < 9; ++c) He[c] = g[c * N];
    gv = g[9 * N];
    float rho, u0, u1, u2, T;
    if (PRIM) {  // a0 = rho, a1 = u(N,3), a2 = Tem
      rho = a0[node]; u0 = a1[node]; u1 = a1[node + NP]; u2 = a1[node + 2 * NP]; T = a2[node];
    } else {     // a0 = rho, a1 = q(N,3), a2 = E
      NodeQ s;
      eos_fast(ph, __frcp_rn(Rgas), 1.f, a0[node], a1[node], a1[node + NP], a1[node + 2 * NP], a2[node], s);
      rho = s.rho; u0 = s.u0; u1 = s.u1; u2 = s.u2; T = s.T;
    }
    sm[el][0][t] = rho; sm[el][1][t] = T;
    sm[el][2][t] = u0; sm[el][3][t] = u1; sm[el][4][t] = u2;
  }
  __syncthreads();
  // the element's 12-wide slots are staged in shared memory and written
  // out with coalesced 16-byte stores
  __shared__ __align__(16) float ost[EPB * N * 12];
  if (active) {
  const int i = t % N1, j = (t / N1) % N1, k = t / (N1 * N1);
  float Di[N1], Dj[N1], Dk[N1];
#pragma unroll
  for (int s = 0; s < N1; ++s) { Di[s] = m.Dnat[i * N1 + s]; Dj[s] = m.Dnat[j * N1 + s]; Dk[s] = m.Dnat[k * N1 + s]; }
  float gR[3], gT[3], gU[3][3];
  iso_grad<P>(sm[el][0], i, j, k, Di, Dj, Dk, gR[0], gR[1], gR[2]);
  iso_grad<P>(sm[el][1], i, j, k, Di, Dj, Dk, gT[0], gT[1], gT[2]);
#pragma unroll
  for (int c = 0; c < 3; ++c) iso_grad<P>(sm[el][2 + c], i, j, k, Di, Dj, Dk, gU[c][0], gU[c][1], gU[c][2]);
  float gradRho[3], gradT[3], gradU[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    gradRho[a] = He[a] * gR[0] + He[a + 3] * gR[1] + He[a + 6] * gR[2];
    gradT[a] = He[a] * gT[0] + He[a + 3] * gT[1] + He[a + 6] * gT[2];
  }
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) gradU[a][b] = He[b] * gU[a][0] + He[b + 3] * gU[a][1] + He[b + 6] * gU[a][2];
  const float divU = gradU[0][0] + gradU[1][1] + gradU[2][2];
  float4 *o = reinterpret_cast<float4 *>(ost + (el * N + t) * 12);
  float tau[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
#pragma unroll
    for (int b = 0; b < 3; ++b) tau[a][b] = gradU[a][b] + gradU[b][a];
    tau[a][a] = tau[a][a] - ph.twoThirds * divU;
  }
  o[0] = make_float4(gv * tau[0][0], gv * tau[0][1], gv * tau[0][2], gv * tau[1][1]);
  o[1] = make_float4(gv * tau[1][2], gv * tau[2][2], gv * gradRho[0], gv * gradRho[1]);
  o[2] = make_float4(gv * gradRho[2], gv * gradT[0], gv * gradT[1], gv * gradT[2]);
  }
  __syncthreads();
  const long long e0 = (long long)blockIdx.x * EPB;
  const long long ne = (m.nelem - e0) < EPB ? (m.nelem - e0) : EPB;
  const float4 *src = reinterpret_cast<const float4 *>(ost);
  float4 *dst = reinterpret_cast<float4 *>(slots + e0 * N * 12);
  for (int q = threadIdx.x; q < ne * N * 3; q += blockDim.x) dst[q] = src[q];
}

// ---------------------------------------------------------------------
// Pass B: convection (full_convec_ijk) and/or stabilised diffusion
// (full_diff_stab_ijk) of one element, summed per element node into slots
// of width 8: {mass, energy, mom x, mom y, mom z, 0, 0, 0}.
//
// MODE_CONV: convective residual * fact_c.
// MODE_DIFF: LPS-stabilised diffusion * fact_d (full_diff_stab_ijk);
//   with MODE_NOLPS the plain diffusion of full_diffusion_ijk
//   (elem_diffu.f90:12-223).
// Input kinds:
//   IN_CONS : a0 = rho, a1 = q(N,3), a2 = E (conserved; EOS fused, h = E:=aux_h)
//   IN_PRIM : convection inputs u, q, rho, pr, E given directly
//   IN_DIFF : diffusion inputs rho, u, Tem, mu_fluid given directly
// ---------------------------------------------------------------------
enum { MODE_CONV = 1, MODE_DIFF = 2, MODE_NOLPS = 4 };
enum { IN_CONS = 0, IN_PRIM = 1, IN_DIFF = 2 };

struct RhsArgs {
  // conserved / primitive inputs (reference layout)
  const float *rho, *q, *E, *u, *pr, *Tem, *mu_fluid;
  float mu_factor;
  // diffusion inputs
  const float *mue_t;     // [nelem][N] tensor order (internal copy of mu_e)
  const float *musgs_t;   // [nelem][N] or null
  const float *tau_stab;  // (nelem)
  const float *rho_n;     // IN_DIFF: density of the nu_e and mu_sgs terms when it differs
                          // from rho (full_diffusion_ijk's rho_n); null: rho
  const float *proj12;    // [npoin][12] mass-inverted projections (internal):
                          // tau00 tau01 tau02 tau11 tau12 tau22 gradRho(3) gradT(3)
  float fact_c, fact_d;
  int *err;  // mapped host flag: set when a bulk-copy wait of pass B gave up
};

// Staged pairs of pass B, one float2 per element node:
//   CONV (and CONV+DIFF): (u0,u1) (u2,rho) (q0,q1) (q2,p) (H,rho*H) [(T,0)]
//   DIFF only           : (u0,u1) (u2,rho) (T,0)
// The 18 product fields of the split form -- q_a u_b and u_a u_b (a <= b),
// rho*H*u_c and H*u_c -- are formed in registers from the staged values of
// each line node as it is read.  A product rounds the same way whether it
// is formed here or before staging, so this only trades shared-memory
// traffic (11 staged values per node instead of 29) for FP32 multiplies.
enum { PB_U01 = 0, PB_U2R = 1, PB_Q01 = 2, PB_Q2P = 3, PB_HRH = 4 };

// Shared-memory plan of k_rhs.  Two prefetch stages (the element group being
// computed and the next one), each holding, per thread of the block: the
// nodal inputs (NIN values gathered through the connectivity), J^-1 and
// gpvol (10), the node-sorted slot position, mu_e and mu_sgs, and the 12
// mass-inverted projections of the node; then the staging area of the
// element kernels (the paired fields, later the contravariant fluxes).
template <int P, int EPB, int MODE, int IN>
struct RhsPlan {
  static constexpr int N1 = P + 1, N = Cfg<P>::N, NT = Cfg<P>::NT, NTB = EPB * NT;
  static constexpr bool CONV = (MODE & MODE_CONV) != 0;
  static constexpr bool DIFF = (MODE & MODE_DIFF) != 0;
  static constexpr bool LPS = (MODE & MODE_NOLPS) == 0;
  static constexpr int NC = LPS ? 5 : 6;  // staged contravariant flux fields of the weak divergence
  static constexpr int NPAIR = CONV ? (DIFF ? 6 : 5) : 3;
  static constexpr int PB_T = CONV ? 5 : 2;
  // IN_CONS: rho q0 q1 q2 E | IN_PRIM: rho u0 u1 u2 q0 q1 q2 p h | IN_DIFF: rho rho_n u0 u1 u2 T mu
  static constexpr int NIN = IN == IN_CONS ? 5 : (IN == IN_PRIM ? 9 : 7);
  static constexpr int O_IN = 0, O_GEO = NIN * NTB, O_POS = O_GEO + 10 * NTB, O_MUE = O_POS + NTB,
                       O_MUS = O_MUE + (DIFF ? NTB : 0), O_PROJ = O_MUS + (DIFF ? NTB : 0);
  static constexpr int STAGE = O_PROJ + (DIFF && LPS ? 12 * NTB : 0);  // floats (multiple of 4)
  static constexpr int SMF = (2 * NPAIR > 3 * NC) ? 2 * NPAIR : 3 * NC;  // staging floats per element node
  static constexpr int O_STG = 2 * STAGE;
  static constexpr size_t BYTES = (size_t)(2 * STAGE + EPB * SMF * N) * sizeof(float);
};


// Persistent element kernel of pass B: a block walks element groups
// blockIdx.x, blockIdx.x + gridDim.x, ... and, while it computes one group,
// its cp.async copies bring the next group's inputs into the other stage.
template <int P, int EPB, int MODE, int IN>
__global__ void __launch_bounds__(EPB *Cfg<P>::NT, SOD_RHS_THREADS_PER_SM / (EPB * Cfg<P>::NT))
k_rhs(MeshDev m, Phys ph, float Rgas, RhsArgs A, float *__restrict__ slots) {
  using L = RhsPlan<P, EPB, MODE, IN>;
  constexpr int N1 = L::N1, N = L::N, NT = L::NT, NTB = L::NTB, NC = L::NC, SMF = L::SMF, PB_T = L::PB_T;
  constexpr bool CONV = L::CONV, DIFF = L::DIFF, LPS = L::LPS;
  extern __shared__ __align__(16) float dsm[];
  const int tid = threadIdx.x, el = tid / NT, t = tid % NT;
  const int i = t % N1, j = (t / N1) % N1, k = t / (N1 * N1);
  const long long NP = m.npoin;
  const long long ngroups = ((long long)m.nelem + EPB - 1) / EPB, G = gridDim.x;
  float *const sf = dsm + L::O_STG + el * SMF * N;
  float2 *const sp = reinterpret_cast<float2 *>(sf);
  const float invR = __frcp_rn(Rgas);
  // P = 3, one element per block: the element's J^-1 and gpvol (2560 B),
  // slot positions and mu_e (256 B each) are contiguous and 16-byte aligned
  // in global memory, and land with the stage's layout (stride N = NTB), so
  // one thread moves them with bulk copies; the gathered state and
  // projections stay per-thread cp.async.
  constexpr bool BULK = (P == 3 && EPB == 1);
  __shared__ __align__(8) unsigned long long mbar[2];
  unsigned phases = 0u;  // bit b: parity of the next completion of mbar[b]
  if (BULK && tid == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (BULK) __syncthreads();

  auto node_of = [&](long long g) -> int {
    const long long e = g * EPB + el;
    return (g < ngroups && e < m.nelem && t < N) ? m.conn[e * N + t] : -1;
  };
  // this thread's copies for group g into stage stg (nd: its node, -1: none)
  auto issue = [&](float *stg, long long g, int nd) {
    if (BULK && tid == 0 && g < ngroups) {
      const long long e0 = g;  // one element per block
      unsigned long long *bar = &mbar[stg == dsm ? 0 : 1];
      const bool mus = DIFF && A.musgs_t;
      const unsigned bytes = (10u + 1u + (DIFF ? 1u : 0u) + (mus ? 1u : 0u)) * N * 4u;
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // earlier reads of this stage first
      mbar_expect_tx(bar, bytes);
      bulk_g2s(stg + L::O_GEO, m.geo + e0 * 10 * N, 10u * N * 4u, bar);
      bulk_g2s(stg + L::O_POS, m.slot_pos + e0 * N, N * 4u, bar);
      if (DIFF) bulk_g2s(stg + L::O_MUE, A.mue_t + e0 * N, N * 4u, bar);
      if (mus) bulk_g2s(stg + L::O_MUS, A.musgs_t + e0 * N, N * 4u, bar);
    }
    if (nd < 0) return;
    const long long e = g * EPB + el;
    if (IN == IN_CONS) {
      cp_async4(stg + L::O_IN + 0 * NTB + tid, A.rho + nd);
      cp_async4(stg + L::O_IN + 1 * NTB + tid, A.q + nd);
      cp_async4(stg + L::O_IN + 2 * NTB + tid, A.q + nd + NP);
      cp_async4(stg + L::O_IN + 3 * NTB + tid, A.q + nd + 2 * NP);
      cp_async4(stg + L::O_IN + 4 * NTB + tid, A.E + nd);
    } else if (IN == IN_PRIM) {
      cp_async4(stg + L::O_IN + 0 * NTB + tid, A.rho + nd);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        cp_async4(stg + L::O_IN + (1 + c) * NTB + tid, A.u + nd + c * NP);
        cp_async4(stg + L::O_IN + (4 + c) * NTB + tid, A.q + nd + c * NP);
      }
      cp_async4(stg + L::O_IN + 7 * NTB + tid, A.pr + nd);
      cp_async4(stg + L::O_IN + 8 * NTB + tid, A.E + nd);
    } else {
      cp_async4(stg + L::O_IN + 0 * NTB + tid, A.rho + nd);
      cp_async4(stg + L::O_IN + 1 * NTB + tid, (A.rho_n ? A.rho_n : A.rho) + nd);
#pragma unroll
      for (int c = 0; c < 3; ++c) cp_async4(stg + L::O_IN + (2 + c) * NTB + tid, A.u + nd + c * NP);
      cp_async4(stg + L::O_IN + 5 * NTB + tid, A.Tem + nd);
      cp_async4(stg + L::O_IN + 6 * NTB + tid, A.mu_fluid + nd);
    }
    if (!BULK) {
      const float *g0 = m.geo + e * 10 * N + t;
#pragma unroll
      for (int c = 0; c < 10; ++c) cp_async4(stg + L::O_GEO + c * NTB + tid, g0 + c * N);
      cp_async4(stg + L::O_POS + tid, m.slot_pos + e * N + t);
    }
    if (DIFF) {
      if (!BULK) {
        cp_async4(stg + L::O_MUE + tid, A.mue_t + e * N + t);
        if (A.musgs_t) cp_async4(stg + L::O_MUS + tid, A.musgs_t + e * N + t);
      }
      if (LPS) {
#pragma unroll
        for (int c = 0; c < 3; ++c) cp_async16(stg + L::O_PROJ + tid * 12 + 4 * c, A.proj12 + (long long)nd * 12 + 4 * c);
      }
    }
  };

  long long g = blockIdx.x;
  issue(dsm, g, node_of(g));
  cp_async_commit();
  int nd_next = node_of(g + G);
  for (int buf = 0; g < ngroups; g += G, buf ^= 1) {
    const float *cur = dsm + buf * L::STAGE;
    float *nxt = dsm + (buf ^ 1) * L::STAGE;
    cp_async_wait_all();  // this thread's copies of the current group have landed
    bool bulk_ok = true;
    if (BULK) {  // and the block's bulk copies of it
      bulk_ok = mbar_wait(&mbar[buf], (phases >> buf) & 1u);
      phases ^= 1u << buf;
    }
    const long long e = g * EPB + el;
    const bool active = (e < m.nelem) && (t < N);
    const float *gm = cur + L::O_GEO + tid;  // J^-1 (9 components) and gpvol, stride NTB
    NodeQ s;
    float mu = 0.f, rhon_in = 0.f, H = 0.f, rH = 0.f;
    if (active) {
      const float *in = cur + L::O_IN + tid;
      if (IN == IN_CONS) {
        eos_fast(ph, invR, A.mu_factor, in[0], in[NTB], in[2 * NTB], in[3 * NTB], in[4 * NTB], s);
        mu = s.mu;
      } else if (IN == IN_PRIM) {
        s.rho = in[0];
        s.u0 = in[NTB]; s.u1 = in[2 * NTB]; s.u2 = in[3 * NTB];
        s.q0 = in[4 * NTB]; s.q1 = in[5 * NTB]; s.q2 = in[6 * NTB];
        s.p = in[7 * NTB]; s.h = in[8 * NTB]; s.T = 0.f;
      } else {
        s.rho = in[0];
        rhon_in = in[NTB];
        s.u0 = in[2 * NTB]; s.u1 = in[3 * NTB]; s.u2 = in[4 * NTB];
        s.T = in[5 * NTB];
        mu = in[6 * NTB];
        s.q0 = s.q1 = s.q2 = 0.f; s.p = 0.f; s.h = 0.f;
      }
      sp[PB_U01 * N + t] = make_float2(s.u0, s.u1);
      sp[PB_U2R * N + t] = make_float2(s.u2, s.rho);
      if (CONV) {
        // H = h + k with k = |u|^2/2: the reference's split-form energy
        // terms for E:=h and for k enter with the same 1/4 weight, so their
        // flux fields are combined (rho*h*u + rho*k*u = rho*H*u, h*u + k*u = H*u).
        float kk = s.u0 * s.u0 * 0.5f;
        kk = kk + s.u1 * s.u1 * 0.5f;
        kk = kk + s.u2 * s.u2 * 0.5f;
        H = s.h + kk;
        rH = s.rho * H;
        sp[PB_Q01 * N + t] = make_float2(s.q0, s.q1);
        sp[PB_Q2P * N + t] = make_float2(s.q2, s.p);
        sp[PB_HRH * N + t] = make_float2(H, rH);
      }
      if (DIFF) sp[PB_T * N + t] = make_float2(s.T, 0.f);
    }
    // staged pairs visible; every thread is done with the other stage
    if (!__syncthreads_and(bulk_ok)) {
      if (tid == 0) *(volatile int *)A.err = 1;  // a bulk copy never completed: stop, nothing else is in flight
      return;
    }
    if (g + G < ngroups) issue(nxt, g + G, nd_next);
    cp_async_commit();
    nd_next = node_of(g + 2 * G);  // consumed one group later

    float res[5] = {0.f, 0.f, 0.f, 0.f, 0.f};  // mass, energy, mom x,y,z
    float gradRho[3] = {0.f, 0.f, 0.f}, gradT[3] = {0.f, 0.f, 0.f};
    float gradU[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
    if (active) {
      // Physical-space sums, accumulated one reference direction d at a
      // time: d_a f = sum_d He(a,d) d_d f, and every convective term is
      // linear in the derivatives, so each direction's derivatives are
      // folded in as soon as they are formed.  Advective terms use the
      // contravariant velocities U_d = sum_b u_b He(b,d), Q_d = sum_b q_b He(b,d).
      float divQ = 0.f, QdH = 0.f, UdRH = 0.f, divRHu = 0.f, divHu = 0.f;
      float UdQ[3] = {0.f, 0.f, 0.f}, gradP[3] = {0.f, 0.f, 0.f}, divF[3] = {0.f, 0.f, 0.f},
            divG[3] = {0.f, 0.f, 0.f};
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const int cd = d == 0 ? i : (d == 1 ? j : k);
        const int stride = d == 0 ? 1 : (d == 1 ? N1 : N1 * N1);
        const int base = t - cd * stride;
        float Dd[N1];
#pragma unroll
        for (int q = 0; q < N1; ++q) Dd[q] = m.Dnat[cd * N1 + q];
        const float2 z2 = make_float2(0.f, 0.f);
        float2 aU01 = z2, aU2R = z2, aQ01 = z2, aQ2P = z2, aHRH = z2, aT = z2;
        float2 aF0 = z2, aF1 = z2, aF2 = z2, aG0 = z2, aG1 = z2, aG2 = z2, aR0 = z2, aR1 = z2, aR2 = z2;
#pragma unroll
        for (int ss = 0; ss < N1; ++ss) {
          const int mm = ref_order<P>(ss);  // the reference's 1-D summation order
          const float2 D2 = make_float2(Dd[mm], Dd[mm]);
          const int tm = base + mm * stride;
          const float2 u01 = sp[PB_U01 * N + tm], u2r = sp[PB_U2R * N + tm];
          aU01 = __ffma2_rn(D2, u01, aU01);
          aU2R = __ffma2_rn(D2, u2r, aU2R);
          if (DIFF) aT = __ffma2_rn(D2, sp[PB_T * N + tm], aT);
          if (CONV) {
            const float2 q01 = sp[PB_Q01 * N + tm], q2p = sp[PB_Q2P * N + tm], hrh = sp[PB_HRH * N + tm];
            aQ01 = __ffma2_rn(D2, q01, aQ01);
            aQ2P = __ffma2_rn(D2, q2p, aQ2P);
            aHRH = __ffma2_rn(D2, hrh, aHRH);
            const float u0 = u01.x, u1 = u01.y, u2 = u2r.x, q0 = q01.x, q1 = q01.y, q2 = q2p.x;
            aF0 = __ffma2_rn(D2, make_float2(q0 * u0, q0 * u1), aF0);
            aF1 = __ffma2_rn(D2, make_float2(q0 * u2, q1 * u1), aF1);
            aF2 = __ffma2_rn(D2, make_float2(q1 * u2, q2 * u2), aF2);
            aG0 = __ffma2_rn(D2, make_float2(u0 * u0, u0 * u1), aG0);
            aG1 = __ffma2_rn(D2, make_float2(u0 * u2, u1 * u1), aG1);
            aG2 = __ffma2_rn(D2, make_float2(u1 * u2, u2 * u2), aG2);
            aR0 = __ffma2_rn(D2, make_float2(hrh.y * u0, hrh.y * u1), aR0);
            aR1 = __ffma2_rn(D2, make_float2(hrh.y * u2, hrh.x * u2), aR1);
            aR2 = __ffma2_rn(D2, make_float2(hrh.x * u0, hrh.x * u1), aR2);
          }
        }
        const float h[3] = {gm[(0 + 3 * d) * NTB], gm[(1 + 3 * d) * NTB], gm[(2 + 3 * d) * NTB]};
        const float dU[3] = {aU01.x, aU01.y, aU2R.x};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          gradRho[a] = gradRho[a] + h[a] * aU2R.y;
          if (DIFF) gradT[a] = gradT[a] + h[a] * aT.x;
#pragma unroll
          for (int b = 0; b < 3; ++b) gradU[a][b] = gradU[a][b] + h[b] * dU[a];
        }
        if (CONV) {
          const float dQ[3] = {aQ01.x, aQ01.y, aQ2P.x};
          // d_d of the symmetric F_ab = q_a u_b and G_ab = u_a u_b (a <= b)
          const float dF[3][3] = {{aF0.x, aF0.y, aF1.x}, {aF0.y, aF1.y, aF2.x}, {aF1.x, aF2.x, aF2.y}};
          const float dG[3][3] = {{aG0.x, aG0.y, aG1.x}, {aG0.y, aG1.y, aG2.x}, {aG1.x, aG2.x, aG2.y}};
          const float dRHu[3] = {aR0.x, aR0.y, aR1.x}, dHu[3] = {aR2.x, aR2.y, aR1.y};
          const float Ud = h[0] * s.u0 + h[1] * s.u1 + h[2] * s.u2;
          const float Qd = h[0] * s.q0 + h[1] * s.q1 + h[2] * s.q2;
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            divQ = divQ + h[a] * dQ[a];
            UdQ[a] = UdQ[a] + Ud * dQ[a];
            gradP[a] = gradP[a] + h[a] * aQ2P.y;
            divRHu = divRHu + h[a] * dRHu[a];
            divHu = divHu + h[a] * dHu[a];
#pragma unroll
            for (int b = 0; b < 3; ++b) {
              divF[a] = divF[a] + h[b] * dF[a][b];
              divG[a] = divG[a] + h[b] * dG[a][b];
            }
          }
          QdH = QdH + Qd * aHRH.x;
          UdRH = UdRH + Ud * aHRH.y;
        }
      }
      if (CONV) {
        const float gv = gm[9 * NTB];
        const float u[3] = {s.u0, s.u1, s.u2}, q[3] = {s.q0, s.q1, s.q2};
        const float divU = gradU[0][0] + gradU[1][1] + gradU[2][2];
        float ugR = 0.f;
#pragma unroll
        for (int a = 0; a < 3; ++a) ugR = ugR + u[a] * gradRho[a];
        const float Rmass = 0.5f * (divQ + s.rho * divU) + 0.5f * ugR;
        const float Rener =
            0.25f * (divRHu + H * divQ + rH * divU + s.rho * divHu) + 0.25f * (QdH + UdRH + H * ugR);
        res[0] = A.fact_c * (gv * Rmass);
        res[1] = A.fact_c * (gv * Rener);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          float QdU = 0.f;
#pragma unroll
          for (int b = 0; b < 3; ++b) QdU = QdU + q[b] * gradU[a][b];
          const float Rmom = 0.25f * (divF[a] + u[a] * divQ + q[a] * divU + s.rho * divG[a]) + gradP[a] +
                             0.25f * (u[a] * ugR + QdU + UdQ[a]);
          res[2 + a] = A.fact_c * (gv * Rmom);
        }
      }
    }

    if (DIFF) {
      // Fluxes at this Gauss point (first Gauss-point loop of
      // full_diff_stab_ijk, elem_stab.f90:296-385, or of full_diffusion_ijk,
      // elem_diffu.f90:99-164), then their contravariant components
      // gpvol * sum_i He(i,d) F_i, staged for the weak divergence.
      float C[NC][3];
      float nu_e = 0.f, kappa_e = 0.f;
      if (active) {
        const float mue = cur[L::O_MUE + tid];
        const float musgs = A.musgs_t ? cur[L::O_MUS + tid] : 0.f;
        const float rhon = IN == IN_DIFF ? rhon_in : s.rho;
        nu_e = ph.c_rho * mue * __frcp_rn(rhon);
        const float mu_fgp = mu + rhon * musgs;
        const float mu_egp = mue;
        kappa_e = mu * ph.cp_pr + ph.c_ener * mue * ph.cp_pr + ph.Cp * rhon * musgs * (1.f / 0.9f);
        const float divU = gradU[0][0] + gradU[1][1] + gradU[2][2];
        const float u[3] = {s.u0, s.u1, s.u2};
        float tau[3][3];
        float Fx[3], Fy[3], Fz[3], FT[3], FR[3];
        if (LPS) {
          const float ts = A.tau_stab[e];
#pragma unroll
          for (int a = 0; a < 3; ++a) {
#pragma unroll
            for (int b = 0; b < 3; ++b) tau[a][b] = gradU[a][b] + gradU[b][a];
            tau[a][a] = tau[a][a] - ph.twoThirds * divU;
          }
          const float4 *pj = reinterpret_cast<const float4 *>(cur + L::O_PROJ + tid * 12);
          const float4 p0 = pj[0], p1 = pj[1], p2 = pj[2];
          const float PX[3] = {p0.x, p0.y, p0.z}, PY[3] = {p0.y, p0.w, p1.x}, PZ[3] = {p0.z, p1.x, p1.y};
          const float PM[3] = {p1.z, p1.w, p2.x}, PE[3] = {p2.y, p2.z, p2.w};
          const float cl = -ph.c_lps * ts;
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            Fx[d] = cl * (PX[d] - tau[0][d]) * rhon;
            Fy[d] = cl * (PY[d] - tau[1][d]) * rhon;
            Fz[d] = cl * (PZ[d] - tau[2][d]) * rhon;
            FT[d] = cl * (PE[d] - gradT[d]) * rhon * ph.cp_pr;
            FR[d] = cl * (PM[d] - gradRho[d]);
          }
        }
        float tauU[3] = {0.f, 0.f, 0.f};
        const float mt = mu_fgp + mu_egp;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
#pragma unroll
          for (int b = 0; b < 3; ++b) {
            tauU[a] = tauU[a] + mt * (gradU[a][b] + gradU[b][a]) * u[b];
            tau[a][b] = mt * (gradU[a][b] + gradU[b][a]);
          }
          tauU[a] = tauU[a] - (mu_fgp)*ph.twoThirds * divU * u[a];
          tau[a][a] = tau[a][a] - (mu_fgp)*ph.twoThirds * divU;
        }
        if (LPS) {
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            Fx[d] = Fx[d] + tau[0][d];
            Fy[d] = Fy[d] + tau[1][d];
            Fz[d] = Fz[d] + tau[2][d];
            FT[d] = FT[d] + kappa_e * gradT[d] + tauU[d];
            FR[d] = FR[d] + nu_e * gradRho[d];
          }
        } else {
          // full_diffusion_ijk scales the neighbours' grad rho and grad T by
          // nu_e and kappa_e of the output Gauss point: stage them unscaled.
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            Fx[d] = tau[0][d];
            Fy[d] = tau[1][d];
            Fz[d] = tau[2][d];
            FT[d] = tauU[d];
            FR[d] = gradRho[d];
          }
        }
        const float gv = gm[9 * NTB];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const float h0 = gm[(0 + 3 * d) * NTB], h1 = gm[(1 + 3 * d) * NTB], h2 = gm[(2 + 3 * d) * NTB];
          C[0][d] = gv * (h0 * FR[0] + h1 * FR[1] + h2 * FR[2]);
          C[1][d] = gv * (h0 * FT[0] + h1 * FT[1] + h2 * FT[2]);
          C[2][d] = gv * (h0 * Fx[0] + h1 * Fx[1] + h2 * Fx[2]);
          C[3][d] = gv * (h0 * Fy[0] + h1 * Fy[1] + h2 * Fy[2]);
          C[4][d] = gv * (h0 * Fz[0] + h1 * Fz[1] + h2 * Fz[2]);
          if (!LPS) C[NC - 1][d] = gv * (h0 * gradT[0] + h1 * gradT[1] + h2 * gradT[2]);
        }
      }
      __syncthreads();  // all reads of the staged pairs are done
      if (active) {
#pragma unroll
        for (int q = 0; q < NC; ++q)
#pragma unroll
          for (int d = 0; d < 3; ++d) sf[(q * 3 + d) * N + t] = C[q][d];
      }
      __syncthreads();
      if (active) {
        // Weak divergence: sum_d sum_m D[m][i_d] C_d(node with d-index m).
        float Dci[N1], Dcj[N1], Dck[N1];
#pragma unroll
        for (int q = 0; q < N1; ++q) { Dci[q] = m.Dnat[q * N1 + i]; Dcj[q] = m.Dnat[q * N1 + j]; Dck[q] = m.Dnat[q * N1 + k]; }
        float wd[NC];
#pragma unroll
        for (int q = 0; q < NC; ++q) {
          const float *c0 = sf + (q * 3 + 0) * N, *c1 = sf + (q * 3 + 1) * N, *c2 = sf + (q * 3 + 2) * N;
          float acc = 0.f;
#pragma unroll
          for (int ss = 0; ss < N1; ++ss) {
            const int mm = ref_order<P>(ss);
            acc = fmaf(Dci[mm], c0[mm + N1 * j + N1 * N1 * k], acc);
            acc = fmaf(Dcj[mm], c1[i + N1 * mm + N1 * N1 * k], acc);
            acc = fmaf(Dck[mm], c2[i + N1 * j + N1 * N1 * mm], acc);
          }
          wd[q] = acc;
        }
        if (LPS) {
#pragma unroll
          for (int q = 0; q < 5; ++q) res[q] = res[q] + A.fact_d * wd[q];
        } else {
          res[0] = res[0] + A.fact_d * (nu_e * wd[0]);
          res[1] = res[1] + A.fact_d * (wd[1] + kappa_e * wd[NC - 1]);
#pragma unroll
          for (int q = 2; q < 5; ++q) res[q] = res[q] + A.fact_d * wd[q];
        }
      }
    }
    if (active) {
      // pass-B slots, node-sorted: [E*N] float4 (mass, energy, mom x, mom y),
      // then [E*N] mom z
      const long long sp5 = __float_as_int(cur[L::O_POS + tid]);
      reinterpret_cast<float4 *>(slots)[sp5] = make_float4(res[0], res[1], res[2], res[3]);
      slots[(long long)m.nelem * N * 4 + sp5] = res[4];
    }
    __syncthreads();  // the staging area is free for the next group
  }
  cp_async_wait_all();
}

// ---------------------------------------------------------------------
// Node-centric assembly: out_f(p) = scale(p) * (base_f(p) + sum of the
// node's slot contributions), Kahan-compensated, slots visited in element
// order (deterministic).  W = slot width, NFO = fields summed.
// Output layout: SoA (reference, out[f][p] = out + f*npoin) when AOS is
// false; node-major [p][W] when true.
// ---------------------------------------------------------------------
struct OutPtrs {
  float *p[16];
};

template <int W, int NFO, bool AOS>
__global__ void k_gather(MeshDev m, const float *__restrict__ slots, float *__restrict__ out,
                         OutPtrs out_soa, int accumulate, int use_invMl) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m.npoin) return;
  constexpr int MS = W >= 12 ? 1 : 4;  // slots whose loads are issued together (registers permitting)
  float sum[NFO], cmp[NFO];
#pragma unroll
  for (int f = 0; f < NFO; ++f) {
    sum[f] = (accumulate && !AOS) ? out_soa.p[f][p] : 0.f;
    cmp[f] = 0.f;
  }
  const int b = m.slot_ptr[p], en = m.slot_ptr[p + 1];
  for (int s0 = b; s0 < en; s0 += MS) {
    int id[MS];
#pragma unroll
    for (int k = 0; k < MS; ++k) id[k] = s0 + k < en ? m.slot_idx[s0 + k] : -1;
    float4 v[MS][W / 4];
#pragma unroll
    for (int k = 0; k < MS; ++k)
#pragma unroll
      for (int c = 0; c < W / 4; ++c)
        v[k][c] = id[k] >= 0 ? reinterpret_cast<const float4 *>(slots + (long long)id[k] * W)[c]
                             : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int k = 0; k < MS; ++k) {
      if (id[k] < 0) break;
      float x[W];
#pragma unroll
      for (int c = 0; c < W / 4; ++c) {
        x[4 * c] = v[k][c].x; x[4 * c + 1] = v[k][c].y; x[4 * c + 2] = v[k][c].z; x[4 * c + 3] = v[k][c].w;
      }
#pragma unroll
      for (int f = 0; f < NFO; ++f) {  // Kahan summation
        const float y = x[f] - cmp[f];
        const float tt = sum[f] + y;
        cmp[f] = (tt - sum[f]) - y;
        sum[f] = tt;
      }
    }
  }
  const float sc = use_invMl ? m.invMl[p] : 1.f;
  if (AOS) {
    float4 *o = reinterpret_cast<float4 *>(out + p * W);
    float r[W];
#pragma unroll
    for (int f = 0; f < W; ++f) r[f] = f < NFO ? sum[f] * sc : 0.f;
#pragma unroll
    for (int c = 0; c < W / 4; ++c) o[c] = make_float4(r[4 * c], r[4 * c + 1], r[4 * c + 2], r[4 * c + 3]);
  } else {
#pragma unroll
    for (int f = 0; f < NFO; ++f) out_soa.p[f][p] = sum[f] * sc;
  }
}

// ---------------------------------------------------------------------
// Assembly from node-sorted slots (written at slot_pos by k_rhs): node p's
// contributions are slots slot_ptr[p] .. slot_ptr[p+1]-1, in element
// order, so a warp streams one contiguous range with no index loads.  Same
// Kahan-compensated order as k_gather (bit-identical sums).
// ---------------------------------------------------------------------
// The 5 residuals from node-sorted pass-B slots into the reference's SoA
// outputs (optionally accumulated onto them), x invMl.
static __global__ void k_gather_sorted_res5(MeshDev m, const float *__restrict__ slots, long long zoff, OutPtrs out_soa,
                                     int accumulate, int use_invMl) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m.npoin) return;
  const float *sz = slots + 4 * zoff;
  const float4 *s4 = reinterpret_cast<const float4 *>(slots);
  float sum[5], cmp[5];
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    sum[f] = accumulate ? out_soa.p[f][p] : 0.f;
    cmp[f] = 0.f;
  }
  const int b = m.slot_ptr[p], en = m.slot_ptr[p + 1];
  const float sc = use_invMl ? m.invMl[p] : 1.f;
  for (int s = b; s < en; ++s) {
    const float4 v = s4[s];
    const float x[5] = {v.x, v.y, v.z, v.w, sz[s]};
#pragma unroll
    for (int f = 0; f < 5; ++f) {
      const float y = x[f] - cmp[f];
      const float tt = sum[f] + y;
      cmp[f] = (tt - sum[f]) - y;
      sum[f] = tt;
    }
  }
#pragma unroll
  for (int f = 0; f < 5; ++f) out_soa.p[f][p] = sum[f] * sc;
}

}  // namespace sod
