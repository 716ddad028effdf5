// Element kernels of the compressible RHS for sm_100a.
//
// Layout (built once by sod_gpu_init):
//   conn[e][t]        0-based node id of tensor position t = i + n1*j + n1^2*k
//                     (natural 1-D GLL order, xi ascending)
//   geo[e][c][t]      c = 0..8: He(i,j) at c = i + 3j (= d xi_j / d x_i);
//                     c = 9: gpvol
//   slots[(e*N+t)*W]  per element-node contributions, W floats (padded)
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
#ifndef SOD_RHS_MINB
#define SOD_RHS_MINB 7
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
#if SOD_VEC_XI
  if constexpr (P == 3) {
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
    return;
  }
#endif
#pragma unroll
  for (int s = 0; s < N1; ++s) {
    const int m = ref_order<P>(s);
    g0 = fmaf(Di[m], f[m + N1 * j + N1 * N1 * k], g0);
    g1 = fmaf(Dj[m], f[i + N1 * m + N1 * N1 * k], g1);
    g2 = fmaf(Dk[m], f[i + N1 * j + N1 * N1 * m], g2);
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

// ---------------------------------------------------------------------
// Pass A: LPS projections (full_proj_ijk, elem_stab.f90:474-562).  Writes
// gpvol * {tau00, tau01, tau02, tau11, tau12, tau22, grad rho (3), grad T
// (3)} per element node into slots of width 12.  tau = grad u + grad u^T
// - 2/3 div u I is symmetric (tau_ab and tau_ba are the same FP32 sum), so
// the reference's ProjMX/MY/MZ rows are read back from its 6 entries.
// Input: conserved state (SoA, reference layout) -> EOS in registers, or
// primitive rho/u/T (prim = true).
// ---------------------------------------------------------------------
template <int P, int EPB, bool PRIM>
__global__ void __launch_bounds__(EPB *Cfg<P>::NT)
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
      eos(ph, Rgas, 1.f, a0[node], a1[node], a1[node + NP], a1[node + 2 * NP], a2[node], s);
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
};

// Shared-memory field indices of pass B.
enum {
  F_RHO = 0, F_P, F_H, F_RH, F_T, F_U0, F_U1, F_U2, F_Q0, F_Q1, F_Q2,
  F_RHU0, F_RHU1, F_RHU2, F_HU0, F_HU1, F_HU2,
  F_F00, F_F01, F_F02, F_F11, F_F12, F_F22,
  F_G00, F_G01, F_G02, F_G11, F_G12, F_G22,
  NF_B
};

__device__ __forceinline__ int sym_idx(int a, int b) {
  // (0,0)->0 (0,1)->1 (0,2)->2 (1,1)->3 (1,2)->4 (2,2)->5
  int lo = a < b ? a : b, hi = a < b ? b : a;
  return lo == 0 ? hi : (lo == 1 ? 2 + hi : 5);
}

template <int P, int EPB, int MODE, int IN>
__global__ void __launch_bounds__(EPB *Cfg<P>::NT, SOD_RHS_MINB)
k_rhs(MeshDev m, Phys ph, float Rgas, RhsArgs A, float *__restrict__ slots) {
  constexpr int N1 = Cfg<P>::N1, N = Cfg<P>::N, NT = Cfg<P>::NT;
  constexpr bool CONV = (MODE & MODE_CONV) != 0;
  constexpr bool DIFF = (MODE & MODE_DIFF) != 0;
  __shared__ __align__(16) float sm[EPB][NF_B][N];
  const int el = threadIdx.x / NT, t = threadIdx.x % NT;
  const long long e = (long long)blockIdx.x * EPB + el;
  const bool active = (e < m.nelem) && (t < N);
  const long long NP = m.npoin;
  NodeQ s;
  float mu = 0.f, rhon_in = 0.f;
  int node = 0;
  float He[9], gv = 0.f;
  if (active) {
    node = m.conn[e * N + t];
    // geometry loads issued before the staging barrier (independent of it)
    const float *g = m.geo + e * 10 * N + t;
#pragma unroll
    for (int c = 0; c < 9; ++c) He[c] = g[c * N];
    gv = g[9 * N];
    if (IN == IN_CONS) {
      eos(ph, Rgas, A.mu_factor, A.rho[node], A.q[node], A.q[node + NP], A.q[node + 2 * NP], A.E[node], s);
      mu = s.mu;
    } else if (IN == IN_PRIM) {
      s.rho = A.rho[node];
      s.u0 = A.u[node]; s.u1 = A.u[node + NP]; s.u2 = A.u[node + 2 * NP];
      s.q0 = A.q[node]; s.q1 = A.q[node + NP]; s.q2 = A.q[node + 2 * NP];
      s.p = A.pr[node]; s.h = A.E[node]; s.T = 0.f;
    } else {
      s.rho = A.rho[node];
      rhon_in = A.rho_n ? A.rho_n[node] : s.rho;
      s.u0 = A.u[node]; s.u1 = A.u[node + NP]; s.u2 = A.u[node + 2 * NP];
      s.T = A.Tem[node];
      mu = A.mu_fluid[node];
      s.q0 = s.q1 = s.q2 = 0.f; s.p = 0.f; s.h = 0.f;
    }
    float(*f)[N] = sm[el];
    f[F_RHO][t] = s.rho;
    f[F_U0][t] = s.u0; f[F_U1][t] = s.u1; f[F_U2][t] = s.u2;
    if (DIFF) f[F_T][t] = s.T;
    if (CONV) {
      // H = h + k with k = |u|^2/2: the reference's split-form energy terms
      // for E:=h and for k enter with the same 1/4 weight, so their flux
      // fields are combined (rho*h*u + rho*k*u = rho*H*u, h*u + k*u = H*u).
      float kk = s.u0 * s.u0 * 0.5f;
      kk = kk + s.u1 * s.u1 * 0.5f;
      kk = kk + s.u2 * s.u2 * 0.5f;
      const float H = s.h + kk, rH = s.rho * H;
      f[F_P][t] = s.p; f[F_H][t] = H; f[F_RH][t] = rH;
      f[F_Q0][t] = s.q0; f[F_Q1][t] = s.q1; f[F_Q2][t] = s.q2;
      f[F_RHU0][t] = rH * s.u0; f[F_RHU1][t] = rH * s.u1; f[F_RHU2][t] = rH * s.u2;
      f[F_HU0][t] = H * s.u0; f[F_HU1][t] = H * s.u1; f[F_HU2][t] = H * s.u2;
      f[F_F00][t] = s.q0 * s.u0; f[F_F01][t] = s.q0 * s.u1; f[F_F02][t] = s.q0 * s.u2;
      f[F_F11][t] = s.q1 * s.u1; f[F_F12][t] = s.q1 * s.u2; f[F_F22][t] = s.q2 * s.u2;
      f[F_G00][t] = s.u0 * s.u0; f[F_G01][t] = s.u0 * s.u1; f[F_G02][t] = s.u0 * s.u2;
      f[F_G11][t] = s.u1 * s.u1; f[F_G12][t] = s.u1 * s.u2; f[F_G22][t] = s.u2 * s.u2;
    }
  }
  __syncthreads();
  const int i = t % N1, j = (t / N1) % N1, k = t / (N1 * N1);
  float Di[N1], Dj[N1], Dk[N1];
  float res[5] = {0.f, 0.f, 0.f, 0.f, 0.f};  // mass, energy, mom x,y,z
  float gradRho[3], gradU[3][3];
  if (active) {
#pragma unroll
    for (int q = 0; q < N1; ++q) { Di[q] = m.Dnat[i * N1 + q]; Dj[q] = m.Dnat[j * N1 + q]; Dk[q] = m.Dnat[k * N1 + q]; }
    float(*f)[N] = sm[el];
    float a0, a1, a2;
    iso_grad<P>(f[F_RHO], i, j, k, Di, Dj, Dk, a0, a1, a2);
#pragma unroll
    for (int a = 0; a < 3; ++a) gradRho[a] = He[a] * a0 + He[a + 3] * a1 + He[a + 6] * a2;
    float gU[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) iso_grad<P>(f[F_U0 + c], i, j, k, Di, Dj, Dk, gU[c][0], gU[c][1], gU[c][2]);
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) gradU[a][b] = He[b] * gU[a][0] + He[b + 3] * gU[a][1] + He[b + 6] * gU[a][2];
    const float divU = gradU[0][0] + gradU[1][1] + gradU[2][2];
    const float u[3] = {s.u0, s.u1, s.u2};

    if (CONV) {
      const float q[3] = {s.q0, s.q1, s.q2};
      float gradP[3], gradH[3], gradRH[3], gradQ[3][3];
      iso_grad<P>(f[F_P], i, j, k, Di, Dj, Dk, a0, a1, a2);
#pragma unroll
      for (int a = 0; a < 3; ++a) gradP[a] = He[a] * a0 + He[a + 3] * a1 + He[a + 6] * a2;
      iso_grad<P>(f[F_H], i, j, k, Di, Dj, Dk, a0, a1, a2);
#pragma unroll
      for (int a = 0; a < 3; ++a) gradH[a] = He[a] * a0 + He[a + 3] * a1 + He[a + 6] * a2;
      iso_grad<P>(f[F_RH], i, j, k, Di, Dj, Dk, a0, a1, a2);
#pragma unroll
      for (int a = 0; a < 3; ++a) gradRH[a] = He[a] * a0 + He[a + 3] * a1 + He[a + 6] * a2;
      float gQ[3][3];
#pragma unroll
      for (int c = 0; c < 3; ++c) iso_grad<P>(f[F_Q0 + c], i, j, k, Di, Dj, Dk, gQ[c][0], gQ[c][1], gQ[c][2]);
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) gradQ[a][b] = He[b] * gQ[a][0] + He[b + 3] * gQ[a][1] + He[b + 6] * gQ[a][2];
      // divergences of vector fields: sum_i sum_j He(i,j) d_j V_i
      float divRHu = 0.f, divHu = 0.f;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        iso_grad<P>(f[F_RHU0 + c], i, j, k, Di, Dj, Dk, a0, a1, a2);
        divRHu += He[c] * a0 + He[c + 3] * a1 + He[c + 6] * a2;
        iso_grad<P>(f[F_HU0 + c], i, j, k, Di, Dj, Dk, a0, a1, a2);
        divHu += He[c] * a0 + He[c + 3] * a1 + He[c + 6] * a2;
      }
      // div of the symmetric tensors F = q (x) u and G = u (x) u:
      // divF_a = sum_b sum_c He(b,c) d_c F_ab
      float divF[3] = {0.f, 0.f, 0.f}, divG[3] = {0.f, 0.f, 0.f};
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = a; b < 3; ++b) {
          const int sidx = sym_idx(a, b);
          iso_grad<P>(f[F_F00 + sidx], i, j, k, Di, Dj, Dk, a0, a1, a2);
          const float dfb = He[b] * a0 + He[b + 3] * a1 + He[b + 6] * a2;  // d_b F_ab
          const float dfa = He[a] * a0 + He[a + 3] * a1 + He[a + 6] * a2;  // d_a F_ab
          divF[a] += dfb;
          if (b != a) divF[b] += dfa;
          iso_grad<P>(f[F_G00 + sidx], i, j, k, Di, Dj, Dk, a0, a1, a2);
          const float dgb = He[b] * a0 + He[b + 3] * a1 + He[b + 6] * a2;
          const float dga = He[a] * a0 + He[a + 3] * a1 + He[a + 6] * a2;
          divG[a] += dgb;
          if (b != a) divG[b] += dga;
        }
      const float divQ = gradQ[0][0] + gradQ[1][1] + gradQ[2][2];
      const float H = f[F_H][t], rH = f[F_RH][t];
      float Rmass = 0.5f * (divQ + s.rho * divU);
      float Rener = 0.25f * (divRHu + H * divQ + rH * divU + s.rho * divHu);
      float Rmom[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        Rmom[a] = 0.25f * (divF[a] + u[a] * divQ + q[a] * divU + s.rho * divG[a]) + gradP[a];
        Rmass = Rmass + 0.5f * (u[a] * gradRho[a]);
        Rener = Rener + 0.25f * (q[a] * gradH[a] + u[a] * gradRH[a] + H * u[a] * gradRho[a]);
#pragma unroll
        for (int b = 0; b < 3; ++b)
          Rmom[a] = Rmom[a] + 0.25f * (u[a] * u[b] * gradRho[b] + q[b] * gradU[a][b] + u[b] * gradQ[a][b]);
      }
      res[0] = A.fact_c * (gv * Rmass);
      res[1] = A.fact_c * (gv * Rener);
      res[2] = A.fact_c * (gv * Rmom[0]);
      res[3] = A.fact_c * (gv * Rmom[1]);
      res[4] = A.fact_c * (gv * Rmom[2]);
    }
  }

  if (DIFF) {
    constexpr bool LPS = (MODE & MODE_NOLPS) == 0;
    constexpr int NC = LPS ? 5 : 6;  // staged contravariant flux fields
    // Fluxes at this Gauss point (first Gauss-point loop of
    // full_diff_stab_ijk, elem_stab.f90:296-385, or of full_diffusion_ijk,
    // elem_diffu.f90:99-164), then their contravariant components
    // gpvol * sum_i He(i,d) F_i, staged for the weak divergence.
    float C[NC][3];
    float nu_e = 0.f, kappa_e = 0.f;
    if (active) {
      float(*f)[N] = sm[el];
      float a0, a1, a2, gradT[3];
      iso_grad<P>(f[F_T], i, j, k, Di, Dj, Dk, a0, a1, a2);
#pragma unroll
      for (int a = 0; a < 3; ++a) gradT[a] = He[a] * a0 + He[a + 3] * a1 + He[a + 6] * a2;
      const float mue = A.mue_t[e * N + t];
      const float musgs = A.musgs_t ? A.musgs_t[e * N + t] : 0.f;
      const float rhon = IN == IN_DIFF ? rhon_in : s.rho;
      nu_e = ph.c_rho * mue / rhon;
      const float mu_fgp = mu + rhon * musgs;
      const float mu_egp = mue;
      kappa_e = mu * ph.Cp / ph.Prt + ph.c_ener * mue * ph.Cp / ph.Prt + ph.Cp * rhon * musgs / 0.9f;
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
        const float4 *pj = reinterpret_cast<const float4 *>(A.proj12 + (long long)node * 12);
        const float4 p0 = pj[0], p1 = pj[1], p2 = pj[2];
        const float PX[3] = {p0.x, p0.y, p0.z}, PY[3] = {p0.y, p0.w, p1.x}, PZ[3] = {p0.z, p1.x, p1.y};
        const float PM[3] = {p1.z, p1.w, p2.x}, PE[3] = {p2.y, p2.z, p2.w};
        const float cl = -ph.c_lps * ts;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          Fx[d] = cl * (PX[d] - tau[0][d]) * rhon;
          Fy[d] = cl * (PY[d] - tau[1][d]) * rhon;
          Fz[d] = cl * (PZ[d] - tau[2][d]) * rhon;
          FT[d] = cl * (PE[d] - gradT[d]) * rhon * ph.Cp / ph.Prt;
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
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const float h0 = He[0 + 3 * d], h1 = He[1 + 3 * d], h2 = He[2 + 3 * d];
        C[0][d] = gv * (h0 * FR[0] + h1 * FR[1] + h2 * FR[2]);
        C[1][d] = gv * (h0 * FT[0] + h1 * FT[1] + h2 * FT[2]);
        C[2][d] = gv * (h0 * Fx[0] + h1 * Fx[1] + h2 * Fx[2]);
        C[3][d] = gv * (h0 * Fy[0] + h1 * Fy[1] + h2 * Fy[2]);
        C[4][d] = gv * (h0 * Fz[0] + h1 * Fz[1] + h2 * Fz[2]);
        if (!LPS) C[NC - 1][d] = gv * (h0 * gradT[0] + h1 * gradT[1] + h2 * gradT[2]);
      }
    }
    __syncthreads();  // all reads of the staged fields are done
    if (active) {
#pragma unroll
      for (int q = 0; q < NC; ++q)
#pragma unroll
        for (int d = 0; d < 3; ++d) sm[el][q * 3 + d][t] = C[q][d];
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
        const float *c0 = sm[el][q * 3 + 0], *c1 = sm[el][q * 3 + 1], *c2 = sm[el][q * 3 + 2];
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
    // pass-B slots: [E*N] float4 (mass, energy, mom x, mom y), then [E*N] mom z
    reinterpret_cast<float4 *>(slots)[e * N + t] = make_float4(res[0], res[1], res[2], res[3]);
    slots[(long long)m.nelem * N * 4 + e * N + t] = res[4];
  }
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

// Assembly of the pass-B slots of k_rhs ([E*N] float4 of mass, energy,
// mom x, mom y, then [E*N] floats of mom z) into the 5 SoA residuals, same
// summation order and Kahan compensation as k_gather.
// zoff = nelem * nodes per element (start of the mom-z block, in floats / 4).
__global__ void k_gather_res5(MeshDev m, const float *__restrict__ slots, long long zoff, OutPtrs out_soa,
                              int accumulate, int use_invMl) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m.npoin) return;
  constexpr int MS = 4;
  const float *sz = slots + 4 * zoff;
  float sum[5], cmp[5];
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    sum[f] = accumulate ? out_soa.p[f][p] : 0.f;
    cmp[f] = 0.f;
  }
  const int b = m.slot_ptr[p], en = m.slot_ptr[p + 1];
  const float4 *s4 = reinterpret_cast<const float4 *>(slots);
  for (int s0 = b; s0 < en; s0 += MS) {
    int id[MS];
#pragma unroll
    for (int k = 0; k < MS; ++k) id[k] = s0 + k < en ? m.slot_idx[s0 + k] : -1;
    float4 v[MS];
    float w[MS];
#pragma unroll
    for (int k = 0; k < MS; ++k) {
      v[k] = id[k] >= 0 ? s4[id[k]] : make_float4(0.f, 0.f, 0.f, 0.f);
      w[k] = id[k] >= 0 ? sz[id[k]] : 0.f;
    }
#pragma unroll
    for (int k = 0; k < MS; ++k) {
      if (id[k] < 0) break;
      const float x[5] = {v[k].x, v[k].y, v[k].z, v[k].w, w[k]};
#pragma unroll
      for (int f = 0; f < 5; ++f) {
        const float y = x[f] - cmp[f];
        const float tt = sum[f] + y;
        cmp[f] = (tt - sum[f]) - y;
        sum[f] = tt;
      }
    }
  }
  const float sc = use_invMl ? m.invMl[p] : 1.f;
#pragma unroll
  for (int f = 0; f < 5; ++f) out_soa.p[f][p] = sum[f] * sc;
}

}  // namespace sod
