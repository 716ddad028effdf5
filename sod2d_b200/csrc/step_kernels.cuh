// Kernels of the compressible time step around the RHS: SSP low-storage RK
// stage update (FP64 or FP32 state), equation of state, entropy-viscosity
// chain with the Ducros limiter, CFL time step and the analysis integrals.
#pragma once
#include "rhs_kernels.cuh"

namespace sod {

// Conserved state: 5 fields (rho, q0, q1, q2, E), each npoin long.
template <class T>
struct State5 {
  T *f[5];
};

// ---- RK stage update (time_integ_ls.f90:323-332 and :350-359) ---------
// first != 0: U2 += g*dt*R.  Otherwise U2 = l1*U1 + li*U2 + g*dt*R.
// The FP32 shadow (reference layout: rho, q(N,3), E) receives the result.
template <class T>
__global__ void k_stage(int npoin_w, long long npoin, const int *__restrict__ lpoin_w, State5<T> U1, State5<T> U2,
                        const float *__restrict__ Rmass, const float *__restrict__ Rmom,
                        const float *__restrict__ Rener, T l1, T li, T gdt, int first, float *__restrict__ rho32,
                        float *__restrict__ q32, float *__restrict__ E32) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const long long p = lpoin_w[t];
  const float R[5] = {Rmass[p], Rmom[p], Rmom[p + npoin], Rmom[p + 2 * npoin], Rener[p]};
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    T v;
    if (first)
      v = U2.f[f][p] + gdt * (T)R[f];
    else
      v = l1 * U1.f[f][p] + li * U2.f[f][p] + gdt * (T)R[f];
    U2.f[f][p] = v;
  }
  rho32[p] = (float)U2.f[0][p];
  q32[p] = (float)U2.f[1][p];
  q32[p + npoin] = (float)U2.f[2][p];
  q32[p + 2 * npoin] = (float)U2.f[3][p];
  E32[p] = (float)U2.f[4][p];
}

// ---- end-of-step EOS (time_integ_ls.f90:391-407) -----------------------
static __global__ void k_eos_end(int npoin_w, long long npoin, const int *__restrict__ lpoin_w, float gm1, float gamma,
                          float Rgas, const float *__restrict__ rho, const float *__restrict__ q,
                          const float *__restrict__ E, float *__restrict__ u, float *__restrict__ eint,
                          float *__restrict__ pr, float *__restrict__ csound, float *__restrict__ machno,
                          float *__restrict__ Tem) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const long long p = lpoin_w[t];
  const float r = rho[p];
  float umag = 0.f;
  float uu[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    uu[d] = q[p + npoin * d] / r;
    u[p + npoin * d] = uu[d];
    umag = umag + uu[d] * uu[d];
  }
  const float ei = (E[p] / r) - 0.5f * umag;
  eint[p] = ei;
  const float pp = r * gm1 * ei;
  pr[p] = pp;
  const float c = sqrtf(gamma * pp / r);
  csound[p] = c;
  machno[p] = sqrtf(umag) / c;
  Tem[p] = pp / (r * Rgas);
}

// ---- thermo_entropy, mod_entropy_viscosity.f90:411-433 ----------------
// eta1 <- eta2; eta2 <- rho/(g-1) log(max(p/p_inf, eps)/(rho/rho_inf)^g);
// feta = u1 * eta1.
static __global__ void k_thermo_entropy(int npoin_w, long long npoin, const int *__restrict__ lpoin_w, float gamma,
                                 float p_inf, float rho_inf, const float *__restrict__ rho,
                                 const float *__restrict__ pr, const float *__restrict__ u1,
                                 float *__restrict__ eta1, float *__restrict__ eta2, float *__restrict__ feta) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const long long p = lpoin_w[t];
  const float e1 = eta2[p];
  eta1[p] = e1;
  const float r = rho[p];
  eta2[p] = (r / (gamma - 1.0f)) * logf(fmaxf(pr[p] / p_inf, 1.1920929e-07f) / powf(r / rho_inf, gamma));
#pragma unroll
  for (int d = 0; d < 3; ++d) feta[p + npoin * d] = u1[p + npoin * d] * e1;
}

// feta = u1 * eta1 at working nodes (first step, time_integ_ls.f90:274-281).
static __global__ void k_feta(int npoin_w, long long npoin, const int *__restrict__ lpoin_w, const float *__restrict__ u1,
                       const float *__restrict__ eta1, float *__restrict__ feta) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const long long p = lpoin_w[t];
#pragma unroll
  for (int d = 0; d < 3; ++d) feta[p + npoin * d] = u1[p + npoin * d] * eta1[p];
}

// ---- entropy flux residual + divergence + vorticity, one element pass --
// Slot fields (width 8): 0 = generic_scalar_convec_ijk of (feta, eta1, u1)
// (elem_convec.f90:472-594), 1 = eval_divergence of u2
// (mod_operators.f90:485-570), 2..4 = compute_vorticity of u2 before the
// per-node averaging (mod_operators.f90:684-775).  WANT_DC = 0 skips 1..4.
template <int P, int EPB, bool WANT_DC>
__global__ void __launch_bounds__(EPB *Cfg<P>::NT)
k_entropy_elem(MeshDev m, const float *__restrict__ feta, const float *__restrict__ eta1,
               const float *__restrict__ u1, const float *__restrict__ u2, float *__restrict__ slots,
               float fact = 1.0f) {
  constexpr int N1 = Cfg<P>::N1, N = Cfg<P>::N, NT = Cfg<P>::NT, NF = 10;
  __shared__ __align__(16) float sm[EPB][NF][N];
  const int el = threadIdx.x / NT, t = threadIdx.x % NT;
  const long long e = (long long)blockIdx.x * EPB + el;
  const bool active = (e < m.nelem) && (t < N);
  const long long NP = m.npoin;
  if (active) {
    const int node = m.conn[e * N + t];
    sm[el][0][t] = eta1[node];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      sm[el][1 + d][t] = u1[node + NP * d];
      sm[el][4 + d][t] = feta[node + NP * d];
      if (WANT_DC) sm[el][7 + d][t] = u2[node + NP * d];
    }
  }
  __syncthreads();
  if (!active) return;
  const int i = t % N1, j = (t / N1) % N1, k = t / (N1 * N1);
  float Di[N1], Dj[N1], Dk[N1];
#pragma unroll
  for (int s = 0; s < N1; ++s) { Di[s] = m.Dnat[i * N1 + s]; Dj[s] = m.Dnat[j * N1 + s]; Dk[s] = m.Dnat[k * N1 + s]; }
  const float *g = m.geo + e * 10 * N + t;
  float He[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) He[c] = g[c * N];
  const float gv = g[9 * N];
  float a0, a1, a2;
  iso_grad<P>(sm[el][0], i, j, k, Di, Dj, Dk, a0, a1, a2);
  float gradE[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) gradE[a] = He[a] * a0 + He[a + 3] * a1 + He[a + 6] * a2;
  float divU = 0.f, divFe = 0.f;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    iso_grad<P>(sm[el][1 + c], i, j, k, Di, Dj, Dk, a0, a1, a2);
    divU += He[c] * a0 + He[c + 3] * a1 + He[c + 6] * a2;
    iso_grad<P>(sm[el][4 + c], i, j, k, Di, Dj, Dk, a0, a1, a2);
    divFe += He[c] * a0 + He[c + 3] * a1 + He[c + 6] * a2;
  }
  const float etal = sm[el][0][t];
  float Re = 0.5f * (divFe + etal * divU);
#pragma unroll
  for (int a = 0; a < 3; ++a) Re = Re + 0.5f * (sm[el][1 + a][t] * gradE[a]);
  float out[5] = {fact * (gv * Re), 0.f, 0.f, 0.f, 0.f};
  if (WANT_DC) {
    float gu[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      iso_grad<P>(sm[el][7 + c], i, j, k, Di, Dj, Dk, a0, a1, a2);
#pragma unroll
      for (int b = 0; b < 3; ++b) gu[c][b] = He[b] * a0 + He[b + 3] * a1 + He[b + 6] * a2;  // d u_c / d x_b
    }
    out[1] = gv * (gu[0][0] + gu[1][1] + gu[2][2]);
    // curl with the reference's Levi-Civita table (CFDSolverBase.f90:1600-1606):
    // curl_0 = g(1,2) - g(2,1), curl_1 = g(2,0) - g(0,2), curl_2 = g(0,1) - g(1,0)
    // where g(j,k) = d u_j / d x_k.
    out[2] = gu[1][2] - gu[2][1];
    out[3] = -gu[0][2] + gu[2][0];
    out[4] = gu[0][1] - gu[1][0];
  }
  float4 *o = reinterpret_cast<float4 *>(slots + (e * N + t) * 8);
  o[0] = make_float4(out[0], out[1], out[2], out[3]);
  o[1] = make_float4(out[4], 0.f, 0.f, 0.f);
}

// Gather of the entropy pass: Reta (lumped: x invMl at working nodes),
// divU (raw), curl / lelpn (working nodes).  Kahan-compensated, element order.
static __global__ void k_gather_entropy(MeshDev m, const float *__restrict__ slots, const int *__restrict__ lelpn,
                                 const int *__restrict__ is_work, float *__restrict__ Reta, float *__restrict__ divU,
                                 float *__restrict__ vort, int want_dc) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m.npoin) return;
  const int nf = want_dc ? 5 : 1;
  float sum[5] = {0.f, 0.f, 0.f, 0.f, 0.f}, cmp[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
  const int b = m.slot_ptr[p], en = m.slot_ptr[p + 1];
  for (int s = b; s < en; ++s) {
    const float4 *v = reinterpret_cast<const float4 *>(slots + (long long)m.slot_idx[s] * 8);
    const float4 x0 = v[0], x1 = v[1];
    const float x[5] = {x0.x, x0.y, x0.z, x0.w, x1.x};
    for (int f = 0; f < nf; ++f) {
      const float y = x[f] - cmp[f];
      const float tt = sum[f] + y;
      cmp[f] = (tt - sum[f]) - y;
      sum[f] = tt;
    }
  }
  Reta[p] = sum[0] * m.invMl[p];
  if (want_dc) {
    divU[p] = sum[1];
    const bool w = is_work[p] != 0;
    const float inv = w ? (float)lelpn[p] : 1.f;
    for (int d = 0; d < 3; ++d) vort[p + m.npoin * d] = w ? sum[2 + d] / inv : sum[2 + d];
  }
}

// auxReta = (1.5 R2 - 0.5 R1) + (eta2 - eta1)/dt; R1 <- R2 (time_integ_ls.f90:437-443)
static __global__ void k_aux_reta(int npoin_w, const int *__restrict__ lpoin_w, float dt, float *__restrict__ Reta1,
                           const float *__restrict__ Reta2, const float *__restrict__ eta1,
                           const float *__restrict__ eta2, float *__restrict__ aux) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const long long p = lpoin_w[t];
  aux[p] = (1.5f * Reta2[p] - 0.5f * Reta1[p]) + 1.0f * (eta2[p] - eta1[p]) / dt;
  Reta1[p] = Reta2[p];
}

// Minimum of rho over working nodes (order-independent, deterministic).
// grid of the node min / max reductions: 8 blocks of 256 per SM
constexpr int MINMAX_BLOCKS = 148 * 8;
static __global__ void k_min_rho(int npoin_w, const int *__restrict__ lpoin_w, const float *__restrict__ rho,
                          unsigned int *__restrict__ out_bits) {
  float v = 100000.0f;
  // four strides per trip with every load issued first (min is order-free)
  const int stride = gridDim.x * blockDim.x;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  for (; t + 3 * stride < npoin_w; t += 4 * stride) {
    int p[4];
    float x[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) p[u] = lpoin_w[t + u * stride];
#pragma unroll
    for (int u = 0; u < 4; ++u) x[u] = rho[p[u]];
#pragma unroll
    for (int u = 0; u < 4; ++u) v = fminf(v, x[u]);
  }
  for (; t < npoin_w; t += stride) v = fminf(v, rho[lpoin_w[t]]);
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) atomicMin(out_bits, __float_as_uint(v));  // rho > 0: bit order = value order
}

// ---- smart_visc_spectral_imex (+ ducros_visc_limit) ---------------------
// mod_entropy_viscosity.f90:113-227 (high-Mach path) and :277-314.
// One warp per element.  mue_t is [e][t]; mue_ref (reference (nelem,ngaus)
// layout) is optional.  ducros = 0 skips the limiter (first step).
struct ViscArgs {
  const float *Reta, *rho, *u, *csound, *divU, *vort, *Ml, *helem, *helem_l_t;
  const unsigned int *min_rho_bits;
  float ce, cmax, cglob, ducros_min, inv_p;
  int ducros;
};

template <int P>
__global__ void k_visc(MeshDev m, ViscArgs A, const int *__restrict__ a_of_t, float *__restrict__ mue_t,
                       float *__restrict__ mue_ref) {
  constexpr int N = Cfg<P>::N;
  const long long e = (long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  if (e >= m.nelem) return;
  const long long NP = m.npoin;
  const float norm = __uint_as_float(*A.min_rho_bits);
  const float he = A.helem[e];
  float betae = 0.f;
  for (int t = lane; t < N; t += 32) {
    const int p = m.conn[e * N + t];
    const float u0 = A.u[p], u1 = A.u[p + NP], u2 = A.u[p + 2 * NP];
    const float aux2 = sqrtf(u0 * u0 + u1 * u1 + u2 * u2);
    const float aux1 = aux2 + 1.0f * A.csound[p];
    betae = fmaxf(betae, (A.rho[p] * he) * (A.cmax * A.inv_p) * aux1);
  }
  for (int o = 16; o > 0; o >>= 1) betae = fmaxf(betae, __shfl_xor_sync(0xffffffffu, betae, o));
  const float hp = he * A.inv_p;
  for (int t = lane; t < N; t += 32) {
    const int p = m.conn[e * N + t];
    const float R1 = A.rho[p] * fabsf(A.Reta[p]) / norm;
    const float Ve = A.ce * R1 * (hp * hp);
    float mu = A.cglob * fminf(Ve, betae);
    if (A.ducros) {
      const float divUl = A.divU[p] / A.Ml[p];
      const float u0 = A.u[p], u1 = A.u[p + NP], u2 = A.u[p + 2 * NP];
      const float aux2 = sqrtf(u0 * u0 + u1 * u1 + u2 * u2);
      const float v0 = A.vort[p], v1 = A.vort[p + NP], v2 = A.vort[p + 2 * NP];
      const float vv = v0 * v0 + v1 * v1 + v2 * v2;
      const float d2 = divUl * divUl;
      const float eps = 1.1920929e-07f;
      const float phi = fminf((4.0f / 3.0f) * d2 / (d2 + vv + eps), 1.0f);
      const float hl = 1.0f * aux2 / A.helem_l_t[e * N + t];
      const float phi2 = d2 / (d2 + hl * hl + eps);
      mu = mu * (fmaxf(phi - A.ducros_min, 0.f) * phi2 + A.ducros_min);
    }
    mue_t[e * N + t] = mu;
    if (mue_ref) mue_ref[e + m.nelem * a_of_t[t]] = mu;
  }
}

// ducros_visc_limit, mod_entropy_viscosity.f90:277-314, on a given mu_e in
// the reference's (nelem, ngaus) layout: mu_e *= max(phi - min, 0) phi2 +
// min with phi, phi2 from div u / Ml, the vorticity and |u| / helem_l (the
// reference's betae is computed there but unused).  Warp per element.
template <int P>
__global__ void k_ducros(MeshDev m, const float *__restrict__ u, const float *__restrict__ divU,
                         const float *__restrict__ vort, const float *__restrict__ Ml,
                         const float *__restrict__ helem_l_t, float ducros_min, const int *__restrict__ a_of_t,
                         float *__restrict__ mue_ref) {
  constexpr int N = Cfg<P>::N;
  const long long e = (long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  if (e >= m.nelem) return;
  const long long NP = m.npoin;
  for (int t = lane; t < N; t += 32) {
    const int p = m.conn[e * N + t];
    const float divUl = divU[p] / Ml[p];
    const float u0 = u[p], u1 = u[p + NP], u2 = u[p + 2 * NP];
    const float aux2 = sqrtf(u0 * u0 + u1 * u1 + u2 * u2);
    const float v0 = vort[p], v1 = vort[p + NP], v2 = vort[p + 2 * NP];
    const float vv = v0 * v0 + v1 * v1 + v2 * v2;
    const float d2 = divUl * divUl;
    const float eps = 1.1920929e-07f;  // epsilon(1.0) of real(4)
    const float phi = fminf((4.0f / 3.0f) * d2 / (d2 + vv + eps), 1.0f);
    const float hl = 1.0f * aux2 / helem_l_t[e * N + t];
    const float phi2 = d2 / (d2 + hl * hl + eps);
    float &mu = mue_ref[e + m.nelem * a_of_t[t]];
    mu = mu * (fmaxf(phi - ducros_min, 0.f) * phi2 + ducros_min);
  }
}

// Stage update of rk_4_ls_main on reference-layout FP32 arrays, working
// nodes, five fields (rho, E, q x/y/z): first stage U2 += (gam dt) R
// (time_integ_ls.f90:325-329), later stages U2 = l1 U1 + li U2 + (gam dt) R
// (:352-356), rounded as the reference (no contraction).
static __global__ void k_ls_stage_ref(int npoin_w, long long npoin, const int *__restrict__ lpoin_w, int first, float l1,
                               float li, float gam, float dt, const float *__restrict__ rho1,
                               const float *__restrict__ q1, const float *__restrict__ E1, float *__restrict__ rho2,
                               float *__restrict__ q2, float *__restrict__ E2, const float *__restrict__ Rmass,
                               const float *__restrict__ Rmom, const float *__restrict__ Rener) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const long long p = lpoin_w[t];
  const float gdt = __fmul_rn(gam, dt);
  auto upd = [&](float u1, float u2, float r) {
    return first ? __fadd_rn(u2, __fmul_rn(gdt, r))
                 : __fadd_rn(__fadd_rn(__fmul_rn(l1, u1), __fmul_rn(li, u2)), __fmul_rn(gdt, r));
  };
  rho2[p] = upd(first ? 0.f : rho1[p], rho2[p], Rmass[p]);
  E2[p] = upd(first ? 0.f : E1[p], E2[p], Rener[p]);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const long long k = p + npoin * d;
    q2[k] = upd(first ? 0.f : q1[k], q2[k], Rmom[k]);
  }
}

// Sutherland viscosity at working nodes.
static __global__ void k_sutherland(int npoin_w, const int *__restrict__ lpoin_w, float mu_factor,
                             const float *__restrict__ Tem, float *__restrict__ mu) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const long long p = lpoin_w[t];
  const float T = Tem[p];
  mu[p] = mu_factor * 1.458e-6f * powf(T, 1.5f) / (T + 110.4f);
}

// ---- adapt_dt_cfl, mod_time_ops.f90:11-62: per element, then min -------
template <int P>
__global__ void k_dt(MeshDev m, const float *__restrict__ helem, const float *__restrict__ u,
                     const float *__restrict__ csound, const float *__restrict__ mu_fluid,
                     const float *__restrict__ mue_t, const float *__restrict__ rho, float cfl_conv, float cfl_diff,
                     unsigned int *__restrict__ out_bits) {
  constexpr int N = Cfg<P>::N;
  const long long e = (long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  if (e >= m.nelem) return;
  const long long NP = m.npoin;
  float L3 = 0.f, maxMU = 0.f;
  for (int t = lane; t < N; t += 32) {
    const int p = m.conn[e * N + t];
    float um = fabsf(u[p]);
    um = fmaxf(um, fabsf(u[p + NP]));
    um = fmaxf(um, fabsf(u[p + 2 * NP]));
    L3 = fmaxf(L3, um + csound[p]);
    maxMU = fmaxf(maxMU, (0.0f + mu_fluid[p] + mue_t[e * N + t]) / rho[p]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    L3 = fmaxf(L3, __shfl_xor_sync(0xffffffffu, L3, o));
    maxMU = fmaxf(maxMU, __shfl_xor_sync(0xffffffffu, maxMU, o));
  }
  if (lane == 0) {
    const float hp = helem[e] / (float)(2 * P + 1);
    const float dconv = cfl_conv * hp / L3;
    const float ddiff = cfl_diff * (hp * hp) / maxMU;
    const float dtl = fminf(dconv, ddiff);
    atomicMin(out_bits, __float_as_uint(dtl));  // dt > 0
  }
}

// ---- analysis (mod_analysis.f90:10-168): per-element FP32 partials -----
// part[e*3 + 0] = sum_g gpvol*sum_a Ngp(g,a)*0.5*rho*|u|^2 (a)   (volAvg_EK)
// part[e*3 + 1] = sum_g gpvol*(mu+mu_e)*|curl u|^2                (eps_S)
// part[e*3 + 2] = sum_g gpvol*mu*(div u)^2                        (eps_D)
template <int P, int EPB>
__global__ void __launch_bounds__(EPB *Cfg<P>::NT)
k_analysis_elem(MeshDev m, const float *__restrict__ rho, const float *__restrict__ u,
                const float *__restrict__ mu_fluid, const float *__restrict__ mue_t,
                const float *__restrict__ Ngp_t /*[g][a] tensor order*/, float *__restrict__ part) {
  constexpr int N1 = Cfg<P>::N1, N = Cfg<P>::N, NT = Cfg<P>::NT;
  __shared__ __align__(16) float sm[EPB][4][N];
  __shared__ float red[EPB][3][NT / 32];
  const int el = threadIdx.x / NT, t = threadIdx.x % NT, lane = threadIdx.x % 32, w = t / 32;
  const long long e = (long long)blockIdx.x * EPB + el;
  const bool active = (e < m.nelem) && (t < N);
  const long long NP = m.npoin;
  int node = 0;
  if (active) {
    node = m.conn[e * N + t];
    const float u0 = u[node], u1 = u[node + NP], u2 = u[node + 2 * NP];
    sm[el][0][t] = u0; sm[el][1][t] = u1; sm[el][2][t] = u2;
    sm[el][3][t] = 0.5f * rho[node] * (u0 * u0 + u1 * u1 + u2 * u2);
  }
  __syncthreads();
  float r[3] = {0.f, 0.f, 0.f};
  if (active) {
    const int i = t % N1, j = (t / N1) % N1, k = t / (N1 * N1);
    float Di[N1], Dj[N1], Dk[N1];
#pragma unroll
    for (int s = 0; s < N1; ++s) { Di[s] = m.Dnat[i * N1 + s]; Dj[s] = m.Dnat[j * N1 + s]; Dk[s] = m.Dnat[k * N1 + s]; }
    const float *g = m.geo + e * 10 * N + t;
    float He[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) He[c] = g[c * N];
    const float gv = g[9 * N];
    float ek = 0.f;
    for (int a = 0; a < N; ++a) ek = fmaf(Ngp_t[t * N + a], sm[el][3][a], ek);
    float gu[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float a0, a1, a2;
      iso_grad<P>(sm[el][c], i, j, k, Di, Dj, Dk, a0, a1, a2);
#pragma unroll
      for (int b = 0; b < 3; ++b) gu[c][b] = He[b] * a0 + He[b + 3] * a1 + He[b + 6] * a2;
    }
    float div = gu[0][0] + gu[1][1] + gu[2][2];
    div = div * div;
    const float c0 = gu[1][2] - gu[2][1], c1 = gu[2][0] - gu[0][2], c2 = gu[0][1] - gu[1][0];
    const float curl2 = c0 * c0 + c1 * c1 + c2 * c2;
    const float mu = mu_fluid[node];
    r[0] = gv * ek;
    r[1] = gv * (mu + mue_t[e * N + t]) * curl2;
    r[2] = gv * mu * div;
  }
  // fixed-order block reduction per element
#pragma unroll
  for (int q = 0; q < 3; ++q)
    for (int o = 16; o > 0; o >>= 1) r[q] += __shfl_down_sync(0xffffffffu, r[q], o);
  if (lane == 0)
    for (int q = 0; q < 3; ++q) red[el][q][w] = r[q];
  __syncthreads();
  if (t == 0 && e < m.nelem) {
    for (int q = 0; q < 3; ++q) {
      float s = 0.f;
      for (int ww = 0; ww < NT / 32; ++ww) s += red[el][q][ww];
      part[e * 3 + q] = s;
    }
  }
}

// Deterministic FP64 sum of per-element partials: one block, fixed order.
static __global__ void k_sum_parts(long long nelem, const float *__restrict__ part, double *__restrict__ out3) {
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
  if (t == 0)
    for (int q = 0; q < 3; ++q) out3[q] = sh[q][0];
}

static __global__ void k_max_mach(int npoin_w, const int *__restrict__ lpoin_w, const float *__restrict__ machno,
                           unsigned int *__restrict__ out_bits) {
  float v = 0.f;
  const int stride = gridDim.x * blockDim.x;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  for (; t + 3 * stride < npoin_w; t += 4 * stride) {
    int p[4];
    float x[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) p[u] = lpoin_w[t + u * stride];
#pragma unroll
    for (int u = 0; u < 4; ++u) x[u] = machno[p[u]];
#pragma unroll
    for (int u = 0; u < 4; ++u) v = fmaxf(v, x[u]);
  }
  for (; t < npoin_w; t += stride) v = fmaxf(v, machno[lpoin_w[t]]);
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out_bits, __float_as_uint(v));
}

}  // namespace sod
