// Kernels of the implicit velocity solve of the incompressible step
// (conjGrad_veloc_incomp with LPS, src/lib_sod2d_incomp/sources/
// mod_solver_incomp.f90:27-251): the element stabilisation time
// (species_tau), the LPS projection of the velocity gradient
// (eval_tau_veloc) and the stabilised viscous operator
// (full_diff_stab_incomp).  Same element layout and deterministic
// slot assembly as the other element kernels.
#pragma once
#include "rhs_kernels.cuh"

namespace sod {

// species_tau, src/lib_species/sources/elem_stab_species.f90:122-148:
// tau_e = max over the element nodes of helem (c / p) |u|; warp per element.
static __global__ void k_species_tau(long long nelem, int N, const int *__restrict__ conn, const float *__restrict__ helem,
                              const float *__restrict__ u, long long npoin, float c_over_p, float *__restrict__ tau) {
  const long long e = (long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  if (e >= nelem) return;
  float taul = 0.f;
  const float he = helem[e];
  for (int t = lane; t < N; t += 32) {
    const int p = conn[e * N + t];
    const float u0 = u[p], u1 = u[p + npoin], u2 = u[p + 2 * npoin];
    taul = fmaxf(taul, he * c_over_p * sqrtf(u0 * u0 + u1 * u1 + u2 * u2));
  }
  for (int o = 16; o > 0; o >>= 1) taul = fmaxf(taul, __shfl_xor_sync(0xffffffffu, taul, o));
  if (lane == 0) tau[e] = taul;
}

// Stage the 3 velocity components of an element and return grad u at the
// thread's Gauss point (gradU[a][b] = d u_a / d x_b).
template <int P, int EPB>
__device__ __forceinline__ void stage_grad_u(const MeshDev &m, const float *__restrict__ u, float (*sm)[Cfg<P>::N],
                                             long long e, int t, bool active, float (&gradU)[3][3], float &gv,
                                             float (&He)[9], int &node) {
  constexpr int N1 = Cfg<P>::N1, N = Cfg<P>::N;
  const long long NP = m.npoin;
  if (active) {
    node = m.conn[e * N + t];
    const float *g = m.geo + e * 10 * N + t;
#pragma unroll
    for (int c = 0; c < 9; ++c) He[c] = g[c * N];
    gv = g[9 * N];
    sm[0][t] = u[node];
    sm[1][t] = u[node + NP];
    sm[2][t] = u[node + 2 * NP];
  }
  __syncthreads();
  if (!active) return;
  const int i = t % N1, j = (t / N1) % N1, k = t / (N1 * N1);
  float Di[N1], Dj[N1], Dk[N1];
#pragma unroll
  for (int q = 0; q < N1; ++q) { Di[q] = m.Dnat[i * N1 + q]; Dj[q] = m.Dnat[j * N1 + q]; Dk[q] = m.Dnat[k * N1 + q]; }
  float gU[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c) iso_grad<P>(sm[c], i, j, k, Di, Dj, Dk, gU[c][0], gU[c][1], gU[c][2]);
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) gradU[a][b] = He[b] * gU[a][0] + He[b + 3] * gU[a][1] + He[b + 6] * gU[a][2];
}

// eval_tau_veloc, src/lib_sod2d_incomp/sources/mod_operators.f90:373-483,
// element part: gpvol * (grad u + grad u^T), whose 6 distinct entries
// (00 01 02 11 12 22) go to 8-wide slots.
template <int P, int EPB>
__global__ void __launch_bounds__(EPB *Cfg<P>::NT)
k_tauv_elem(MeshDev m, const float *__restrict__ u, float *__restrict__ slots) {
  constexpr int N = Cfg<P>::N, NT = Cfg<P>::NT;
  __shared__ __align__(16) float sm[EPB][3][N];
  const int el = threadIdx.x / NT, t = threadIdx.x % NT;
  const long long e = (long long)blockIdx.x * EPB + el;
  const bool active = (e < m.nelem) && (t < N);
  float gradU[3][3], gv = 0.f, He[9];
  int node = 0;
  stage_grad_u<P, EPB>(m, u, sm[el], e, t, active, gradU, gv, He, node);
  if (!active) return;
  float4 *o = reinterpret_cast<float4 *>(slots + (e * N + t) * 8);
  o[0] = make_float4(gv * (gradU[0][0] + gradU[0][0]), gv * (gradU[0][1] + gradU[1][0]),
                     gv * (gradU[0][2] + gradU[2][0]), gv * (gradU[1][1] + gradU[1][1]));
  o[1] = make_float4(gv * (gradU[1][2] + gradU[2][1]), gv * (gradU[2][2] + gradU[2][2]), 0.f, 0.f);
}

// Assembly of the projection slots (Kahan, element order) divided by the
// lumped mass (lumped_solver_vect, mod_solver.f90:61-79), node-major
// [npoin][8] (6 used); nodes without slots get 0.
static __global__ void k_gather_tauv(MeshDev m, const float *__restrict__ slots, const float *__restrict__ Ml,
                              float *__restrict__ tauP) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m.npoin) return;
  const int b = m.slot_ptr[p], en = m.slot_ptr[p + 1];
  float sum[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, cmp[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  for (int s = b; s < en; ++s) {
    const float4 *v = reinterpret_cast<const float4 *>(slots + (long long)m.slot_idx[s] * 8);
    const float4 v0 = v[0], v1 = v[1];
    const float x[6] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y};
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const float y = x[f] - cmp[f];
      const float tt = sum[f] + y;
      cmp[f] = (tt - sum[f]) - y;
      sum[f] = tt;
    }
  }
  if (b != en) {
    const float ml = Ml[p];
#pragma unroll
    for (int f = 0; f < 6; ++f) sum[f] = sum[f] / ml;
  }
  float4 *o = reinterpret_cast<float4 *>(tauP + p * 8);
  o[0] = make_float4(sum[0], sum[1], sum[2], sum[3]);
  o[1] = make_float4(sum[4], sum[5], 0.f, 0.f);
}

// Reference layout GradX/GradY/GradZ (npoin,3) <-> node-major symmetric [p][8].
static __global__ void k_unpack_tauv(long long npoin, const float *__restrict__ tauP, float *__restrict__ GX,
                              float *__restrict__ GY, float *__restrict__ GZ) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npoin) return;
  const float *s = tauP + p * 8;
  GX[p] = s[0]; GX[p + npoin] = s[1]; GX[p + 2 * npoin] = s[2];
  GY[p] = s[1]; GY[p + npoin] = s[3]; GY[p + 2 * npoin] = s[4];
  GZ[p] = s[2]; GZ[p + npoin] = s[4]; GZ[p + 2 * npoin] = s[5];
}
static __global__ void k_pack_tauv(long long npoin, const float *__restrict__ GX, const float *__restrict__ GY,
                            const float *__restrict__ GZ, float *__restrict__ tauP) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npoin) return;
  float4 *o = reinterpret_cast<float4 *>(tauP + p * 8);
  o[0] = make_float4(GX[p], GX[p + npoin], GX[p + 2 * npoin], GY[p + npoin]);
  o[1] = make_float4(GY[p + 2 * npoin], GZ[p + 2 * npoin], 0.f, 0.f);
}

// full_diff_stab_incomp, src/lib_sod2d_incomp/sources/elem_stab_incomp.f90:
// 12-153: fluxes F_r = (mu_fluid + mu_sgs + tau_e)(grad u + grad u^T)(r,:)
// - tau_e TauP(r,:) at each Gauss point, their contravariant components
// staged, then the weak divergence; 3 residuals per element node into
// 4-wide slots.
template <int P, int EPB>
__global__ void __launch_bounds__(EPB *Cfg<P>::NT)
k_diffv_elem(MeshDev m, const float *__restrict__ u, const float *__restrict__ mu_fluid,
             const float *__restrict__ musgs_t, const float *__restrict__ tauP, const float *__restrict__ tau_e,
             float *__restrict__ slots) {
  constexpr int N1 = Cfg<P>::N1, N = Cfg<P>::N, NT = Cfg<P>::NT;
  __shared__ __align__(16) float sm[EPB][9][N];
  const int el = threadIdx.x / NT, t = threadIdx.x % NT;
  const long long e = (long long)blockIdx.x * EPB + el;
  const bool active = (e < m.nelem) && (t < N);
  float gradU[3][3], gv = 0.f, He[9];
  int node = 0;
  stage_grad_u<P, EPB>(m, u, reinterpret_cast<float(*)[N]>(sm[el]), e, t, active, gradU, gv, He, node);
  float C[3][3];
  if (active) {
    const float ts = tau_e[e];
    const float mu_fgp = mu_fluid[node] + (musgs_t ? musgs_t[e * N + t] : 0.f) + ts;
    const float4 *tp = reinterpret_cast<const float4 *>(tauP + (long long)node * 8);
    const float4 t0 = tp[0], t1 = tp[1];
    const float TP[3][3] = {{t0.x, t0.y, t0.z}, {t0.y, t0.w, t1.x}, {t0.z, t1.x, t1.y}};
    float F[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int d = 0; d < 3; ++d) F[r][d] = mu_fgp * (gradU[r][d] + gradU[d][r]) - ts * TP[r][d];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float h0 = He[0 + 3 * d], h1 = He[1 + 3 * d], h2 = He[2 + 3 * d];
#pragma unroll
      for (int r = 0; r < 3; ++r) C[r][d] = gv * (h0 * F[r][0] + h1 * F[r][1] + h2 * F[r][2]);
    }
  }
  __syncthreads();  // the staged velocity is no longer read
  if (active) {
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int d = 0; d < 3; ++d) sm[el][r * 3 + d][t] = C[r][d];
  }
  __syncthreads();
  if (!active) return;
  const int i = t % N1, j = (t / N1) % N1, k = t / (N1 * N1);
  float Dci[N1], Dcj[N1], Dck[N1];
#pragma unroll
  for (int q = 0; q < N1; ++q) { Dci[q] = m.Dnat[q * N1 + i]; Dcj[q] = m.Dnat[q * N1 + j]; Dck[q] = m.Dnat[q * N1 + k]; }
  float wd[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const float *c0 = sm[el][r * 3 + 0], *c1 = sm[el][r * 3 + 1], *c2 = sm[el][r * 3 + 2];
    float acc = 0.f;
#pragma unroll
    for (int ss = 0; ss < N1; ++ss) {
      const int mm = ref_order<P>(ss);
      acc = fmaf(Dci[mm], c0[mm + N1 * j + N1 * N1 * k], acc);
      acc = fmaf(Dcj[mm], c1[i + N1 * mm + N1 * N1 * k], acc);
      acc = fmaf(Dck[mm], c2[i + N1 * j + N1 * N1 * mm], acc);
    }
    wd[r] = acc;
  }
  reinterpret_cast<float4 *>(slots)[e * N + t] = make_float4(wd[0], wd[1], wd[2], 0.f);
}

// qn = v Ml + qn fact dt over working nodes, 3 components (npoin,3)
static __global__ void k_veloc_op(int npoin_w, long long npoin, const int *__restrict__ lpoin_w,
                           const float *__restrict__ Ml, const float *__restrict__ v, float fact, float dt,
                           float *__restrict__ qn) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const long long p = lpoin_w[t];
  const float ml = Ml[p];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const long long k = p + npoin * d;
    qn[k] = v[k] * ml + qn[k] * fact * dt;
  }
}

// Vector updates of the velocity CG over working nodes, 3 components:
// mode 0: r = b - qn ; z = r / (Ml/dt) ; p = z
// mode 1: x += alpha p ; r -= alpha q ; z1 = z ; z = r / (Ml/dt)
// mode 2: p = z + beta p
static __global__ void k_veloc_vec(int mode, int npoin_w, long long npoin, const int *__restrict__ lpoin_w,
                            const float *__restrict__ Ml, float dt, float alpha, float beta,
                            const float *__restrict__ b, float *__restrict__ x, float *__restrict__ r,
                            float *__restrict__ p, const float *__restrict__ q, float *__restrict__ z,
                            float *__restrict__ z1) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const long long n = lpoin_w[t];
  const float Mu = Ml[n] / dt;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const long long k = n + npoin * d;
    if (mode == 0) {
      r[k] = b[k] - q[k];
      z[k] = r[k] / Mu;
      p[k] = z[k];
    } else if (mode == 1) {
      x[k] = x[k] + alpha * p[k];
      r[k] = r[k] - alpha * q[k];
      z1[k] = z[k];
      z[k] = r[k] / Mu;
    } else {
      p[k] = z[k] + beta * p[k];
    }
  }
}

}  // namespace sod
