// Kernels of the incompressible pressure path: matrix-free Laplacian
// (eval_laplacian_mult), its Jacobi diagonal, gradient, divergence,
// skew-symmetric convection, and the vector kernels of the (flexible)
// conjugate-gradient solvers with deterministic FP64 reductions.
#pragma once
#include "rhs_kernels.cuh"

namespace sod {

// ---- Laplacian: ResP = sum_e int grad N . grad p  (mod_operators.f90:16-112)
// One thread per Gauss point; V = float (reference arithmetic) or double.
// Writes one V per element node into slots (width 1), element-ordered.
// DIR (the CG iteration): the operand is the new search direction
// z + beta p, formed on the fly from z, the previous p and *beta (the
// update p = z + beta p itself is stored by k_cg_q), and the slots are
// written node-sorted (slot_pos) for k_cg_q's contiguous sums.
template <int P, int EPB, class V, bool DIR = false>
__global__ void __launch_bounds__(EPB *Cfg<P>::NT)
k_lap_elem(MeshDev m, const V *__restrict__ p, V *__restrict__ slots, const int *__restrict__ stop = nullptr,
           const V *__restrict__ z = nullptr, const V *__restrict__ beta = nullptr) {
  constexpr int N1 = Cfg<P>::N1, N = Cfg<P>::N, NT = Cfg<P>::NT;
  if (stop && *stop) return;
  __shared__ V sm[EPB][4][N];
  const int el = threadIdx.x / NT, t = threadIdx.x % NT;
  const long long e = (long long)blockIdx.x * EPB + el;
  const bool active = (e < m.nelem) && (t < N);
  if (active) {
    const int n = m.conn[e * N + t];
    if (DIR) {
      const V bt = *beta;
      sm[el][0][t] = z[n] + bt * p[n];
    } else {
      sm[el][0][t] = p[n];
    }
  }
  __syncthreads();
  const int i = t % N1, j = (t / N1) % N1, k = t / (N1 * N1);
  V C0 = 0, C1 = 0, C2 = 0;
  V Di[N1], Dj[N1], Dk[N1];
  if (active) {
#pragma unroll
    for (int s = 0; s < N1; ++s) {
      Di[s] = (V)m.Dnat[i * N1 + s]; Dj[s] = (V)m.Dnat[j * N1 + s]; Dk[s] = (V)m.Dnat[k * N1 + s];
    }
    const float *g = m.geo + e * 10 * N + t;
    V He[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) He[c] = (V)g[c * N];
    const V gv = (V)g[9 * N];
    const V *f = sm[el][0];
    V g0 = 0, g1 = 0, g2 = 0;
#pragma unroll
    for (int s = 0; s < N1; ++s) {
      const int mm = ref_order<P>(s);
      g0 += Di[mm] * f[mm + N1 * j + N1 * N1 * k];
      g1 += Dj[mm] * f[i + N1 * mm + N1 * N1 * k];
      g2 += Dk[mm] * f[i + N1 * j + N1 * N1 * mm];
    }
    V gP[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) gP[a] = He[a] * g0 + He[a + 3] * g1 + He[a + 6] * g2;
    C0 = gv * (He[0] * gP[0] + He[1] * gP[1] + He[2] * gP[2]);
    C1 = gv * (He[3] * gP[0] + He[4] * gP[1] + He[5] * gP[2]);
    C2 = gv * (He[6] * gP[0] + He[7] * gP[1] + He[8] * gP[2]);
  }
  __syncthreads();
  if (active) { sm[el][1][t] = C0; sm[el][2][t] = C1; sm[el][3][t] = C2; }
  __syncthreads();
  if (!active) return;
  V acc = 0;
#pragma unroll
  for (int s = 0; s < N1; ++s) {
    const int mm = ref_order<P>(s);
    acc += (V)m.Dnat[mm * N1 + i] * sm[el][1][mm + N1 * j + N1 * N1 * k];
    acc += (V)m.Dnat[mm * N1 + j] * sm[el][2][i + N1 * mm + N1 * N1 * k];
    acc += (V)m.Dnat[mm * N1 + k] * sm[el][3][i + N1 * j + N1 * N1 * mm];
  }
  slots[DIR ? (long long)m.slot_pos[e * N + t] : e * N + t] = acc;
}

// Scalar-slot assembly out(p) = scale * sum(slots of p); float sums are
// Kahan-compensated.  Only nodes with slots are written (masters).
template <class V>
__global__ void k_gather1(MeshDev m, const V *__restrict__ slots, V *__restrict__ out, int use_invMl) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m.npoin) return;
  const int b = m.slot_ptr[p], en = m.slot_ptr[p + 1];
  V sum = 0, cmp = 0;
  for (int s = b; s < en; ++s) {
    const V y = slots[m.slot_idx[s]] - cmp;
    const V tt = sum + y;
    cmp = (tt - sum) - y;
    sum = tt;
  }
  out[p] = use_invMl ? sum * (V)m.invMl[p] : sum;
}

// ---- eval_laplacian_diag, mod_operators.f90:638-682 --------------------
// d(a) = sum_g gpvol(g) |grad N_a(g)|^2; with GLL collocation grad N_a(g)
// is non-zero only on the three lines through a.  One thread per node a
// of an element loops over the Gauss points of those lines.
template <int P>
__global__ void k_lap_diag_elem(MeshDev m, float *__restrict__ slots) {
  constexpr int N1 = Cfg<P>::N1, N = Cfg<P>::N;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)m.nelem * N) return;
  const long long e = idx / N;
  const int a = (int)(idx % N);
  const int ia = a % N1, ja = (a / N1) % N1, ka = a / (N1 * N1);
  const float *g = m.geo + e * 10 * N;
  float d = 0.f;
  for (int gp = 0; gp < N; ++gp) {
    const int i = gp % N1, j = (gp / N1) % N1, k = gp / (N1 * N1);
    // iso-derivatives of N_a at gp: D[i][ia] d_{j,ja} d_{k,ka}, ...
    float d0 = (j == ja && k == ka) ? m.Dnat[i * N1 + ia] : 0.f;
    float d1 = (i == ia && k == ka) ? m.Dnat[j * N1 + ja] : 0.f;
    float d2 = (i == ia && j == ja) ? m.Dnat[k * N1 + ka] : 0.f;
    if (d0 == 0.f && d1 == 0.f && d2 == 0.f) continue;
    const float gv = g[9 * N + gp];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float gc = g[c * N + gp] * d0 + g[(c + 3) * N + gp] * d1 + g[(c + 6) * N + gp] * d2;
      d += gv * gc * gc;
    }
  }
  slots[idx] = d;
}

// ---- gradient / divergence / incompressible convection ----------------
// MODE 0: gradient of a scalar x: slots (width 4) = gpvol*grad x (3)
// MODE 1: divergence of u: slot[0] = gpvol * div u
// MODE 2: full_convec_ijk_incomp (elem_convec_incomp.f90:19-125): slots
//         (width 4) = gpvol * 0.5*(div(q u) + u div q + (u.grad) q)
template <int P, int EPB, int MODE>
__global__ void __launch_bounds__(EPB *Cfg<P>::NT)
k_vec_elem(MeshDev m, const float *__restrict__ x, const float *__restrict__ u, const float *__restrict__ q,
           float *__restrict__ slots) {
  constexpr int N1 = Cfg<P>::N1, N = Cfg<P>::N, NT = Cfg<P>::NT;
  constexpr int NF = MODE == 0 ? 1 : (MODE == 1 ? 3 : 12);
  __shared__ __align__(16) float sm[EPB][NF][N];
  const int el = threadIdx.x / NT, t = threadIdx.x % NT;
  const long long e = (long long)blockIdx.x * EPB + el;
  const bool active = (e < m.nelem) && (t < N);
  const long long NP = m.npoin;
  float ul[3] = {0.f, 0.f, 0.f}, ql[3] = {0.f, 0.f, 0.f};
  if (active) {
    const int node = m.conn[e * N + t];
    if (MODE == 0) sm[el][0][t] = x[node];
    if (MODE >= 1)
      for (int d = 0; d < 3; ++d) { ul[d] = u[node + NP * d]; sm[el][d][t] = (MODE == 1) ? ul[d] : 0.f; }
    if (MODE == 2) {
      for (int d = 0; d < 3; ++d) { ql[d] = q[node + NP * d]; sm[el][d][t] = ql[d]; }
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) sm[el][3 + a * 3 + b][t] = ql[a] * ul[b];
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
  float out[3] = {0.f, 0.f, 0.f};
  float a0, a1, a2;
  if (MODE == 0) {
    iso_grad<P>(sm[el][0], i, j, k, Di, Dj, Dk, a0, a1, a2);
#pragma unroll
    for (int a = 0; a < 3; ++a) out[a] = gv * (He[a] * a0 + He[a + 3] * a1 + He[a + 6] * a2);
  } else if (MODE == 1) {
    float dv = 0.f;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      iso_grad<P>(sm[el][c], i, j, k, Di, Dj, Dk, a0, a1, a2);
      dv += He[c] * a0 + He[c + 3] * a1 + He[c + 6] * a2;
    }
    out[0] = gv * dv;
  } else {
    float gradQ[3][3], divF[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      iso_grad<P>(sm[el][c], i, j, k, Di, Dj, Dk, a0, a1, a2);
#pragma unroll
      for (int b = 0; b < 3; ++b) gradQ[c][b] = He[b] * a0 + He[b + 3] * a1 + He[b + 6] * a2;
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        iso_grad<P>(sm[el][3 + a * 3 + b], i, j, k, Di, Dj, Dk, a0, a1, a2);
        divF[a] += He[b] * a0 + He[b + 3] * a1 + He[b + 6] * a2;
      }
    const float divU = gradQ[0][0] + gradQ[1][1] + gradQ[2][2];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float r = 0.5f * (divF[a] + ul[a] * divU);
#pragma unroll
      for (int b = 0; b < 3; ++b) r = r + 0.5f * (ul[b] * gradQ[a][b]);
      out[a] = gv * r;
    }
  }
  reinterpret_cast<float4 *>(slots + (e * N + t) * 4)[0] = make_float4(out[0], out[1], out[2], 0.f);
}

// ---- CG vector kernels (FP64 reductions, deterministic) ---------------
// Dot products over working nodes with FP64 accumulation, summed in a
// fixed order (deterministic).
constexpr int DOT_BLOCKS = 592;  // 4 blocks per SM on 148 SMs
constexpr int DOT_THREADS = 256;

// dot d = sum a[d]*(b[d] - c[d]) (c[d] may be null)
template <class V, int ND>
struct DotArgs {
  const V *a[ND];
  const V *b[ND];
  const V *c[ND];
};

// Single-block sum of DOT_BLOCKS partials per value, in a fixed order.
static __global__ void k_dot_final(int nd, const double *__restrict__ part, double *__restrict__ out) {
  __shared__ double sh[1024];
  for (int d = 0; d < nd; ++d) {
    double s = 0.0;
    for (int b = threadIdx.x; b < DOT_BLOCKS; b += blockDim.x) s += part[d * DOT_BLOCKS + b];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
      if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[d] = sh[0];
    __syncthreads();
  }
}

// ND dot products in one launch: each block reduces its grid-stride share
// in a fixed order and stores a partial; the last block to take the ticket
// adds the partials in block order (deterministic) and resets the ticket.
template <class V, int ND>
__global__ void __launch_bounds__(DOT_THREADS) k_dot(int npoin_w, const int *__restrict__ lpoin_w,
                                                     DotArgs<V, ND> A, double *__restrict__ part,
                                                     unsigned *__restrict__ ticket, double *__restrict__ out) {
  __shared__ double sh[ND][DOT_THREADS];
  __shared__ bool last;
  double s[ND];
#pragma unroll
  for (int d = 0; d < ND; ++d) s[d] = 0.0;
  // grid-stride over the nodes; four strides per trip with every load issued
  // before the first product (same per-thread order as one stride per trip)
  const int stride = gridDim.x * blockDim.x;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  for (; t + 3 * stride < npoin_w; t += 4 * stride) {
    int p[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) p[u] = lpoin_w[t + u * stride];
    V av[4][ND], bv[4][ND];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int d = 0; d < ND; ++d) {
        av[u][d] = A.a[d][p[u]];
        bv[u][d] = A.c[d] ? (V)(A.b[d][p[u]] - A.c[d][p[u]]) : A.b[d][p[u]];
      }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int d = 0; d < ND; ++d) s[d] += (double)(av[u][d] * bv[u][d]);
  }
  for (; t < npoin_w; t += stride) {
    const int p = lpoin_w[t];
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      const V bb = A.c[d] ? (V)(A.b[d][p] - A.c[d][p]) : A.b[d][p];
      s[d] += (double)(A.a[d][p] * bb);
    }
  }
#pragma unroll
  for (int d = 0; d < ND; ++d) sh[d][threadIdx.x] = s[d];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int d = 0; d < ND; ++d) sh[d][threadIdx.x] += sh[d][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
#pragma unroll
    for (int d = 0; d < ND; ++d) part[d * gridDim.x + blockIdx.x] = sh[d][0];
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    double v = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) v += __ldcg(part + d * gridDim.x + b);
    sh[d][threadIdx.x] = v;
  }
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int d = 0; d < ND; ++d) sh[d][threadIdx.x] += sh[d][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
#pragma unroll
    for (int d = 0; d < ND; ++d) out[d] = sh[d][0];
    *ticket = 0u;
  }
}

// ---- device-resident preconditioned CG -------------------------------------
// Scalars of the iteration kept in device memory between launches, so that
// the host only reads them once per batch of iterations.  Every iteration
// kernel returns at once when status != 0.
struct CgScal {
  double rz;     // r . z of the current residual
  double pq;     // p . A p
  double alpha, beta;
  double rr;     // ||r||^2 after the last update
  double thr2;   // (tol ||b||)^2
  int iter;      // iterations done in this solve
  int status;    // 0 running, 1 converged (recursive residual), 2 breakdown, 3 non-finite
};

constexpr int CG_THREADS = 256, CG_U = 4;

// Node loops of the CG kernels handle several nodes per thread and issue all
// their loads before any store, so that each thread keeps several memory
// round trips in flight.
inline unsigned cg_blocks(long long n, int u) {
  const long long b = (n + (long long)CG_THREADS * u - 1) / ((long long)CG_THREADS * u);
  return (unsigned)(b < 1 ? 1 : b);
}

// Deterministic grid-wide sum of ND doubles: each block reduces its values
// in a fixed order and stores one partial; the last block to take a ticket
// adds the partials in block order.  Returns true (in every thread of that
// block only) with tot filled; the ticket is reset for the next launch.
template <int ND>
__device__ bool grid_sum(double (&v)[ND], double *__restrict__ part, unsigned *ticket, double (&tot)[ND]) {
  __shared__ double sh[ND][32];
  __shared__ bool last;
  const int lane = threadIdx.x % 32, warp = threadIdx.x / 32, nw = blockDim.x / 32;
#pragma unroll
  for (int d = 0; d < ND; ++d)
    for (int o = 16; o > 0; o >>= 1) v[d] += __shfl_xor_sync(0xffffffffu, v[d], o);
  if (lane == 0)
    for (int d = 0; d < ND; ++d) sh[d][warp] = v[d];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int d = 0; d < ND; ++d) {
      double s = 0.0;
      for (int w = 0; w < nw; ++w) s += sh[d][w];
      part[d * gridDim.x + blockIdx.x] = s;
    }
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    double s = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) s += __ldcg(part + d * gridDim.x + b);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __syncthreads();
    if (lane == 0) sh[d][warp] = s;
    __syncthreads();
    double t = 0.0;
    for (int w = 0; w < nw; ++w) t += sh[d][w];
    tot[d] = t;
  }
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

// q = assembled Laplacian slots (Kahan, as k_gather1) with the p.q partials;
// the last block sets alpha = rz / pq.  DIR: the slots are node-sorted
// (k_lap_elem<DIR>), and the new search direction p = z + beta p is formed
// and stored here for every node with slots (the working nodes).
template <bool DIR = false>
__global__ void __launch_bounds__(CG_THREADS)
k_cg_q(MeshDev m, const double *__restrict__ slots, double *__restrict__ p, double *__restrict__ q,
       CgScal *S, double *__restrict__ part, unsigned *ticket, const double *__restrict__ z = nullptr) {
  if (S->status) return;
  constexpr int U = 2, MS = 8;  // nodes per thread, slots loaded ahead per node
  const double bt = DIR ? S->beta : 0.0;
  double v[1] = {0.0};
  for (long long base = (long long)blockIdx.x * blockDim.x * U + threadIdx.x; base < m.npoin;
       base += (long long)gridDim.x * blockDim.x * U) {
    int b[U], en[U];
    double pn[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const long long n = base + (long long)u * blockDim.x;
      b[u] = en[u] = 0;
      pn[u] = 0.0;
      if (n < m.npoin) {
        b[u] = m.slot_ptr[n]; en[u] = m.slot_ptr[n + 1]; pn[u] = p[n];
        if (DIR) pn[u] = z[n] + bt * pn[u];
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const long long n = base + (long long)u * blockDim.x;
      if (n >= m.npoin) continue;
      if (DIR && b[u] != en[u]) p[n] = pn[u];
      double sum = 0.0, cmp = 0.0;
      for (int s0 = b[u]; s0 < en[u]; s0 += MS) {
        int id[MS];
        double y[MS];
#pragma unroll
        for (int k = 0; k < MS; ++k) id[k] = s0 + k < en[u] ? (DIR ? s0 + k : m.slot_idx[s0 + k]) : -1;
#pragma unroll
        for (int k = 0; k < MS; ++k) y[k] = id[k] >= 0 ? slots[id[k]] : 0.0;
#pragma unroll
        for (int k = 0; k < MS; ++k) {
          if (id[k] < 0) break;
          const double yy = y[k] - cmp;
          const double tt = sum + yy;
          cmp = (tt - sum) - yy;
          sum = tt;
        }
      }
      q[n] = sum;
      if (b[u] != en[u]) v[0] += pn[u] * sum;
    }
  }
  double tot[1];
  if (grid_sum<1>(v, part, ticket, tot) && threadIdx.x == 0) {
    S->pq = tot[0];
    if (!isfinite(tot[0])) {
      S->status = 3;
    } else if (!(tot[0] > 0.0)) {
      S->status = 2;
    } else {
      S->alpha = S->rz / tot[0];
    }
  }
}

// x += alpha p ; r -= alpha q ; with JAC also z = Minv r (reading the old z),
// otherwise, when uf is given, uf = (float)(Dh r); the last block records
// ||r||^2, detects convergence and, with JAC, sets the Polak-Ribiere
// beta = r.(z - z_old) / rz_old.
template <bool JAC>
__global__ void __launch_bounds__(CG_THREADS)
k_cg_update(int npoin_w, const int *__restrict__ lpoin_w, const double *__restrict__ p,
            const double *__restrict__ q, const double *__restrict__ Minv, double *__restrict__ x,
            double *__restrict__ r, double *__restrict__ z, CgScal *S, double *__restrict__ hist, int hist_cap,
            double *__restrict__ part, unsigned *ticket, const double *__restrict__ Dh = nullptr,
            float *__restrict__ uf = nullptr) {
  if (S->status) return;
  constexpr int U = CG_U;
  const double a = S->alpha;
  double v[3] = {0.0, 0.0, 0.0};
  for (long long base = (long long)blockIdx.x * blockDim.x * U + threadIdx.x; base < npoin_w;
       base += (long long)gridDim.x * blockDim.x * U) {
    int id[U];
    double pv[U], qv[U], xv[U], rv[U], mv[U], zv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const long long t = base + (long long)u * blockDim.x;
      id[u] = t < npoin_w ? lpoin_w[t] : -1;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (id[u] < 0) continue;
      const int i = id[u];
      pv[u] = p[i]; qv[u] = q[i]; xv[u] = x[i]; rv[u] = r[i];
      if (JAC) { mv[u] = Minv[i]; zv[u] = z[i]; }
      if (!JAC && uf) mv[u] = Dh[i];
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (id[u] < 0) continue;
      const int i = id[u];
      x[i] = xv[u] + a * pv[u];
      const double rn = rv[u] - a * qv[u];
      r[i] = rn;
      v[0] += rn * rn;
      if (JAC) {
        const double zn = rn * mv[u];
        z[i] = zn;
        v[1] += rn * zn;
        v[2] += rn * zv[u];
      } else if (uf) {
        uf[i] = (float)(mv[u] * rn);  // D^-1/2 r for the learned preconditioner
      }
    }
  }
  double tot[3];
  if (grid_sum<3>(v, part, ticket, tot) && threadIdx.x == 0) {
    const int it = S->iter + 1;
    S->iter = it;
    S->rr = tot[0];
    hist[(it - 1) % hist_cap] = tot[0];
    if (!isfinite(tot[0])) {
      S->status = 3;
    } else if (tot[0] < S->thr2) {
      S->status = 1;
    }
    if (JAC) {
      S->beta = (tot[1] - tot[2]) / S->rz;
      S->rz = tot[1];
    }
  }
}

// Learned preconditioner: z(n) = D^-1/2(n) (exp(alpha) D^-1/2(n) r(n) + sum of
// the node's contributions, stored contiguously from pptr[n]) (as
// k_patch_gather_perm), with the partials r.z and r.z_old; the last block
// sets beta and rz.
static __global__ void __launch_bounds__(CG_THREADS)
k_cg_patch_z(long long npoin, const int *__restrict__ pptr, const float *__restrict__ ctr,
             const double *__restrict__ r, const double *__restrict__ Dh, const float *__restrict__ prm, int o_alpha,
             double *__restrict__ z, CgScal *S, double *__restrict__ part, unsigned *ticket) {
  if (S->status) return;
  constexpr int U = CG_U;
  const double gam = exp((double)prm[o_alpha]);
  double v[2] = {0.0, 0.0};
  for (long long base = (long long)blockIdx.x * blockDim.x * U + threadIdx.x; base < npoin;
       base += (long long)gridDim.x * blockDim.x * U) {
    int b[U], en[U];
    double dv[U], rv[U], zo[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const long long n = base + (long long)u * blockDim.x;
      b[u] = en[u] = 0;
      if (n < npoin) {
        b[u] = pptr[n]; en[u] = pptr[n + 1];
        dv[u] = Dh[n]; rv[u] = r[n]; zo[u] = z[n];
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (b[u] == en[u]) continue;
      const long long n = base + (long long)u * blockDim.x;
      double acc = 0.0;
      for (int s0 = b[u]; s0 < en[u]; s0 += 8) {
        float y[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) y[k] = s0 + k < en[u] ? ctr[s0 + k] : 0.f;
#pragma unroll
        for (int k = 0; k < 8; ++k) acc += (double)y[k];
      }
      const double zn = dv[u] * (gam * dv[u] * rv[u] + acc);
      z[n] = zn;
      v[0] += rv[u] * zn;
      v[1] += rv[u] * zo[u];
    }
  }
  double tot[2];
  if (grid_sum<2>(v, part, ticket, tot) && threadIdx.x == 0) {
    S->beta = (tot[0] - tot[1]) / S->rz;
    S->rz = tot[0];
    if (!isfinite(S->beta)) S->status = 3;
  }
}

// harvest snapshot of the iterate and residual (skipped once stopped)
static __global__ void k_cg_snapshot(int npoin_w, const int *__restrict__ lpoin_w, const double *__restrict__ x,
                              const double *__restrict__ r, double *__restrict__ xs, float *__restrict__ rs,
                              const CgScal *S) {
  if (S->status) return;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < npoin_w; t += gridDim.x * blockDim.x) {
    const int i = lpoin_w[t];
    xs[i] = x[i];
    rs[i] = (float)r[i];
  }
}

}  // namespace sod

