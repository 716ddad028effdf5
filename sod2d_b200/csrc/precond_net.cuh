// Learned element-patch preconditioner for the pressure Poisson problem:
// inference, training forward/backward and Adam kernels.
//
// For element order P (n1 = P+1, N = n1^3 own nodes) the patch of element e
// is its N own nodes plus the first node layer of each of its 6 face
// neighbours, NP = N + 6 n1^2 slots (160 for P=3, 275 for P=4), listed in
// a per-element patch table (-1 where a face has no neighbour).  With
// D = Jacobi diagonal, u = D^-1/2 r:
//   x_e = u on the patch,  h_e = B x_e  (K = 32 modes, B shared, K x NP)
//   s_e = softplus(MLP(f_e))  (K gains from 8 element geometry features,
//                              MLP 8 -> 32 -> 32 -> K with tanh)
//   z   = D^-1/2 ( exp(alpha) u + sum_e P_e^T B^T diag(s_e) B P_e u )
// M is linear in r and symmetric positive definite for every parameter
// value; B = 0, alpha = 0 is Jacobi.
// Parameter vector (FP32), contiguous in this order:
//   B[K][NP] alpha W1T[F][H] b1[H] W2T[H][H] b2[H] W3T[H][K] b3[K]
#pragma once
#include "rhs_kernels.cuh"

namespace sod {

constexpr int NET_H = 32, NET_K = 32, NET_F = 8;

template <int P>
struct NetDims {
  static constexpr int N1 = P + 1, N = N1 * N1 * N1, FACE = N1 * N1, NP = N + 6 * FACE;
  static constexpr int NPP = (NP + 3) / 4 * 4;  // padded patch length for float4 staging
  static constexpr int O_B = 0, O_ALPHA = NET_K * NP, O_W1T = O_ALPHA + 1, O_B1 = O_W1T + NET_F * NET_H,
                       O_W2T = O_B1 + NET_H, O_B2 = O_W2T + NET_H * NET_H, O_W3T = O_B2 + NET_H,
                       O_B3 = O_W3T + NET_H * NET_K, NPARAM = O_B3 + NET_K;
  static constexpr int NMLP = NPARAM - O_W1T;
  static constexpr int EPW = 4;  // elements per warp in the patch kernels
  // dynamic shared memory of the patch kernels (bytes) for `warps` warps
  static constexpr size_t apply_smem(int warps) {
    return (size_t)(2 * NPP * NET_K + warps * EPW * (NPP + NET_K)) * 4;
  }
};

__device__ __forceinline__ float softplusf(float a) { return a > 20.f ? a : log1pf(expf(a)); }
__device__ __forceinline__ float sigmoidf(float a) { return 1.f / (1.f + expf(-a)); }

// Raw geometry features per element (FP64), warp per element: mean
// reference metric G_jk = sum_i dxi_j/dx_i dxi_k/dx_i over the Gauss points,
// vol = sum gpvol.  raw = [log(3 G_bb / tr G) (3), G_01, G_02, G_12
// correlations, log vol, log(tr G) + 2/3 log vol].
template <int P>
__global__ void k_elem_features(MeshDev m, double *__restrict__ raw) {
  constexpr int N = Cfg<P>::N;
  const long long e = (long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  if (e >= m.nelem) return;
  double g[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int t = lane; t < N; t += 32) {
    const float *q = m.geo + e * 10 * N + t;
    double h[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) h[c] = (double)q[c * N];
    auto G = [&](int j, int k) { return h[3 * j] * h[3 * k] + h[3 * j + 1] * h[3 * k + 1] + h[3 * j + 2] * h[3 * k + 2]; };
    g[0] += G(0, 0); g[1] += G(1, 1); g[2] += G(2, 2);
    g[3] += G(0, 1); g[4] += G(0, 2); g[5] += G(1, 2);
    g[6] += (double)q[9 * N];
  }
#pragma unroll
  for (int c = 0; c < 7; ++c)
    for (int o = 16; o > 0; o >>= 1) g[c] += __shfl_xor_sync(0xffffffffu, g[c], o);
  if (lane == 0) {
    for (int c = 0; c < 6; ++c) g[c] /= (double)N;
    const double tr = g[0] + g[1] + g[2];
    double *o = raw + e * NET_F;
    o[0] = log(3.0 * g[0] / tr);
    o[1] = log(3.0 * g[1] / tr);
    o[2] = log(3.0 * g[2] / tr);
    o[3] = g[3] / sqrt(g[0] * g[1]);
    o[4] = g[4] / sqrt(g[0] * g[2]);
    o[5] = g[5] / sqrt(g[1] * g[2]);
    o[6] = log(g[6]);
    o[7] = log(tr) + (2.0 / 3.0) * log(g[6]);
  }
}

// Per-element mode gains s_e = softplus(MLP(f_e)), warp per element (lane =
// hidden unit / mode).
template <int P>
__global__ void k_mlp_gains(long long nelem, const float *__restrict__ feat, const float *__restrict__ prm,
                            float *__restrict__ gains) {
  using D = NetDims<P>;
  constexpr int H = NET_H, K = NET_K;
  const long long e = (long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  if (e >= nelem) return;
  float a = prm[D::O_B1 + lane];
#pragma unroll
  for (int f = 0; f < NET_F; ++f) a = fmaf(prm[D::O_W1T + f * H + lane], feat[e * NET_F + f], a);
  const float h1 = tanhf(a);
  a = prm[D::O_B2 + lane];
#pragma unroll 8
  for (int i = 0; i < H; ++i) a = fmaf(prm[D::O_W2T + i * H + lane], __shfl_sync(0xffffffffu, h1, i), a);
  const float h2 = tanhf(a);
  a = prm[D::O_B3 + lane];
#pragma unroll 8
  for (int i = 0; i < H; ++i) a = fmaf(prm[D::O_W3T + i * K + lane], __shfl_sync(0xffffffffu, h2, i), a);
  gains[e * K + lane] = softplusf(a);
}

// Stage B into shared memory: BT[j][k] (encoder, lane = mode) and, when
// DEC, Bk[k][j] (decoder, lane = patch slot); rows/columns >= NP are zero.
template <int P, bool DEC>
__device__ void stage_B(const float *__restrict__ prm, float *BT, float *Bk) {
  using D = NetDims<P>;
  for (int i = threadIdx.x; i < D::NPP * NET_K; i += blockDim.x) {
    const int j = i / NET_K, k = i % NET_K;
    BT[i] = j < D::NP ? prm[D::O_B + k * D::NP + j] : 0.f;
  }
  if (DEC)
    for (int i = threadIdx.x; i < NET_K * D::NPP; i += blockDim.x) {
      const int k = i / D::NPP, j = i % D::NPP;
      Bk[i] = j < D::NP ? prm[D::O_B + k * D::NP + j] : 0.f;
    }
}

// Gather D^-1/2 v over the patches of EPW elements into xs[EPW][NPP]; per
// element the lane's slot indices are loaded first, then their values.
template <int P>
__device__ __forceinline__ void gather_patch(long long e0, long long nelem, const int *__restrict__ pt,
                                             const double *__restrict__ v, const double *__restrict__ Dh, float *xs,
                                             int lane) {
  using D = NetDims<P>;
  constexpr int JN = (D::NPP + 31) / 32;
#pragma unroll
  for (int el = 0; el < D::EPW; ++el) {
    const long long e = e0 + el;
    int id[JN];
#pragma unroll
    for (int q = 0; q < JN; ++q) {
      const int j = lane + 32 * q;
      id[q] = (e < nelem && j < D::NP) ? pt[e * D::NP + j] : -1;
    }
    double dv[JN], vv[JN];
#pragma unroll
    for (int q = 0; q < JN; ++q) {
      dv[q] = 0.0;
      vv[q] = 0.0;
      if (id[q] >= 0) { dv[q] = Dh[id[q]]; vv[q] = v[id[q]]; }
    }
#pragma unroll
    for (int q = 0; q < JN; ++q) {
      const int j = lane + 32 * q;
      if (j < D::NPP) xs[el * D::NPP + j] = (float)(dv[q] * vv[q]);
    }
  }
}

// h[el] = sum_j B[lane][j] xs[el][j]
template <int P>
__device__ __forceinline__ void encode(const float *BT, const float *xs, int lane, float (&h)[NetDims<P>::EPW]) {
  using D = NetDims<P>;
#pragma unroll
  for (int el = 0; el < D::EPW; ++el) h[el] = 0.f;
#pragma unroll 2
  for (int j = 0; j < D::NPP; j += 4) {
    const float b0 = BT[(j + 0) * NET_K + lane], b1 = BT[(j + 1) * NET_K + lane];
    const float b2 = BT[(j + 2) * NET_K + lane], b3 = BT[(j + 3) * NET_K + lane];
#pragma unroll
    for (int el = 0; el < D::EPW; ++el) {
      const float4 x = *reinterpret_cast<const float4 *>(xs + el * D::NPP + j);
      h[el] = fmaf(b0, x.x, fmaf(b1, x.y, fmaf(b2, x.z, fmaf(b3, x.w, h[el]))));
    }
  }
}

// Inference: per element o_e = B^T diag(s_e) B x_e written to patch slots
// [e][NP] (FP32).  EPW elements per warp, grid-stride over element groups.
template <int P>
__global__ void __launch_bounds__(256)
k_patch_apply(long long nelem, const int *__restrict__ pt, const double *__restrict__ r,
              const double *__restrict__ Dh, const float *__restrict__ prm, const float *__restrict__ gains,
              float *__restrict__ slots) {
  using D = NetDims<P>;
  constexpr int NPP = D::NPP, K = NET_K, EPW = D::EPW;
  extern __shared__ __align__(16) float smem[];
  float *BT = smem, *Bk = smem + NPP * K;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32, nwarps = blockDim.x / 32;
  float *xs = Bk + K * NPP + warp * EPW * (NPP + K), *ys = xs + EPW * NPP;
  stage_B<P, true>(prm, BT, Bk);
  __syncthreads();
  for (long long g = (long long)blockIdx.x * nwarps + warp; g * EPW < nelem; g += (long long)gridDim.x * nwarps) {
    const long long e0 = g * EPW;
    gather_patch<P>(e0, nelem, pt, r, Dh, xs, lane);
    __syncwarp();
    float h[EPW];
    encode<P>(BT, xs, lane, h);
#pragma unroll
    for (int el = 0; el < EPW; ++el) ys[el * K + lane] = (e0 + el < nelem) ? gains[(e0 + el) * K + lane] * h[el] : 0.f;
    __syncwarp();
    for (int j = lane; j < D::NP; j += 32) {
      float o[EPW];
#pragma unroll
      for (int el = 0; el < EPW; ++el) o[el] = 0.f;
#pragma unroll 2
      for (int k = 0; k < K; k += 4) {
        const float b0 = Bk[(k + 0) * NPP + j], b1 = Bk[(k + 1) * NPP + j];
        const float b2 = Bk[(k + 2) * NPP + j], b3 = Bk[(k + 3) * NPP + j];
#pragma unroll
        for (int el = 0; el < EPW; ++el) {
          const float4 y = *reinterpret_cast<const float4 *>(ys + el * K + k);
          o[el] = fmaf(b0, y.x, fmaf(b1, y.y, fmaf(b2, y.z, fmaf(b3, y.w, o[el]))));
        }
      }
#pragma unroll
      for (int el = 0; el < EPW; ++el)
        if (e0 + el < nelem) slots[(e0 + el) * D::NP + j] = o[el];
    }
    __syncwarp();
  }
}

// ---- tensor-core inference (mma.sync m16n8k8, TF32 operands, FP32 accumulate)
// Each warp applies the patch operator to 16 elements at a time:
//   H[16 x K] = X[16 x NP] B^T,  Y = gains * H,  O[16 x NP] = Y B.
// Operands are staged in shared memory with row strides chosen so that the
// fragment loads are free of bank conflicts.
// The B fragment of an m16n8k8 step is the pair (k0 + t, k0 + t + 4) of the
// k index; both copies of B in shared memory store each block of 8 k values
// in the order 0 4 1 5 2 6 3 7, so that the pair is one aligned 8-byte load.
// Row strides of 8 or 24 mod 32 words keep those loads free of bank
// conflicts.
__host__ __device__ constexpr int kpair_pos(int k) {
  const int r = k & 7;
  return (k & ~7) | (r < 4 ? 2 * r : 2 * (r - 4) + 1);
}
__host__ __device__ constexpr int stride_8_24(int n) { return n + ((8 - n % 16) + 16) % 16; }

template <int P>
struct TcDims {
  using D = NetDims<P>;
  static constexpr int KP = (D::NP + 7) / 8 * 8;                   // slots padded to the mma k/n step
  static constexpr int S1 = stride_8_24(KP);                       // B as [mode][slot, paired]
  static constexpr int S2 = stride_8_24(NET_K);                    // B as [slot][mode, paired]
  static constexpr int SY = NET_K + 4;                             // Y tile [16][SY]
  static constexpr int WARPS = 16;                                 // one block per SM
  static constexpr int KC = 10;                                    // k-steps whose operands are gathered together
  static constexpr int NC = 10;                                    // output n-tiles whose positions are loaded together
  static constexpr size_t smem() { return (size_t)(NET_K * S1 + KP * S2 + WARPS * 16 * SY) * 4; }
};

__device__ __forceinline__ void mma_tf32(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// uf = (float)(D^-1/2 r) over the working nodes
static __global__ void k_scale_f32(int npoin_w, const int *__restrict__ lpoin_w, const double *__restrict__ r,
                            const double *__restrict__ Dh, float *__restrict__ uf) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const int i = lpoin_w[t];
  uf[i] = (float)(Dh[i] * r[i]);
}

// Each lane gathers exactly the A-fragment entries it needs (rows g, g+8 of
// the 16 patches, columns t, t+4 of each k-step) straight from the patch
// table, so no X tile is staged; outputs go to their node-ordered positions
// pos[e][j] so that the assembly reads each node's contributions
// contiguously.
template <int P>
__global__ void __launch_bounds__(TcDims<P>::WARPS * 32)
k_patch_apply_tc(long long nelem, const int *__restrict__ pt, const int *__restrict__ pos,
                 const float *__restrict__ uf, const float *__restrict__ prm, const float *__restrict__ gains,
                 float *__restrict__ out, const int *__restrict__ stop) {
  using D = NetDims<P>;
  using T = TcDims<P>;
  constexpr int NP = D::NP, KP = T::KP, K = NET_K, NT2 = KP / 8, KS = KP / 8, KC = T::KC;
  if (stop && *stop) return;
  extern __shared__ __align__(16) float smem[];
  float *B1 = smem, *B2 = B1 + K * T::S1;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  float *Y = B2 + KP * T::S2 + warp * 16 * T::SY;
  for (int i = threadIdx.x; i < K * KP; i += blockDim.x) {
    const int k = i / KP, j = i % KP;
    const float b = j < NP ? prm[D::O_B + k * NP + j] : 0.f;
    B1[k * T::S1 + kpair_pos(j)] = b;
    B2[j * T::S2 + kpair_pos(k)] = b;
  }
  __syncthreads();
  const int g = lane >> 2, t = lane & 3;
  const long long ngroups = (nelem + 15) / 16;
  // groups dealt round-robin over the blocks, so that every SM holds the
  // same number of groups to within one
  for (long long grp = (long long)warp * gridDim.x + blockIdx.x; grp < ngroups;
       grp += (long long)gridDim.x * T::WARPS) {
    const long long ea = grp * 16 + g, eb = ea + 8;
    const bool va = ea < nelem, vb = eb < nelem;
    const int *pa = pt + ea * NP, *pb = pt + eb * NP;
    // H = X B^T : 4 n-tiles of 8 modes, KS k-steps gathered KC at a time
    float h[4][4];
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q) h[nt][q] = 0.f;
#pragma unroll 1
    for (int c0 = 0; c0 < KS; c0 += KC) {
      int id[KC][4];
#pragma unroll
      for (int kk = 0; kk < KC; ++kk) {
        const int k0 = (c0 + kk) * 8, ca = k0 + t, cb = k0 + t + 4;
        const bool in = c0 + kk < KS;
        id[kk][0] = (in && va && ca < NP) ? pa[ca] : -1;
        id[kk][1] = (in && vb && ca < NP) ? pb[ca] : -1;
        id[kk][2] = (in && va && cb < NP) ? pa[cb] : -1;
        id[kk][3] = (in && vb && cb < NP) ? pb[cb] : -1;
      }
      float xv[KC][4];
#pragma unroll
      for (int kk = 0; kk < KC; ++kk)
#pragma unroll
        for (int q = 0; q < 4; ++q) xv[kk][q] = id[kk][q] >= 0 ? uf[id[kk][q]] : 0.f;
#pragma unroll
      for (int kk = 0; kk < KC; ++kk) {
        if (c0 + kk >= KS) break;
        const int k0 = (c0 + kk) * 8;
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          const float2 bb = *reinterpret_cast<const float2 *>(B1 + (nt * 8 + g) * T::S1 + k0 + 2 * t);
          mma_tf32(h[nt], __float_as_uint(xv[kk][0]), __float_as_uint(xv[kk][1]), __float_as_uint(xv[kk][2]),
                   __float_as_uint(xv[kk][3]), __float_as_uint(bb.x), __float_as_uint(bb.y));
        }
      }
    }
    // Y = gains * H (through shared memory into the A-fragment layout)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      const int col = nt * 8 + 2 * t;
      const float2 sa = va ? *reinterpret_cast<const float2 *>(gains + ea * K + col) : make_float2(0.f, 0.f);
      const float2 sb = vb ? *reinterpret_cast<const float2 *>(gains + eb * K + col) : make_float2(0.f, 0.f);
      Y[g * T::SY + col] = sa.x * h[nt][0];
      Y[g * T::SY + col + 1] = sa.y * h[nt][1];
      Y[(g + 8) * T::SY + col] = sb.x * h[nt][2];
      Y[(g + 8) * T::SY + col + 1] = sb.y * h[nt][3];
    }
    __syncwarp();
    uint32_t a[4][4];
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      const int k0 = kk * 8;
      a[kk][0] = __float_as_uint(Y[g * T::SY + k0 + t]);
      a[kk][1] = __float_as_uint(Y[(g + 8) * T::SY + k0 + t]);
      a[kk][2] = __float_as_uint(Y[g * T::SY + k0 + t + 4]);
      a[kk][3] = __float_as_uint(Y[(g + 8) * T::SY + k0 + t + 4]);
    }
    __syncwarp();
    // O = Y B : KP/8 n-tiles of 8 slots, 4 k-steps; scattered to pos, whose
    // entries are loaded NC n-tiles at a time
    const int *qa = pos + ea * NP, *qb = pos + eb * NP;
#pragma unroll 1
    for (int n0 = 0; n0 < NT2; n0 += T::NC) {
      int w[T::NC][4];
#pragma unroll
      for (int nn = 0; nn < T::NC; ++nn) {
        const int col = (n0 + nn) * 8 + 2 * t;
        const bool in = n0 + nn < NT2;
        w[nn][0] = (in && va && col < NP) ? qa[col] : -1;
        w[nn][1] = (in && va && col + 1 < NP) ? qa[col + 1] : -1;
        w[nn][2] = (in && vb && col < NP) ? qb[col] : -1;
        w[nn][3] = (in && vb && col + 1 < NP) ? qb[col + 1] : -1;
      }
#pragma unroll
      for (int nn = 0; nn < T::NC; ++nn) {
        if (n0 + nn >= NT2) break;
        const int nt = n0 + nn;
        float o[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
          const int k0 = kk * 8;
          const float2 bb = *reinterpret_cast<const float2 *>(B2 + (nt * 8 + g) * T::S2 + k0 + 2 * t);
          mma_tf32(o, a[kk][0], a[kk][1], a[kk][2], a[kk][3], __float_as_uint(bb.x), __float_as_uint(bb.y));
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (w[nn][q] >= 0) out[w[nn][q]] = o[q];
      }
    }
  }
}

// z(n) = D^-1/2(n) (exp(alpha) D^-1/2(n) r(n) + sum of the node's
// contributions, stored contiguously from pptr[n]), FP64.
static __global__ void k_patch_gather_perm(long long npoin, const int *__restrict__ pptr, const float *__restrict__ ctr,
                                    const double *__restrict__ r, const double *__restrict__ Dh,
                                    const float *__restrict__ prm, int o_alpha, double *__restrict__ z) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= npoin) return;
  const int b = pptr[n], en = pptr[n + 1];
  if (b == en) return;
  double acc = 0.0;
  for (int s = b; s < en; ++s) acc += (double)ctr[s];
  const double d = Dh[n];
  z[n] = d * (exp((double)prm[o_alpha]) * d * r[n] + acc);
}

// z(n) = D^-1/2(n) (exp(alpha) D^-1/2(n) r(n) + sum of the node's patch
// slots), FP64, for nodes that own patch slots (the working nodes).
static __global__ void k_patch_gather(long long npoin, const int *__restrict__ pptr, const int *__restrict__ pslot,
                               const float *__restrict__ slots, const double *__restrict__ r,
                               const double *__restrict__ Dh, const float *__restrict__ prm, int o_alpha,
                               double *__restrict__ z) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= npoin) return;
  const int b = pptr[n], en = pptr[n + 1];
  if (b == en) return;
  double acc = 0.0;
  for (int s = b; s < en; ++s) acc += (double)slots[pslot[s]];
  const double d = Dh[n];
  z[n] = d * (exp((double)prm[o_alpha]) * d * r[n] + acc);
}

// Training backward of the patch operator with its B-gradient reduction.
// Per element: x = patch of D^-1/2 r, w = patch of D^-1/2 g (g = dL/dz),
// h = B x, a = B w; dS = h a (dL/ds) goes to global memory for the gain
// MLP, and
//   dB[k][j] += Y[e][k] W[e][j] + SA[e][k] X[e][j],  Y = s h, SA = s a,
// is summed in registers: every round the block's 8 warps stage the rows of
// 4 elements each in shared memory, and each thread adds them to its tile
// of 4 modes x JB slots, in (warp, element) order.  Block b writes its tile
// to part[b * stride + O_B + k NP + j], or adds it there (accumulate: the
// samples of a batch, one launch each, in order; all of it deterministic).
template <int P>
struct BwdDims {
  using D = NetDims<P>;
  static constexpr int WARPS = 8, JB = (D::NP + 31) / 32;
  static constexpr int ROW = 2 * D::EPW * D::NPP + 2 * D::EPW * NET_K;  // floats per warp: x, w, Y, SA rows
  static constexpr size_t smem() { return (size_t)(D::NPP * NET_K + WARPS * ROW) * 4; }
};

template <int P>
__global__ void __launch_bounds__(256)
k_patch_bwd_dB(long long nelem, const int *__restrict__ pt, const double *__restrict__ r,
               const double *__restrict__ g, const double *__restrict__ Dh, const float *__restrict__ prm,
               const float *__restrict__ gains, float *__restrict__ dS, float *__restrict__ part, long long stride,
               int accumulate) {
  using D = NetDims<P>;
  using Q = BwdDims<P>;
  constexpr int NPP = D::NPP, NP = D::NP, K = NET_K, EPW = D::EPW, WARPS = Q::WARPS, JB = Q::JB;
  static_assert(K == 32, "8 blocks of 4 modes");
  extern __shared__ __align__(16) float smem[];
  float *BT = smem;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  auto xs_of = [&](int w) { return BT + NPP * K + w * Q::ROW; };
  float *xs = xs_of(warp), *ws = xs + EPW * NPP, *ys = ws + EPW * NPP, *sas = ys + EPW * K;
  stage_B<P, false>(prm, BT, nullptr);
  const int k0 = 4 * (threadIdx.x / 32), j0 = JB * (threadIdx.x % 32);
  float acc[4][JB];
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int b = 0; b < JB; ++b) acc[q][b] = 0.f;
  __syncthreads();
  const long long ngroups = (nelem + EPW - 1) / EPW;
  for (long long base = (long long)blockIdx.x * WARPS; base < ngroups; base += (long long)gridDim.x * WARPS) {
    const long long e0 = (base + warp) * EPW;  // past the end: zero rows, no contribution
    gather_patch<P>(e0, nelem, pt, r, Dh, xs, lane);
    gather_patch<P>(e0, nelem, pt, g, Dh, ws, lane);
    __syncwarp();
    float h[EPW], a[EPW];
    encode<P>(BT, xs, lane, h);
    encode<P>(BT, ws, lane, a);
#pragma unroll
    for (int el = 0; el < EPW; ++el) {
      const long long e = e0 + el;
      const float sg = e < nelem ? gains[e * K + lane] : 0.f;
      ys[el * K + lane] = sg * h[el];
      sas[el * K + lane] = sg * a[el];
      if (e < nelem) dS[e * K + lane] = h[el] * a[el];
    }
    __syncthreads();  // the round's rows of every warp are staged
    for (int w = 0; w < WARPS; ++w) {
      const float *xw = xs_of(w), *ww = xw + EPW * NPP, *yw = ww + EPW * NPP, *sw = yw + EPW * K;
#pragma unroll
      for (int el = 0; el < EPW; ++el) {
        const float4 y4 = *reinterpret_cast<const float4 *>(yw + el * K + k0);
        const float4 s4 = *reinterpret_cast<const float4 *>(sw + el * K + k0);
        const float yv[4] = {y4.x, y4.y, y4.z, y4.w}, sv[4] = {s4.x, s4.y, s4.z, s4.w};
        float wv[JB], xv[JB];
#pragma unroll
        for (int b = 0; b < JB; ++b) {
          const bool in = j0 + b < NP;
          wv[b] = in ? ww[el * NPP + j0 + b] : 0.f;
          xv[b] = in ? xw[el * NPP + j0 + b] : 0.f;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int b = 0; b < JB; ++b) acc[q][b] = fmaf(yv[q], wv[b], fmaf(sv[q], xv[b], acc[q][b]));
      }
    }
    __syncthreads();  // the rows are rewritten by the next round
  }
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int b = 0; b < JB; ++b)
      if (j0 + b < NP) {
        float *o = part + blockIdx.x * stride + D::O_B + (k0 + q) * NP + j0 + b;
        *o = (accumulate ? *o : 0.f) + acc[q][b];
      }
}

// Gradient of the gain MLP from dS = dL/ds; block b covers the contiguous
// element range [b E / nb, (b+1) E / nb).  The weights are staged in shared
// memory (W2 and W3 also transposed, so the backward matrix-vector products
// read rows lane by lane); each lane accumulates its column of every weight
// gradient in registers over its warp's elements, and the block adds the
// warps' gradients in warp order into part, or onto it (accumulate).
template <int P>
__global__ void __launch_bounds__(256)
k_mlp_bwd(long long nelem, const float *__restrict__ feat, const float *__restrict__ prm,
          const float *__restrict__ dS, float *__restrict__ part, long long stride, int accumulate) {
  using D = NetDims<P>;
  constexpr int H = NET_H, K = NET_K, F = NET_F, NM = D::NMLP;
  static_assert(H == 32 && K == 32, "one lane per hidden unit and per mode");
  constexpr int R_W1T = 0, R_B1 = R_W1T + F * H, R_W2T = R_B1 + H, R_B2 = R_W2T + H * H, R_W3T = R_B2 + H,
                R_B3 = R_W3T + H * K;
  __shared__ float sW1T[F * H], sb1[H], sW2T[H * H], sW2[H * H], sb2[H], sW3T[H * K], sW3[K * H], sb3[K];
  __shared__ float acc[NM];
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32, nwarps = blockDim.x / 32;
  for (int i = threadIdx.x; i < H * H; i += blockDim.x) {
    const int r = i / H, q = i % H;
    sW2T[i] = prm[D::O_W2T + i];
    sW3T[i] = prm[D::O_W3T + i];
    sW2[q * H + r] = prm[D::O_W2T + i];  // sW2[j][l] = W2T[l][j]
    sW3[q * H + r] = prm[D::O_W3T + i];  // sW3[k][l] = W3T[l][k]
  }
  for (int i = threadIdx.x; i < F * H; i += blockDim.x) sW1T[i] = prm[D::O_W1T + i];
  for (int i = threadIdx.x; i < H; i += blockDim.x) {
    sb1[i] = prm[D::O_B1 + i];
    sb2[i] = prm[D::O_B2 + i];
    sb3[i] = prm[D::O_B3 + i];
  }
  for (int i = threadIdx.x; i < NM; i += blockDim.x) acc[i] = 0.f;
  __syncthreads();
  float g3[H], g2[H], g1[F], gb3 = 0.f, gb2 = 0.f, gb1 = 0.f;
#pragma unroll
  for (int i = 0; i < H; ++i) { g3[i] = 0.f; g2[i] = 0.f; }
#pragma unroll
  for (int q = 0; q < F; ++q) g1[q] = 0.f;
  const long long lo = nelem * blockIdx.x / gridDim.x, hi = nelem * (blockIdx.x + 1) / gridDim.x;
  for (long long e = lo + warp; e < hi; e += nwarps) {
    float f[F];
#pragma unroll
    for (int q = 0; q < F; ++q) f[q] = feat[e * F + q];
    float a = sb1[lane];
#pragma unroll
    for (int q = 0; q < F; ++q) a = fmaf(sW1T[q * H + lane], f[q], a);
    const float h1 = tanhf(a);
    a = sb2[lane];
#pragma unroll
    for (int i = 0; i < H; ++i) a = fmaf(sW2T[i * H + lane], __shfl_sync(0xffffffffu, h1, i), a);
    const float h2 = tanhf(a);
    a = sb3[lane];
#pragma unroll
    for (int i = 0; i < H; ++i) a = fmaf(sW3T[i * K + lane], __shfl_sync(0xffffffffu, h2, i), a);
    const float dO = dS[e * K + lane] * sigmoidf(a);  // lane = mode
    // layer 3
    gb3 += dO;
#pragma unroll
    for (int i = 0; i < H; ++i) g3[i] += __shfl_sync(0xffffffffu, h2, i) * dO;
    float dh2 = 0.f;  // lane = hidden unit
#pragma unroll
    for (int k = 0; k < K; ++k) dh2 = fmaf(sW3[k * H + lane], __shfl_sync(0xffffffffu, dO, k), dh2);
    const float dz2 = dh2 * (1.f - h2 * h2);
    // layer 2
    gb2 += dz2;
#pragma unroll
    for (int i = 0; i < H; ++i) g2[i] += __shfl_sync(0xffffffffu, h1, i) * dz2;
    float dh1 = 0.f;
#pragma unroll
    for (int j = 0; j < H; ++j) dh1 = fmaf(sW2[j * H + lane], __shfl_sync(0xffffffffu, dz2, j), dh1);
    const float dz1 = dh1 * (1.f - h1 * h1);
    // layer 1
    gb1 += dz1;
#pragma unroll
    for (int q = 0; q < F; ++q) g1[q] += f[q] * dz1;
  }
  for (int w = 0; w < nwarps; ++w) {
    if (warp == w) {
      acc[R_B3 + lane] += gb3;
      acc[R_B2 + lane] += gb2;
      acc[R_B1 + lane] += gb1;
#pragma unroll
      for (int i = 0; i < H; ++i) {
        acc[R_W3T + i * K + lane] += g3[i];
        acc[R_W2T + i * H + lane] += g2[i];
      }
#pragma unroll
      for (int q = 0; q < F; ++q) acc[R_W1T + q * H + lane] += g1[q];
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < NM; i += blockDim.x) {
    float *o = part + blockIdx.x * stride + D::O_W1T + i;
    *o = (accumulate ? *o : 0.f) + acc[i];
  }
}

// dL/dalpha partial: exp(alpha) sum over the block's working nodes of
// (D^-1/2 g)(D^-1/2 r), written to part[b * stride + o_alpha].
static __global__ void k_alpha_part(int npoin_w, const int *__restrict__ lpoin_w, const double *__restrict__ r,
                             const double *__restrict__ g, const double *__restrict__ Dh,
                             const float *__restrict__ prm, int o_alpha, float *__restrict__ part, long long stride,
                             int accumulate) {
  __shared__ double sh[256];
  const long long lo = (long long)npoin_w * blockIdx.x / gridDim.x,
                  hi = (long long)npoin_w * (blockIdx.x + 1) / gridDim.x;
  double s = 0.0;
  for (long long t = lo + threadIdx.x; t < hi; t += blockDim.x) {
    const int n = lpoin_w[t];
    s += (Dh[n] * g[n]) * (Dh[n] * r[n]);
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    float *o = part + blockIdx.x * stride + o_alpha;
    *o = (accumulate ? *o : 0.f) + (float)(exp((double)prm[o_alpha]) * sh[0]);
  }
}

// grad[i] = sum over blocks of part[b][i] (fixed order), then Adam.
static __global__ void k_adam(int nparam, int nblocks, const float *__restrict__ part, float *__restrict__ params,
                       float *__restrict__ m1, float *__restrict__ m2, float lr, float b1, float b2, float eps,
                       float bc1, float bc2, float gscale, float *__restrict__ grad_out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nparam) return;
  float g = 0.f;
  for (int b = 0; b < nblocks; ++b) g += part[(long long)b * nparam + i];
  g *= gscale;
  if (grad_out) grad_out[i] = g;
  if (lr == 0.f) return;
  const float a = b1 * m1[i] + (1.f - b1) * g;
  const float v = b2 * m2[i] + (1.f - b2) * g * g;
  m1[i] = a;
  m2[i] = v;
  params[i] -= lr * (a / bc1) / (sqrtf(v / bc2) + eps);
}

}  // namespace sod
