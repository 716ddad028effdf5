// Learned element-patch preconditioner for the pressure Poisson problem:
// forward (inference and training), backward and Adam kernels.
//
// Network, per element e (P = element order, N = (P+1)^3 nodes):
//   input  x  = [ (r * Minv)(nodes of e) (N values, tensor order),
//                 mean of (r * Minv) over each of the 6 face neighbours ]
//   scale  s  = RMS(x) (the map is positively homogeneous: M(a r) = a M(r))
//   h1 = tanh(W1 x/s + b1)   (32)
//   h2 = tanh(W2 h1 + b2)    (32)
//   y  = W3 h2 + b3          (N)
//   contribution to z at node(e,a): s * w(e,a) * (x[a]/s + y[a]), w =
//   1/(elements sharing the node), summed over elements in a fixed order.
//   The skip term makes the map Jacobi (z = r/diag) when W3 = b3 = 0, the
//   initial state; training adds a learned correction.
// Parameter vector (FP32), contiguous in this order:
//   W1T[NIN][H] b1[H] W2T[H][H] b2[H] W3T[H][N] b3[N]
// (the transposed blocks make the per-lane reads of the forward pass
// conflict-free in shared memory).
#pragma once
#include "rhs_kernels.cuh"

namespace sod {

constexpr int NET_H = 32;

template <int P>
struct NetDims {
  static constexpr int N = (P + 1) * (P + 1) * (P + 1);
  static constexpr int NIN = N + 6;
  static constexpr int O_W1T = 0;
  static constexpr int O_B1 = O_W1T + NIN * NET_H;
  static constexpr int O_W2T = O_B1 + NET_H;
  static constexpr int O_B2 = O_W2T + NET_H * NET_H;
  static constexpr int O_W3T = O_B2 + NET_H;
  static constexpr int O_B3 = O_W3T + NET_H * N;
  static constexpr int NPARAM = O_B3 + N;
  // saved activations per element: s, x/s (NIN), h1 (H), h2 (H)
  static constexpr int NACT = 1 + NIN + 2 * NET_H;
};

// Mean of (r*Minv) over each element.
__global__ void k_elem_mean(MeshDev m, int N, const double *__restrict__ r, const double *__restrict__ Minv,
                            float *__restrict__ mean) {
  const long long e = (long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  if (e >= m.nelem) return;
  float s = 0.f;
  for (int t = lane; t < N; t += 32) {
    const int p = m.conn[e * N + t];
    s += (float)(r[p] * Minv[p]);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) mean[e] = s / (float)N;
}

// Forward pass, one warp per element (grid-stride), parameters staged in
// shared memory.  TRAIN saves the activations needed by the backward pass.
template <int P, bool TRAIN>
__global__ void __launch_bounds__(256)
k_net_fwd(MeshDev m, const int *__restrict__ nbr, const float *__restrict__ emean, const double *__restrict__ r,
          const double *__restrict__ Minv, const float *__restrict__ wts, const float *__restrict__ params,
          float *__restrict__ out_slots, float *__restrict__ act) {
  using D = NetDims<P>;
  constexpr int N = D::N, NIN = D::NIN, H = NET_H;
  extern __shared__ float smem[];
  float *W = smem;                              // NPARAM
  float *scr = smem + D::NPARAM;                // per warp: NIN + 2H
  for (int i = threadIdx.x; i < D::NPARAM; i += blockDim.x) W[i] = params[i];
  __syncthreads();
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32, nwarps = blockDim.x / 32;
  float *x = scr + warp * (NIN + 2 * H), *h1 = x + NIN, *h2 = h1 + H;
  for (long long e = (long long)blockIdx.x * nwarps + warp; e < m.nelem; e += (long long)gridDim.x * nwarps) {
    float ss = 0.f;
    for (int t = lane; t < N; t += 32) {
      const int p = m.conn[e * N + t];
      const float v = (float)(r[p] * Minv[p]);
      x[t] = v;
      ss += v * v;
    }
    if (lane < 6) {
      const float v = emean[nbr[e * 6 + lane]];
      x[N + lane] = v;
      ss += v * v;
    }
    for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    const float s = sqrtf(ss / (float)NIN);
    const float inv = s > 0.f ? 1.f / s : 0.f;
    __syncwarp();
    for (int t = lane; t < NIN; t += 32) x[t] *= inv;
    __syncwarp();
    float a = W[D::O_B1 + lane];
    for (int i = 0; i < NIN; ++i) a = fmaf(W[D::O_W1T + i * H + lane], x[i], a);
    h1[lane] = tanhf(a);
    __syncwarp();
    a = W[D::O_B2 + lane];
#pragma unroll 8
    for (int i = 0; i < H; ++i) a = fmaf(W[D::O_W2T + i * H + lane], h1[i], a);
    h2[lane] = tanhf(a);
    __syncwarp();
    for (int o = lane; o < N; o += 32) {
      float y = W[D::O_B3 + o];
#pragma unroll 8
      for (int j = 0; j < H; ++j) y = fmaf(W[D::O_W3T + j * N + o], h2[j], y);
      out_slots[e * N + o] = s * wts[e * N + o] * (x[o] + y);
    }
    if (TRAIN) {
      float *ac = act + e * D::NACT;
      if (lane == 0) ac[0] = s;
      for (int t = lane; t < NIN; t += 32) ac[1 + t] = x[t];
      ac[1 + NIN + lane] = h1[lane];
      ac[1 + NIN + H + lane] = h2[lane];
    }
    __syncwarp();
  }
}

// Backward pass: g = dL/dz at nodes (FP64).  Each warp accumulates the
// parameter gradient of its elements in its own shared-memory slice; the
// block sums its slices in warp order and writes one partial per block
// (deterministic).  Shared memory: params + transposed copies + nwarps
// gradient slices.
template <int P>
__global__ void __launch_bounds__(256)
k_net_bwd(MeshDev m, const double *__restrict__ g, const float *__restrict__ wts, const float *__restrict__ params,
          const float *__restrict__ act, float *__restrict__ part) {
  using D = NetDims<P>;
  constexpr int N = D::N, NIN = D::NIN, H = NET_H, NP = D::NPARAM;
  extern __shared__ float smem[];
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32, nwarps = blockDim.x / 32;
  float *W = smem;                 // NP (transposed layout as the parameter vector)
  float *W3 = W + NP;              // [N][H] row-major (a, j)
  float *W2 = W3 + N * H;          // [H][H] row-major (j, i)
  float *G = W2 + H * H;           // nwarps x NP gradient slices
  float *scr = G + nwarps * NP;    // per warp: N (dy) + 2H
  for (int i = threadIdx.x; i < NP; i += blockDim.x) W[i] = params[i];
  __syncthreads();
  for (int i = threadIdx.x; i < N * H; i += blockDim.x) {
    const int a = i / H, j = i % H;
    W3[i] = W[D::O_W3T + j * N + a];
  }
  for (int i = threadIdx.x; i < H * H; i += blockDim.x) {
    const int j = i / H, ii = i % H;
    W2[i] = W[D::O_W2T + ii * H + j];
  }
  for (int i = threadIdx.x; i < nwarps * NP; i += blockDim.x) G[i] = 0.f;
  __syncthreads();
  float *Gw = G + warp * NP;
  float *dy = scr + warp * (N + 2 * H), *dz2 = dy + N, *dz1 = dz2 + H;
  for (long long e = (long long)blockIdx.x * nwarps + warp; e < m.nelem; e += (long long)gridDim.x * nwarps) {
    const float *ac = act + e * D::NACT;
    const float s = ac[0];
    const float *x = ac + 1, *h1 = x + NIN, *h2 = h1 + H;
    for (int o = lane; o < N; o += 32) {
      const int p = m.conn[e * N + o];
      dy[o] = (float)g[p] * s * wts[e * N + o];
    }
    __syncwarp();
    // layer 3: dW3T[j][a] += dy[a] h2[j], db3[a] += dy[a]
    for (int o = lane; o < N; o += 32) {
      Gw[D::O_B3 + o] += dy[o];
      for (int j = 0; j < H; ++j) Gw[D::O_W3T + j * N + o] += dy[o] * h2[j];
    }
    float dh2 = 0.f;
    for (int o = 0; o < N; ++o) dh2 = fmaf(W3[o * H + lane], dy[o], dh2);
    const float hv2 = h2[lane];
    dz2[lane] = dh2 * (1.f - hv2 * hv2);
    __syncwarp();
    // layer 2: dW2T[i][j] += dz2[j] h1[i]
    Gw[D::O_B2 + lane] += dz2[lane];
    for (int i = 0; i < H; ++i) Gw[D::O_W2T + i * H + lane] += dz2[lane] * h1[i];
    float dh1 = 0.f;
    for (int j = 0; j < H; ++j) dh1 = fmaf(W2[j * H + lane], dz2[j], dh1);
    const float hv1 = h1[lane];
    dz1[lane] = dh1 * (1.f - hv1 * hv1);
    __syncwarp();
    // layer 1: dW1T[i][j] += dz1[j] x[i]
    Gw[D::O_B1 + lane] += dz1[lane];
    for (int i = 0; i < NIN; ++i) Gw[D::O_W1T + i * H + lane] += dz1[lane] * x[i];
    __syncwarp();
  }
  __syncthreads();
  for (int i = threadIdx.x; i < NP; i += blockDim.x) {
    float s = 0.f;
    for (int w = 0; w < nwarps; ++w) s += G[w * NP + i];
    part[(long long)blockIdx.x * NP + i] = s;
  }
}

// grad[i] = sum over blocks of part[b][i] (fixed order), then Adam.
__global__ void k_adam(int nparam, int nblocks, const float *__restrict__ part, float *__restrict__ params,
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
