// Node kernels of the IMEX time integrator (imex_main,
// src/lib_sod2d/sources/time_integ_imex.f90:181-525) and of its implicit
// solve (conjGrad_imex, src/lib_sod2d/sources/mod_solver_imex.f90:25-342).
//
// Five-variable blocks are stored [mass N][energy N][momentum 3N], the
// order of the reference's x_vars(:,1..5).  Arithmetic is FP32 with the
// reference's operation order; the _rn intrinsics keep the compiler from
// contracting products into FMAs, so that the stage sums round as the
// reference's do.
#pragma once

namespace sod {

// Butcher tables, 1-based (ae explicit, ai implicit)
struct ImexCoef {
  float ae[5][5], ai[5][5];
};

// Stage right-hand side over all nodes, time_integ_imex.f90:342-391 (no
// source, wall model or buoyancy):
//   U2 = -dt R_stab - sum_{j<is} (dt ae(is,j) R_j + dt ai(is,j) D_j) + U1 Ml
// R, D: stage-major five-variable blocks; stab, lvl1: five-variable blocks.
static __global__ void k_imex_comb(long long npoin, int is, ImexCoef k, float dt, const float *__restrict__ Ml,
                            const float *__restrict__ R, const float *__restrict__ D, const float *__restrict__ stab,
                            const float *__restrict__ lvl1, float *__restrict__ rho2, float *__restrict__ E2,
                            float *__restrict__ q2) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npoin) return;
  const long long B = 5 * npoin;
  const float ml = Ml[p];
  float *out[5] = {rho2, E2, q2, q2 + npoin, q2 + 2 * npoin};
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    const long long o = p + npoin * v;
    float a = __fmul_rn(-dt, stab[o]);
    for (int js = 1; js < is; ++js) {
      a = __fsub_rn(a, __fmul_rn(__fmul_rn(dt, k.ae[is][js]), R[(js - 1) * B + o]));
      a = __fsub_rn(a, __fmul_rn(__fmul_rn(dt, k.ai[is][js]), D[(js - 1) * B + o]));
    }
    out[v][p] = __fadd_rn(a, __fmul_rn(lvl1[o], ml));
  }
}

// h = gamma/(gamma-1) p / rho over the working nodes (time_integ_imex.f90:433)
static __global__ void k_aux_h(int npoin_w, const int *__restrict__ lpoin_w, float g_gm1, const float *__restrict__ rho,
                        const float *__restrict__ pr, float *__restrict__ h) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const int p = lpoin_w[t];
  h[p] = __fdiv_rn(__fmul_rn(g_gm1, pr[p]), rho[p]);
}

// Velocity and temperature of the CG argument v over the iterate's density
// (mod_solver_imex.f90:97-107, 160-167, 310-320): u = v_mom / x_mass,
// T = x_mass (gamma-1) (v_E / x_mass - |u|^2/2) / (x_mass Rgas).
static __global__ void k_imex_prim(int npoin_w, long long npoin, const int *__restrict__ lpoin_w, float gm1, float Rgas,
                            const float *__restrict__ x, const float *__restrict__ v, float *__restrict__ au,
                            float *__restrict__ aT) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const long long p = lpoin_w[t];
  const float rhol = x[p], El = v[p + npoin];
  float umag = 0.f;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float ud = __fdiv_rn(v[p + npoin * (2 + d)], rhol);
    au[p + npoin * d] = ud;
    umag = __fadd_rn(umag, __fmul_rn(ud, ud));
  }
  const float e = __fsub_rn(__fdiv_rn(El, rhol), __fmul_rn(0.5f, umag));
  aT[p] = __fdiv_rn(__fmul_rn(__fmul_rn(rhol, gm1), e), __fmul_rn(rhol, Rgas));
}

// qn = v Ml + qn fact dt over the working nodes, five variables
static __global__ void k_imex_op(int npoin_w, long long npoin, const int *__restrict__ lpoin_w, const float *__restrict__ Ml,
                          const float *__restrict__ v, float fact, float dt, float *__restrict__ qn) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const long long p = lpoin_w[t];
  const float ml = Ml[p];
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const long long o = p + npoin * k;
    qn[o] = __fadd_rn(__fmul_rn(v[o], ml), __fmul_rn(__fmul_rn(qn[o], fact), dt));
  }
}

// CG vector updates over the working nodes, five variables, M = Ml / dt:
//   mode 0: r = b - qn; z = r / M; p = z
//   mode 1: x += alpha p; r -= alpha qn; z1 = z; z = r / M
//   mode 2: p = z + beta p
static __global__ void k_imex_vec(int mode, int npoin_w, long long npoin, const int *__restrict__ lpoin_w,
                           const float *__restrict__ Ml, float dt, float alpha, float beta,
                           const float *__restrict__ b, float *__restrict__ x, float *__restrict__ r,
                           float *__restrict__ p, const float *__restrict__ qn, float *__restrict__ z,
                           float *__restrict__ z1) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const long long n = lpoin_w[t];
  const float M = __fdiv_rn(Ml[n], dt);
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const long long o = n + npoin * k;
    if (mode == 0) {
      const float rr = __fsub_rn(b[o], qn[o]);
      r[o] = rr;
      const float zz = __fdiv_rn(rr, M);
      z[o] = zz;
      p[o] = zz;
    } else if (mode == 1) {
      x[o] = __fadd_rn(x[o], __fmul_rn(alpha, p[o]));
      const float rr = __fsub_rn(r[o], __fmul_rn(alpha, qn[o]));
      r[o] = rr;
      z1[o] = z[o];
      z[o] = __fdiv_rn(rr, M);
    } else {
      p[o] = __fadd_rn(z[o], __fmul_rn(beta, p[o]));
    }
  }
}

// (rho, E, q) = x over the working nodes (mod_solver_imex.f90:331-338)
static __global__ void k_imex_out(int npoin_w, long long npoin, const int *__restrict__ lpoin_w, const float *__restrict__ x,
                           float *__restrict__ rho, float *__restrict__ E, float *__restrict__ q) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npoin_w) return;
  const long long p = lpoin_w[t];
  rho[p] = x[p];
  E[p] = x[p + npoin];
#pragma unroll
  for (int d = 0; d < 3; ++d) q[p + npoin * d] = x[p + npoin * (2 + d)];
}

}  // namespace sod
