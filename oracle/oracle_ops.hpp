// ORACLE -- test infrastructure only.  A CPU restatement of the SOD2D
// reference's arithmetic for the spectral-element RHS hot path, used by
// tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the
// arithmetic the CUDA results are compared with.  Never part of the
// product path.
//
// Every routine follows the loop structure and operation order of the
// Fortran routine it cites (paths relative to the reference project), in a
// generic precision R (float = the reference's USE_RP=4 build, double =
// USE_RP=8).  Arrays use the reference's Fortran layout (column-major,
// 1-based connectivity values).  Element results are computed in parallel
// into per-element buffers and scattered serially in element order, so the
// oracle is deterministic (the reference's atomics are not).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <initializer_list>
#include <vector>
#include <algorithm>
#include <limits>

namespace oracle {

struct Mesh {
  int porder = 0, np1 = 0, nnode = 0, nelem = 0, npoin = 0, npoin_w = 0;
  const int *connec = nullptr;   // connecWork(E,n)
  const int *lpoin_w = nullptr;  // (N_w)
  const int *invA = nullptr;     // invAtoIJK(P+1,P+1,P+1)
  const int *gI = nullptr, *gJ = nullptr, *gK = nullptr;  // gmshAtoI/J/K(n)
  const int *lelpn = nullptr;
  const int *atoIJK = nullptr;
};

template <class R>
struct Geo {
  const R *He = nullptr;       // He(3,3,n,E)
  const R *gpvol = nullptr;    // gpvol(1,n,E)
  const R *dl = nullptr;       // dlxigp_ip(n,3,P+1)
  const R *dNgp = nullptr;     // dNgp(3,n,n)
  const R *Ngp = nullptr;      // Ngp(n,n)
  const R *Ml = nullptr, *invMl = nullptr;
  const R *helem = nullptr;    // helem(E)
  const R *helem_l = nullptr;  // helem_l(E,n)
  R volT = 0;
};

// ---- index helpers ------------------------------------------------------
struct Idx {
  const Mesh &m;
  explicit Idx(const Mesh &mm) : m(mm) {}
  inline int node(long long e, int a) const { return m.connec[e + (long long)m.nelem * a] - 1; }
  inline int inv(int i, int j, int k) const { return m.invA[i + m.np1 * (j + m.np1 * k)] - 1; }
};
template <class R>
inline R HE(const Geo<R> &g, const Mesh &m, int i, int j, int gp, long long e) {
  return g.He[i + 3 * (j + 3 * (gp + (long long)m.nnode * e))];
}
template <class R>
inline R GV(const Geo<R> &g, const Mesh &m, int gp, long long e) {
  return g.gpvol[gp + (long long)m.nnode * e];
}
template <class R>
inline R DL(const Geo<R> &g, const Mesh &m, int gp, int d, int ii) {
  return g.dl[gp + m.nnode * (d + 3 * ii)];
}

// Serial scatter of per-element buffers buf[e][a][f] into nodal arrays.
template <class R>
void scatter(const Mesh &m, const std::vector<R> &buf, int nf, R *const *dst, R fact) {
  Idx ix(m);
  for (long long e = 0; e < m.nelem; ++e)
    for (int a = 0; a < m.nnode; ++a) {
      int p = ix.node(e, a);
      const R *b = &buf[((size_t)e * m.nnode + a) * nf];
      for (int f = 0; f < nf; ++f) dst[f][p] = dst[f][p] + fact * b[f];
    }
}

// ---- full_convec_ijk, src/lib_sod2d/sources/elem_convec.f90:227-470 ----
template <class R>
void full_convec_ijk(const Mesh &m, const Geo<R> &g, const R *u, const R *q, const R *rho,
                     const R *pr, const R *E, R *Rmass, R *Rmom, R *Rener, bool init, R fact) {
  const long long N = m.npoin;
  const int n = m.nnode, np1 = m.np1;
  if (init) {
    for (long long p = 0; p < N; ++p) { Rmass[p] = 0; Rener[p] = 0; Rmom[p] = 0; Rmom[p + N] = 0; Rmom[p + 2 * N] = 0; }
  }
  std::vector<R> buf((size_t)m.nelem * n * 5);
  Idx ix(m);
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < m.nelem; ++e) {
    std::vector<R> ul(n * 3), ql(n * 3), rhol(n), prl(n), El(n), REl(n), kl(n), Rkl(n);
    for (int a = 0; a < n; ++a) {
      int p = ix.node(e, a);
      kl[a] = 0;
      for (int d = 0; d < 3; ++d) kl[a] = kl[a] + u[p + N * d] * u[p + N * d] * R(0.5);
      rhol[a] = rho[p];
      El[a] = E[p];
      REl[a] = rho[p] * E[p];
      Rkl[a] = rho[p] * kl[a];
      prl[a] = pr[p];
      for (int d = 0; d < 3; ++d) { ul[a * 3 + d] = u[p + N * d]; ql[a * 3 + d] = q[p + N * d]; }
    }
    for (int gp = 0; gp < n; ++gp) {
      R dl[3][17];
      for (int ii = 0; ii < np1; ++ii)
        for (int d = 0; d < 3; ++d) dl[d][ii] = DL(g, m, gp, d, ii);
      int I = m.gI[gp] - 1, J = m.gJ[gp] - 1, K = m.gK[gp] - 1;
      R gRho[3] = {0, 0, 0}, gP[3] = {0, 0, 0}, gE[3] = {0, 0, 0}, gRE[3] = {0, 0, 0}, gk[3] = {0, 0, 0}, gRk[3] = {0, 0, 0};
      R gU[3][3] = {}, gQ[3][3] = {}, gFe[3][3] = {}, gFue[3][3] = {}, gFk[3][3] = {}, gFuk[3][3] = {};
      R gF[3][3][3] = {}, gFuu[3][3][3] = {};
      for (int ii = 0; ii < np1; ++ii) {
        int an[3] = {ix.inv(ii, J, K), ix.inv(I, ii, K), ix.inv(I, J, ii)};
        for (int d = 0; d < 3; ++d) {
          int a = an[d];
          R c = dl[d][ii];
          gRho[d] = gRho[d] + c * rhol[a];
          gP[d] = gP[d] + c * prl[a];
          gE[d] = gE[d] + c * (El[a]);
          gRE[d] = gRE[d] + c * (REl[a]);
          gk[d] = gk[d] + c * (kl[a]);
          gRk[d] = gRk[d] + c * (Rkl[a]);
        }
        for (int i = 0; i < 3; ++i) {
          for (int d = 0; d < 3; ++d) {
            int a = an[d];
            R c = dl[d][ii];
            gU[i][d] = gU[i][d] + c * ul[a * 3 + i];
            gQ[i][d] = gQ[i][d] + c * ql[a * 3 + i];
            gFe[i][d] = gFe[i][d] + c * rhol[a] * El[a] * ul[a * 3 + i];
            gFue[i][d] = gFue[i][d] + c * El[a] * ul[a * 3 + i];
            gFk[i][d] = gFk[i][d] + c * rhol[a] * kl[a] * ul[a * 3 + i];
            gFuk[i][d] = gFuk[i][d] + c * kl[a] * ul[a * 3 + i];
          }
          for (int j = 0; j < 3; ++j)
            for (int d = 0; d < 3; ++d) {
              int a = an[d];
              R c = dl[d][ii];
              gF[i][j][d] = gF[i][j][d] + c * ql[a * 3 + i] * ul[a * 3 + j];
              gFuu[i][j][d] = gFuu[i][j][d] + c * ul[a * 3 + i] * ul[a * 3 + j];
            }
        }
      }
      R gradRho[3] = {0, 0, 0}, gradP[3] = {0, 0, 0}, gradE[3] = {0, 0, 0}, gradRE[3] = {0, 0, 0}, gradk[3] = {0, 0, 0}, gradRk[3] = {0, 0, 0};
      R gradU[3][3] = {}, gradQ[3][3] = {}, divF[3] = {0, 0, 0}, divFuu[3] = {0, 0, 0};
      R divFe = 0, divFue = 0, divFk = 0, divFuk = 0;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          R h = HE(g, m, i, j, gp, e);
          gradRho[i] = gradRho[i] + h * gRho[j];
          gradP[i] = gradP[i] + h * gP[j];
          gradE[i] = gradE[i] + h * gE[j];
          gradRE[i] = gradRE[i] + h * gRE[j];
          divFe = divFe + h * gFe[i][j];
          divFue = divFue + h * gFue[i][j];
          gradk[i] = gradk[i] + h * gk[j];
          gradRk[i] = gradRk[i] + h * gRk[j];
          divFk = divFk + h * gFk[i][j];
          divFuk = divFuk + h * gFuk[i][j];
          for (int k = 0; k < 3; ++k) {
            R hjk = HE(g, m, j, k, gp, e);
            gradU[i][j] = gradU[i][j] + hjk * gU[i][k];
            gradQ[i][j] = gradQ[i][j] + hjk * gQ[i][k];
            divF[i] = divF[i] + hjk * gF[i][j][k];
            divFuu[i] = divFuu[i] + hjk * gFuu[i][j][k];
          }
        }
      R divU = gradU[0][0] + gradU[1][1] + gradU[2][2];
      R divQ = gradQ[0][0] + gradQ[1][1] + gradQ[2][2];
      R Re_mass = R(0.5) * (divQ + rhol[gp] * divU);
      R Re_ener = R(0.25) * (divFe + El[gp] * divQ + REl[gp] * divU + rhol[gp] * divFue) +
                  R(0.25) * (divFk + kl[gp] * divQ + Rkl[gp] * divU + rhol[gp] * divFuk);
      R Re_mom[3];
      R gv = GV(g, m, gp, e);
      for (int i = 0; i < 3; ++i) {
        Re_mom[i] = R(0.25) * (divF[i] + ul[gp * 3 + i] * divQ + ql[gp * 3 + i] * divU + rhol[gp] * divFuu[i]) + gradP[i];
        Re_mass = Re_mass + R(0.5) * (ul[gp * 3 + i] * gradRho[i]);
        Re_ener = Re_ener + R(0.25) * (ql[gp * 3 + i] * gradE[i] + ul[gp * 3 + i] * gradRE[i] + El[gp] * ul[gp * 3 + i] * gradRho[i]) +
                  R(0.25) * (ql[gp * 3 + i] * gradk[i] + ul[gp * 3 + i] * gradRk[i] + kl[gp] * ul[gp * 3 + i] * gradRho[i]);
        for (int j = 0; j < 3; ++j) {
          R aux = ul[gp * 3 + i] * ul[gp * 3 + j];
          Re_mom[i] = Re_mom[i] + R(0.25) * (aux * gradRho[j] + ql[gp * 3 + j] * gradU[i][j] + ul[gp * 3 + j] * gradQ[i][j]);
        }
        Re_mom[i] = gv * Re_mom[i];
      }
      Re_mass = gv * Re_mass;
      Re_ener = gv * Re_ener;
      R *b = &buf[((size_t)e * n + gp) * 5];
      b[0] = Re_mass; b[1] = Re_ener; b[2] = Re_mom[0]; b[3] = Re_mom[1]; b[4] = Re_mom[2];
    }
  }
  R *dst[5] = {Rmass, Rener, Rmom, Rmom + N, Rmom + 2 * N};
  scatter(m, buf, 5, dst, fact);
}

// ---- generic_scalar_convec_ijk, elem_convec.f90:472-594 ----------------
template <class R>
void generic_scalar_convec_ijk(const Mesh &m, const Geo<R> &g, const R *q, const R *eta, const R *u,
                               R *Rconvec, bool init, R fact) {
  const long long N = m.npoin;
  const int n = m.nnode, np1 = m.np1;
  if (init)
    for (long long p = 0; p < N; ++p) Rconvec[p] = 0;
  std::vector<R> buf((size_t)m.nelem * n);
  Idx ix(m);
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < m.nelem; ++e) {
    std::vector<R> ul(n * 3), fel(n * 3), etal(n);
    for (int a = 0; a < n; ++a) {
      int p = ix.node(e, a);
      for (int d = 0; d < 3; ++d) { ul[a * 3 + d] = u[p + N * d]; fel[a * 3 + d] = q[p + N * d]; }
      etal[a] = eta[p];
    }
    for (int gp = 0; gp < n; ++gp) {
      int I = m.gI[gp] - 1, J = m.gJ[gp] - 1, K = m.gK[gp] - 1;
      R gE[3] = {0, 0, 0}, gU[3][3] = {}, gFe[3][3] = {};
      for (int ii = 0; ii < np1; ++ii) {
        int an[3] = {ix.inv(ii, J, K), ix.inv(I, ii, K), ix.inv(I, J, ii)};
        for (int d = 0; d < 3; ++d) gE[d] = gE[d] + DL(g, m, gp, d, ii) * etal[an[d]];
        for (int i = 0; i < 3; ++i)
          for (int d = 0; d < 3; ++d) {
            gU[i][d] = gU[i][d] + DL(g, m, gp, d, ii) * ul[an[d] * 3 + i];
            gFe[i][d] = gFe[i][d] + DL(g, m, gp, d, ii) * fel[an[d] * 3 + i];
          }
      }
      R gradE[3] = {0, 0, 0}, divU = 0, divFe = 0;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          R h = HE(g, m, i, j, gp, e);
          gradE[i] = gradE[i] + h * gE[j];
          divU = divU + h * gU[i][j];
          divFe = divFe + h * gFe[i][j];
        }
      R Re = R(0.5) * (divFe + etal[gp] * divU);
      for (int i = 0; i < 3; ++i) Re = Re + R(0.5) * (ul[gp * 3 + i] * gradE[i]);
      buf[(size_t)e * n + gp] = GV(g, m, gp, e) * Re;
    }
  }
  R *dst[1] = {Rconvec};
  scatter(m, buf, 1, dst, fact);
}

// Gradients of rho, T, u at one Gauss point (shared by proj / diff_stab).
template <class R>
inline void grads_rTu(const Mesh &m, const Geo<R> &g, const Idx &ix, long long e, int gp,
                      const R *rhol, const R *Teml, const R *ul, R gradRho[3], R gradT[3], R gradU[3][3]) {
  int I = m.gI[gp] - 1, J = m.gJ[gp] - 1, K = m.gK[gp] - 1;
  R gR[3] = {0, 0, 0}, gT[3] = {0, 0, 0}, gU[3][3] = {};
  for (int ii = 0; ii < m.np1; ++ii) {
    int an[3] = {ix.inv(ii, J, K), ix.inv(I, ii, K), ix.inv(I, J, ii)};
    for (int d = 0; d < 3; ++d) gR[d] = gR[d] + DL(g, m, gp, d, ii) * rhol[an[d]];
    for (int d = 0; d < 3; ++d) gT[d] = gT[d] + DL(g, m, gp, d, ii) * Teml[an[d]];
    for (int i = 0; i < 3; ++i)
      for (int d = 0; d < 3; ++d) gU[i][d] = gU[i][d] + DL(g, m, gp, d, ii) * ul[an[d] * 3 + i];
  }
  for (int i = 0; i < 3; ++i) { gradRho[i] = 0; gradT[i] = 0; for (int j = 0; j < 3; ++j) gradU[i][j] = 0; }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      gradRho[i] = gradRho[i] + HE(g, m, i, j, gp, e) * gR[j];
      gradT[i] = gradT[i] + HE(g, m, i, j, gp, e) * gT[j];
      for (int k = 0; k < 3; ++k) gradU[i][j] = gradU[i][j] + HE(g, m, j, k, gp, e) * gU[i][k];
    }
}

// ---- lumped_solver_{scal,vect}_opt, mod_solver.f90:41-104 ---------------
template <class R>
void lumped_solver(const Mesh &m, const Geo<R> &g, R *Rv, int ncomp) {
  const long long N = m.npoin;
  for (int t = 0; t < m.npoin_w; ++t) {
    int p = m.lpoin_w[t] - 1;
    R aux1 = g.invMl[p];
    for (int c = 0; c < ncomp; ++c) Rv[p + N * c] = Rv[p + N * c] * aux1;
  }
}

// ---- halo sum of a partitioned mesh ------------------------------------
// The points where the reference calls mpi_halo_atomic_update_* on a rank
// of a partitioned mesh (elem_stab.f90:563-571 for the projections,
// time_integ_ls.f90:663-667 for the residuals), as a hook: the test that
// runs the oracle on sub-meshes installs a function that exchanges and adds
// the neighbours' contributions (mod_comms.f90:467-627); without one the
// mesh is whole and nothing happens.  comp[k] is component k, npoin values.
template <class R>
struct HaloHook {
  static inline void (*fn)(void *user, R *const *comp, int ncomp, long long npoin) = nullptr;
  static inline void *user = nullptr;
};
template <class R>
inline void halo_update(std::initializer_list<R *> comps, long long npoin) {
  if (!HaloHook<R>::fn) return;
  std::vector<R *> v(comps);
  HaloHook<R>::fn(HaloHook<R>::user, v.data(), (int)v.size(), npoin);
}

// The reference's MPI_Allreduce calls of the explicit step, as a hook of the
// same kind: vals reduced in place over the ranks, kind 0 min, 1 max,
// 2 sum.  Without one the mesh is whole and nothing happens.
struct ReduceHook {
  static inline void (*fn)(void *user, double *vals, int count, int kind) = nullptr;
  static inline void *user = nullptr;
};
inline void reduce_all(double *vals, int count, int kind) {
  if (ReduceHook::fn) ReduceHook::fn(ReduceHook::user, vals, count, kind);
}
template <class R>
inline R reduce_min(R v) {
  double d = (double)v;
  reduce_all(&d, 1, 0);
  return (R)d;
}

// ---- full_proj_ijk, src/lib_sod2d/sources/elem_stab.f90:441-586 --------
// Outputs, each (N,3): ProjMass, ProjEner, ProjMX, ProjMY, ProjMZ.
template <class R>
void full_proj_ijk(const Mesh &m, const Geo<R> &g, const R *rho, const R *u, const R *Tem,
                   R *PMass, R *PEner, R *PMX, R *PMY, R *PMZ) {
  const long long N = m.npoin;
  const int n = m.nnode;
  const R twoThirds = R(2.0) / R(3.0);
  for (long long p = 0; p < 3 * N; ++p) { PMass[p] = 0; PEner[p] = 0; PMX[p] = 0; PMY[p] = 0; PMZ[p] = 0; }
  std::vector<R> buf((size_t)m.nelem * n * 15);
  Idx ix(m);
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < m.nelem; ++e) {
    std::vector<R> ul(n * 3), rhol(n), Teml(n);
    for (int a = 0; a < n; ++a) {
      int p = ix.node(e, a);
      rhol[a] = rho[p];
      Teml[a] = Tem[p];
      for (int d = 0; d < 3; ++d) ul[a * 3 + d] = u[p + N * d];
    }
    for (int gp = 0; gp < n; ++gp) {
      R gradRho[3], gradT[3], gradU[3][3];
      grads_rTu(m, g, ix, e, gp, rhol.data(), Teml.data(), ul.data(), gradRho, gradT, gradU);
      R divU = gradU[0][0] + gradU[1][1] + gradU[2][2];
      R tau[3][3];
      for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) tau[i][j] = (gradU[i][j] + gradU[j][i]);
        tau[i][i] = tau[i][i] - twoThirds * divU;
      }
      R gv = GV(g, m, gp, e);
      R *b = &buf[((size_t)e * n + gp) * 15];
      for (int d = 0; d < 3; ++d) {
        b[0 + d] = gv * tau[0][d];   // ProjMX
        b[3 + d] = gv * tau[1][d];   // ProjMY
        b[6 + d] = gv * tau[2][d];   // ProjMZ
        b[9 + d] = gv * gradRho[d];  // ProjMass
        b[12 + d] = gv * gradT[d];   // ProjEner
      }
    }
  }
  R *dst[15] = {PMX, PMX + N, PMX + 2 * N, PMY, PMY + N, PMY + 2 * N, PMZ, PMZ + N, PMZ + 2 * N,
                PMass, PMass + N, PMass + 2 * N, PEner, PEner + N, PEner + 2 * N};
  scatter(m, buf, 15, dst, R(1));
  halo_update<R>({PMX, PMX + N, PMX + 2 * N}, N);
  halo_update<R>({PMY, PMY + N, PMY + 2 * N}, N);
  halo_update<R>({PMZ, PMZ + N, PMZ + 2 * N}, N);
  halo_update<R>({PMass, PMass + N, PMass + 2 * N}, N);
  halo_update<R>({PEner, PEner + N, PEner + 2 * N}, N);
  lumped_solver(m, g, PMX, 3);
  lumped_solver(m, g, PMY, 3);
  lumped_solver(m, g, PMZ, 3);
  lumped_solver(m, g, PMass, 3);
  lumped_solver(m, g, PEner, 3);
}

// Weak-form divergence sum_d sum_ii He(:,d,gp')*gpvol(gp')*dl(gp',d,iso_d)*F(gp',:)
// at output node gp, as the second Gauss-point loop of full_diff_stab_ijk.
template <class R>
inline R weak_div(const Mesh &m, const Geo<R> &g, const Idx &ix, long long e, int gp, const R *F /*[n][3]*/) {
  int I = m.gI[gp] - 1, J = m.gJ[gp] - 1, K = m.gK[gp] - 1;
  R s = 0;
  for (int ii = 0; ii < m.np1; ++ii) {
    int a1 = ix.inv(ii, J, K), a2 = ix.inv(I, ii, K), a3 = ix.inv(I, J, ii);
    for (int i = 0; i < 3; ++i) {
      s = s + HE(g, m, i, 0, a1, e) * GV(g, m, a1, e) * DL(g, m, a1, 0, I) * F[a1 * 3 + i];
      s = s + HE(g, m, i, 1, a2, e) * GV(g, m, a2, e) * DL(g, m, a2, 1, J) * F[a2 * 3 + i];
      s = s + HE(g, m, i, 2, a3, e) * GV(g, m, a3, e) * DL(g, m, a3, 2, K) * F[a3 * 3 + i];
    }
  }
  return s;
}

// ---- full_diff_stab_ijk, src/lib_sod2d/sources/elem_stab.f90:207-438 ---
// c_lps is c_lps_comp (0.1, CFDSolverBase.f90:768), c_rho = c_ener = 1.
template <class R>
void full_diff_stab_ijk(const Mesh &m, const Geo<R> &g, R Cp, R Pr, const R *rho_n, const R *rho,
                        const R *u, const R *Tem, const R *mu_fluid, const R *mu_e, const R *mu_sgs,
                        const R *PMass, const R *PEner, const R *PMX, const R *PMY, const R *PMZ,
                        const R *tau_stab, R *Rmass, R *Rmom, R *Rener, bool init, R fact,
                        R c_lps = R(0.1f), R c_rho = R(1), R c_ener = R(1)) {
  const long long N = m.npoin;
  const int n = m.nnode;
  const R twoThirds = R(2.0) / R(3.0);
  if (init)
    for (long long p = 0; p < N; ++p) { Rmass[p] = 0; Rener[p] = 0; Rmom[p] = 0; Rmom[p + N] = 0; Rmom[p + 2 * N] = 0; }
  std::vector<R> buf((size_t)m.nelem * n * 5);
  Idx ix(m);
  const long long NE = m.nelem;
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < m.nelem; ++e) {
    std::vector<R> ul(n * 3), rhol(n), rhonl(n), Teml(n), mufl(n);
    std::vector<R> pMass(n * 3), pEner(n * 3), pMX(n * 3), pMY(n * 3), pMZ(n * 3);
    std::vector<R> tauX(n * 3, 0), tauY(n * 3, 0), tauZ(n * 3, 0), gTl(n * 3, 0), gRl(n * 3, 0);
    for (int a = 0; a < n; ++a) {
      int p = ix.node(e, a);
      rhol[a] = rho[p]; rhonl[a] = rho_n[p]; Teml[a] = Tem[p]; mufl[a] = mu_fluid[p];
      for (int d = 0; d < 3; ++d) {
        ul[a * 3 + d] = u[p + N * d];
        pMass[a * 3 + d] = PMass[p + N * d]; pEner[a * 3 + d] = PEner[p + N * d];
        pMX[a * 3 + d] = PMX[p + N * d]; pMY[a * 3 + d] = PMY[p + N * d]; pMZ[a * 3 + d] = PMZ[p + N * d];
      }
    }
    R taustabl = tau_stab[e];
    for (int gp = 0; gp < n; ++gp) {
      R mue = mu_e[e + NE * gp], musgs = mu_sgs[e + NE * gp];
      R nu_e = c_rho * mue / rhonl[gp];
      R mu_fgp = mufl[gp] + rhonl[gp] * musgs;
      R mu_egp = mue;
      R kappa_e = mufl[gp] * Cp / Pr + c_ener * mue * Cp / Pr + Cp * rhonl[gp] * musgs / R(0.9);
      R gradRho[3], gradT[3], gradU[3][3];
      grads_rTu(m, g, ix, e, gp, rhol.data(), Teml.data(), ul.data(), gradRho, gradT, gradU);
      R divU = gradU[0][0] + gradU[1][1] + gradU[2][2];
      R tau[3][3];
      for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) tau[i][j] = (gradU[i][j] + gradU[j][i]);
        tau[i][i] = tau[i][i] - twoThirds * divU;
      }
      for (int d = 0; d < 3; ++d) {
        tauX[gp * 3 + d] = -c_lps * taustabl * (pMX[gp * 3 + d] - tau[0][d]) * rhonl[gp];
        tauY[gp * 3 + d] = -c_lps * taustabl * (pMY[gp * 3 + d] - tau[1][d]) * rhonl[gp];
        tauZ[gp * 3 + d] = -c_lps * taustabl * (pMZ[gp * 3 + d] - tau[2][d]) * rhonl[gp];
        gTl[gp * 3 + d] = -c_lps * taustabl * (pEner[gp * 3 + d] - gradT[d]) * rhonl[gp] * Cp / Pr;
        gRl[gp * 3 + d] = -c_lps * taustabl * (pMass[gp * 3 + d] - gradRho[d]);
      }
      R tauU[3] = {0, 0, 0};
      for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) {
          tauU[i] = tauU[i] + (mu_fgp + mu_egp) * (gradU[i][j] + gradU[j][i]) * ul[gp * 3 + j];
          tau[i][j] = (mu_fgp + mu_egp) * (gradU[i][j] + gradU[j][i]);
        }
        tauU[i] = tauU[i] - (mu_fgp)*twoThirds * divU * ul[gp * 3 + i];
        tau[i][i] = tau[i][i] - (mu_fgp)*twoThirds * divU;
      }
      for (int d = 0; d < 3; ++d) {
        tauX[gp * 3 + d] = tauX[gp * 3 + d] + tau[0][d];
        tauY[gp * 3 + d] = tauY[gp * 3 + d] + tau[1][d];
        tauZ[gp * 3 + d] = tauZ[gp * 3 + d] + tau[2][d];
        gTl[gp * 3 + d] = gTl[gp * 3 + d] + kappa_e * gradT[d] + tauU[d];
        gRl[gp * 3 + d] = gRl[gp * 3 + d] + nu_e * gradRho[d];
      }
    }
    for (int gp = 0; gp < n; ++gp) {
      R *b = &buf[((size_t)e * n + gp) * 5];
      b[0] = weak_div(m, g, ix, e, gp, gRl.data());
      b[1] = weak_div(m, g, ix, e, gp, gTl.data());
      b[2] = weak_div(m, g, ix, e, gp, tauX.data());
      b[3] = weak_div(m, g, ix, e, gp, tauY.data());
      b[4] = weak_div(m, g, ix, e, gp, tauZ.data());
    }
  }
  R *dst[5] = {Rmass, Rener, Rmom, Rmom + N, Rmom + 2 * N};
  scatter(m, buf, 5, dst, fact);
}

// ---- full_diffusion_ijk, src/lib_sod2d/sources/elem_diffu.f90:12-223 ----
template <class R>
void full_diffusion_ijk(const Mesh &m, const Geo<R> &g, R Cp, R Pr, const R *rho_n, const R *rho,
                        const R *u, const R *Tem, const R *mu_fluid, const R *mu_e, const R *mu_sgs,
                        R *Rmass, R *Rmom, R *Rener, bool init, R fact, R c_rho = R(1), R c_ener = R(1)) {
  const long long N = m.npoin;
  const int n = m.nnode;
  const R twoThirds = R(2.0) / R(3.0);
  if (init)
    for (long long p = 0; p < N; ++p) { Rmass[p] = 0; Rener[p] = 0; Rmom[p] = 0; Rmom[p + N] = 0; Rmom[p + 2 * N] = 0; }
  std::vector<R> buf((size_t)m.nelem * n * 5);
  Idx ix(m);
  const long long NE = m.nelem;
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < m.nelem; ++e) {
    std::vector<R> ul(n * 3), rhol(n), rhonl(n), Teml(n), mufl(n);
    std::vector<R> tauX(n * 3, 0), tauY(n * 3, 0), tauZ(n * 3, 0), gTl(n * 3, 0), gRl(n * 3, 0), tUl(n * 3, 0);
    for (int a = 0; a < n; ++a) {
      int p = ix.node(e, a);
      rhol[a] = rho[p]; rhonl[a] = rho_n[p]; Teml[a] = Tem[p]; mufl[a] = mu_fluid[p];
      for (int d = 0; d < 3; ++d) ul[a * 3 + d] = u[p + N * d];
    }
    for (int gp = 0; gp < n; ++gp) {
      R mu_fgp = mufl[gp] + rhonl[gp] * mu_sgs[e + NE * gp];
      R mu_egp = mu_e[e + NE * gp];
      R gradRho[3], gradT[3], gradU[3][3];
      grads_rTu(m, g, ix, e, gp, rhol.data(), Teml.data(), ul.data(), gradRho, gradT, gradU);
      R divU = gradU[0][0] + gradU[1][1] + gradU[2][2];
      R tau[3][3], tauU[3] = {0, 0, 0};
      for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) {
          tauU[i] = tauU[i] + (mu_fgp + mu_egp) * (gradU[i][j] + gradU[j][i]) * ul[gp * 3 + j];
          tau[i][j] = (mu_fgp + mu_egp) * (gradU[i][j] + gradU[j][i]);
        }
        tauU[i] = tauU[i] - (mu_fgp)*twoThirds * divU * ul[gp * 3 + i];
        tau[i][i] = tau[i][i] - (mu_fgp)*twoThirds * divU;
      }
      for (int d = 0; d < 3; ++d) {
        tauX[gp * 3 + d] = tau[0][d]; tauY[gp * 3 + d] = tau[1][d]; tauZ[gp * 3 + d] = tau[2][d];
        gTl[gp * 3 + d] = gradT[d]; gRl[gp * 3 + d] = gradRho[d]; tUl[gp * 3 + d] = tauU[d];
      }
    }
    for (int gp = 0; gp < n; ++gp) {
      R mue = mu_e[e + NE * gp], musgs = mu_sgs[e + NE * gp];
      R nu_e = c_rho * mue / rhonl[gp];
      R kappa_e = mufl[gp] * Cp / Pr + c_ener * mue * Cp / Pr + Cp * rhonl[gp] * musgs / R(0.9);
      std::vector<R> fe(n * 3);
      for (int a = 0; a < n; ++a)
        for (int d = 0; d < 3; ++d) fe[a * 3 + d] = (tUl[a * 3 + d] + kappa_e * gTl[a * 3 + d]);
      R *b = &buf[((size_t)e * n + gp) * 5];
      b[0] = nu_e * weak_div(m, g, ix, e, gp, gRl.data());
      b[1] = weak_div(m, g, ix, e, gp, fe.data());
      b[2] = weak_div(m, g, ix, e, gp, tauX.data());
      b[3] = weak_div(m, g, ix, e, gp, tauY.data());
      b[4] = weak_div(m, g, ix, e, gp, tauZ.data());
    }
  }
  R *dst[5] = {Rmass, Rener, Rmom, Rmom + N, Rmom + 2 * N};
  scatter(m, buf, 5, dst, fact);
}

// ---- comp_tau, src/lib_sod2d/sources/elem_stab.f90:589-616 -------------
template <class R>
void comp_tau(const Mesh &m, const Geo<R> &g, const R *csound, const R *u, R *tau, R c_species_stab = R(0.5)) {
  const long long N = m.npoin, NE = m.nelem;
  Idx ix(m);
  for (long long e = 0; e < NE; ++e) {
    R taul = 0;
    for (int a = 0; a < m.nnode; ++a) {
      int p = ix.node(e, a);
      R uu = u[p] * u[p] + u[p + N] * u[p + N] + u[p + 2 * N] * u[p + 2 * N];
      R aux1 = R(1) * csound[p] + std::sqrt(uu);
      taul = std::max(taul, (g.helem[e]) * (c_species_stab / R(m.porder)) * aux1);
    }
    tau[e] = taul;
  }
}

// ---- sutherland_viscosity, mod_fluid_viscosity.f90:21-41 ---------------
template <class R>
void sutherland(long long npoin, const R *Tem, const R *mu_factor, R *mu_fluid) {
  const R C1 = R(0.000001458), S = R(110.4);
  for (long long p = 0; p < npoin; ++p)
    mu_fluid[p] = mu_factor[p] * C1 * std::pow(Tem[p], R(1.5)) / (Tem[p] + S);
}

// ---- thermo_entropy, mod_entropy_viscosity.f90:411-433 -----------------
// eta is the reference's eta(N,4) array (levels 1 and 2 are touched).
template <class R>
void thermo_entropy(const Mesh &m, R gamma, R p_inf, R rho_inf, const R *rho, const R *pr, const R *u1,
                    R *eta, R *feta) {
  const long long N = m.npoin;
  for (int t = 0; t < m.npoin_w; ++t) {
    long long p = m.lpoin_w[t] - 1;
    eta[p] = eta[p + N];
    eta[p + N] = (rho[p] / (gamma - R(1))) *
                 std::log(std::max(pr[p] / p_inf, std::numeric_limits<R>::epsilon()) / std::pow(rho[p] / rho_inf, gamma));
    for (int d = 0; d < 3; ++d) feta[p + N * d] = u1[p + N * d] * eta[p];
  }
}

// ---- smart_visc_spectral_imex, mod_entropy_viscosity.f90:113-227 -------
// High-Mach path (flag_high_mach, TGVCompSolver.f90:128): norm = min rho over
// working nodes and ce = ce_comp.
template <class R>
void smart_visc_spectral_imex(const Mesh &m, const Geo<R> &g, const R *Reta, const R *rho, const R *u,
                              const R *csound, R *mu_e, R ce = R(1), R cmax = R(0.5), R cglob = R(1)) {
  const long long N = m.npoin, NE = m.nelem;
  R maxRl = R(100000.0);
  for (int t = 0; t < m.npoin_w; ++t) maxRl = std::min(maxRl, rho[m.lpoin_w[t] - 1]);
  R norm = reduce_min(maxRl);  // MPI_Allreduce MIN, mod_entropy_viscosity.f90:161
  Idx ix(m);
  for (long long e = 0; e < NE; ++e) {
    R betae = 0;
    for (int a = 0; a < m.nnode; ++a) {
      int p = ix.node(e, a);
      R aux2 = std::sqrt(u[p] * u[p] + u[p + N] * u[p + N] + u[p + 2 * N] * u[p + 2 * N]);
      R aux3 = R(1) * csound[p];
      R aux1 = aux2 + aux3;
      betae = std::max(betae, (rho[p] * g.helem[e]) * (cmax / R(m.porder)) * aux1);
    }
    for (int a = 0; a < m.nnode; ++a) {
      int p = ix.node(e, a);
      R R1 = rho[p] * std::fabs(Reta[p]) / norm;
      R hp = g.helem[e] / R(m.porder);
      R Ve = ce * R1 * (hp * hp);
      mu_e[e + NE * a] = cglob * std::min(Ve, betae);
    }
  }
}

// ---- ducros_visc_limit, mod_entropy_viscosity.f90:277-314 --------------
template <class R>
void ducros_visc_limit(const Mesh &m, const Geo<R> &g, const R *rho, const R *u, const R *divU,
                       const R *vorti, const R *csound, R *mu_e, R cmax = R(0.5), R ducros_min_val = R(0.1)) {
  const long long N = m.npoin, NE = m.nelem;
  const R eps = std::numeric_limits<R>::epsilon();
  Idx ix(m);
  for (long long e = 0; e < NE; ++e)
    for (int a = 0; a < m.nnode; ++a) {
      int p = ix.node(e, a);
      R divUl = divU[p] / g.Ml[p];
      R aux2 = std::sqrt(u[p] * u[p] + u[p + N] * u[p + N] + u[p + 2 * N] * u[p + 2 * N]);
      R vv = vorti[p] * vorti[p] + vorti[p + N] * vorti[p + N] + vorti[p + 2 * N] * vorti[p + 2 * N];
      R d2 = divUl * divUl;
      R phi = std::min((R(4.0) / R(3.0)) * d2 / (d2 + vv + eps), R(1));
      R hl = R(1) * aux2 / g.helem_l[e + NE * a];
      R phi2 = d2 / (d2 + hl * hl + eps);
      mu_e[e + NE * a] = mu_e[e + NE * a] * (std::max(phi - ducros_min_val, R(0)) * phi2 + ducros_min_val);
    }
}

// ---- eval_divergence, src/lib_sod2d_incomp/sources/mod_operators.f90:485-570
template <class R>
void eval_divergence(const Mesh &m, const Geo<R> &g, const R *u, R *Rdiv) {
  const long long N = m.npoin;
  const int n = m.nnode;
  for (long long p = 0; p < N; ++p) Rdiv[p] = 0;
  std::vector<R> buf((size_t)m.nelem * n);
  Idx ix(m);
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < m.nelem; ++e) {
    std::vector<R> ul(n * 3);
    for (int a = 0; a < n; ++a) {
      int p = ix.node(e, a);
      for (int d = 0; d < 3; ++d) ul[a * 3 + d] = u[p + N * d];
    }
    for (int gp = 0; gp < n; ++gp) {
      int I = m.gI[gp] - 1, J = m.gJ[gp] - 1, K = m.gK[gp] - 1;
      R gU[3][3] = {};
      for (int ii = 0; ii < m.np1; ++ii) {
        int an[3] = {ix.inv(ii, J, K), ix.inv(I, ii, K), ix.inv(I, J, ii)};
        for (int i = 0; i < 3; ++i)
          for (int d = 0; d < 3; ++d) gU[i][d] = gU[i][d] + DL(g, m, gp, d, ii) * ul[an[d] * 3 + i];
      }
      R divU = 0;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) divU = divU + HE(g, m, i, j, gp, e) * gU[i][j];
      buf[(size_t)e * n + gp] = GV(g, m, gp, e) * divU;
    }
  }
  R *dst[1] = {Rdiv};
  scatter(m, buf, 1, dst, R(1));
  halo_update<R>({Rdiv}, N);  // mod_operators.f90:566
}

// ---- compute_vorticity, mod_operators.f90:684-775 (makeConti = true) ---
// leviCivi as set at CFDSolverBase.f90:1600-1606.
template <class R>
void compute_vorticity(const Mesh &m, const Geo<R> &g, const R *u, R *curlU) {
  const long long N = m.npoin;
  const int n = m.nnode;
  for (long long p = 0; p < 3 * N; ++p) curlU[p] = 0;
  R lc[3][3][3] = {};
  lc[1][2][0] = 1; lc[2][1][0] = -1; lc[0][2][1] = -1; lc[2][0][1] = 1; lc[0][1][2] = 1; lc[1][0][2] = -1;
  std::vector<R> buf((size_t)m.nelem * n * 27);
  Idx ix(m);
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < m.nelem; ++e) {
    std::vector<R> ul(n * 3);
    for (int a = 0; a < n; ++a) {
      int p = ix.node(e, a);
      for (int d = 0; d < 3; ++d) ul[a * 3 + d] = u[p + N * d];
    }
    for (int gp = 0; gp < n; ++gp) {
      int I = m.gI[gp] - 1, J = m.gJ[gp] - 1, K = m.gK[gp] - 1;
      R gU[3][3] = {};
      for (int ii = 0; ii < m.np1; ++ii) {
        int an[3] = {ix.inv(ii, J, K), ix.inv(I, ii, K), ix.inv(I, J, ii)};
        for (int i = 0; i < 3; ++i)
          for (int d = 0; d < 3; ++d) gU[i][d] = gU[i][d] + DL(g, m, gp, d, ii) * ul[an[d] * 3 + i];
      }
      R gu[3][3] = {};
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          for (int k = 0; k < 3; ++k) gu[i][j] = gu[i][j] + HE(g, m, j, k, gp, e) * gU[i][k];
      R *b = &buf[((size_t)e * n + gp) * 27];
      int t = 0;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          for (int k = 0; k < 3; ++k) b[t++] = lc[i][j][k] * gu[j][k];
    }
  }
  // 27 sequential atomic-style adds per Gauss point, in (i,j,k) order.
  for (long long e = 0; e < m.nelem; ++e)
    for (int gp = 0; gp < n; ++gp) {
      int p = ix.node(e, gp);
      const R *b = &buf[((size_t)e * n + gp) * 27];
      int t = 0;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          for (int k = 0; k < 3; ++k) curlU[p + N * i] = curlU[p + N * i] + b[t++];
    }
  halo_update<R>({curlU, curlU + N, curlU + 2 * N}, N);  // mod_operators.f90:759
  for (int t = 0; t < m.npoin_w; ++t) {
    int p = m.lpoin_w[t] - 1;
    for (int d = 0; d < 3; ++d) curlU[p + N * d] = curlU[p + N * d] / R(m.lelpn[p]);
  }
}

// ---- adapt_dt_cfl, src/lib_sod2d/sources/mod_time_ops.f90:11-62 --------
template <class R>
R adapt_dt_cfl(const Mesh &m, const Geo<R> &g, const R *u, const R *csound, R cfl_conv, R cfl_diff,
               const R *mu_fluid, const R *mu_sgs, const R *mu_e, const R *rho) {
  const long long N = m.npoin, NE = m.nelem;
  R dt_conv = R(100000000000000.0), dt_diff = R(100000000000000.0), dt_l = R(100000000000000.0);
  Idx ix(m);
  for (long long e = 0; e < NE; ++e) {
    R L3 = 0;
    for (int a = 0; a < m.nnode; ++a) {
      int p = ix.node(e, a);
      R umag = std::fabs(u[p]);
      umag = std::max(umag, std::fabs(u[p + N]));
      umag = std::max(umag, std::fabs(u[p + 2 * N]));
      R aux1 = umag + csound[p];
      L3 = std::max(L3, aux1);
    }
    R hp = g.helem[e] / R(R(2.0) * m.porder + 1);
    R aux2 = cfl_conv * hp / L3;
    dt_conv = std::min(dt_conv, aux2);
    R max_MU = 0;
    for (int a = 0; a < m.nnode; ++a) {
      int p = ix.node(e, a);
      max_MU = std::max(max_MU, (mu_sgs[e + NE * a] + mu_fluid[p] + mu_e[e + NE * a]) / rho[p]);
    }
    R aux4 = cfl_diff * (hp * hp) / max_MU;
    dt_diff = std::min(dt_diff, aux4);
    dt_l = std::min(dt_conv, dt_diff);
  }
  return reduce_min(dt_l);  // MPI_Allreduce MIN, mod_time_ops.f90:59
}

// ---- volAvg_EK, src/lib_sod2d/sources/mod_analysis.f90:10-44 -----------
template <class R>
double volAvg_EK(const Mesh &m, const Geo<R> &g, R rho0, const R *rho, const R *u) {
  const long long N = m.npoin;
  const int n = m.nnode;
  Idx ix(m);
  double EK = 0.0;
  for (long long e = 0; e < m.nelem; ++e) {
    R R1 = 0;
    for (int gp = 0; gp < n; ++gp)
      for (int a = 0; a < n; ++a) {
        int p = ix.node(e, a);
        R uu = u[p] * u[p] + u[p + N] * u[p + N] + u[p + 2 * N] * u[p + 2 * N];
        R1 = R1 + GV(g, m, gp, e) * g.Ngp[gp + n * a] * R(0.5) * rho[p] * uu;
      }
    EK += (double)R1;
  }
  reduce_all(&EK, 1, 2);  // MPI_Allreduce SUM, mod_analysis.f90:39
  R twopi = R(2.0) * R(3.14159f);
  EK = EK / (double)(rho0 * std::pow(twopi, R(3.0)));
  return EK;
}

// ---- visc_dissipationRate, mod_analysis.f90:46-144 ---------------------
template <class R>
void visc_dissipationRate(const Mesh &m, const Geo<R> &g, R rho0, const R *mu_fluid, const R *mu_e,
                          const R *u, R volT, double *eps_S, double *eps_D, double *eps_T) {
  const long long N = m.npoin, NE = m.nelem;
  const int n = m.nnode;
  R lc[3][3][3] = {};
  lc[1][2][0] = 1; lc[2][1][0] = -1; lc[0][2][1] = -1; lc[2][0][1] = 1; lc[0][1][2] = 1; lc[1][0][2] = -1;
  Idx ix(m);
  std::vector<double> s1(NE), s2(NE);
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < NE; ++e) {
    R R1 = 0, R2 = 0;
    std::vector<R> gpcar(3 * n);
    for (int gp = 0; gp < n; ++gp) {
      for (int i = 0; i < 3; ++i)
        for (int a = 0; a < n; ++a) {
          R s = 0;
          for (int j = 0; j < 3; ++j) s = s + HE(g, m, i, j, gp, e) * g.dNgp[j + 3 * (a + n * gp)];
          gpcar[i + 3 * a] = s;
        }
      R gradU[3][3];
      for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 3; ++k) {
          R aux = 0;
          for (int a = 0; a < n; ++a) aux = aux + gpcar[j + 3 * a] * u[ix.node(e, a) + N * k];
          gradU[j][k] = aux;
        }
      R div2U = gradU[0][0] + gradU[1][1] + gradU[2][2];
      div2U = div2U * div2U;
      R curl2U = 0;
      for (int i = 0; i < 3; ++i) {
        R aux2 = 0;
        for (int j = 0; j < 3; ++j)
          for (int k = 0; k < 3; ++k) aux2 = aux2 + (lc[i][j][k] * gradU[j][k]);
        curl2U = curl2U + aux2 * aux2;
      }
      int pg = ix.node(e, gp);
      R1 = R1 + GV(g, m, gp, e) * (mu_fluid[pg] + mu_e[e + NE * gp]) * curl2U;
      R2 = R2 + GV(g, m, gp, e) * mu_fluid[pg] * div2U;
    }
    s1[e] = (double)R1;
    s2[e] = (double)R2;
  }
  double S = 0, D = 0;
  for (long long e = 0; e < NE; ++e) { S += s1[e]; D += s2[e]; }
  double SD[2] = {S, D};
  reduce_all(SD, 2, 2);  // MPI_Allreduce SUM, mod_analysis.f90:134-135
  S = SD[0];
  D = SD[1];
  R alpha = R(1.0) / (rho0 * volT);
  S = S * (double)alpha;
  D = (double)(4.0f / 3.0f) * D * (double)alpha;  // default-real literal 4.0/3.0
  *eps_T = (double)(R)(S + D);
  *eps_S = (double)(R)S;
  *eps_D = (double)(R)D;
}


// ---- eval_laplacian_mult, src/lib_sod2d_incomp/sources/mod_operators.f90:16-112
// ResP = sum_e int grad N . grad p (no fixed-pressure node: periodic TGV).
template <class R>
void eval_laplacian_mult(const Mesh &m, const Geo<R> &g, const R *p, R *ResP) {
  const long long N = m.npoin;
  const int n = m.nnode;
  for (long long i = 0; i < N; ++i) ResP[i] = 0;
  std::vector<R> buf((size_t)m.nelem * n);
  Idx ix(m);
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < m.nelem; ++e) {
    std::vector<R> pl(n), gP(n * 3);
    for (int a = 0; a < n; ++a) pl[a] = p[ix.node(e, a)];
    for (int gp = 0; gp < n; ++gp) {
      int I = m.gI[gp] - 1, J = m.gJ[gp] - 1, K = m.gK[gp] - 1;
      R gi[3] = {0, 0, 0};
      for (int ii = 0; ii < m.np1; ++ii) {
        gi[0] = gi[0] + DL(g, m, gp, 0, ii) * pl[ix.inv(ii, J, K)];
        gi[1] = gi[1] + DL(g, m, gp, 1, ii) * pl[ix.inv(I, ii, K)];
        gi[2] = gi[2] + DL(g, m, gp, 2, ii) * pl[ix.inv(I, J, ii)];
      }
      for (int i = 0; i < 3; ++i) {
        R s = 0;
        for (int j = 0; j < 3; ++j) s = s + HE(g, m, i, j, gp, e) * gi[j];
        gP[gp * 3 + i] = s;
      }
    }
    for (int gp = 0; gp < n; ++gp) buf[(size_t)e * n + gp] = weak_div(m, g, ix, e, gp, gP.data());
  }
  R *dst[1] = {ResP};
  scatter(m, buf, 1, dst, R(1));
}

// ---- eval_laplacian_diag, mod_operators.f90:638-682 ----------------------
template <class R>
void eval_laplacian_diag(const Mesh &m, const Geo<R> &g, R *d) {
  const long long N = m.npoin;
  const int n = m.nnode;
  for (long long i = 0; i < N; ++i) d[i] = 0;
  Idx ix(m);
  std::vector<R> gpcar(3 * n);
  for (long long e = 0; e < m.nelem; ++e)
    for (int gp = 0; gp < n; ++gp) {
      for (int i = 0; i < 3; ++i)
        for (int a = 0; a < n; ++a) {
          R s = 0;
          for (int j = 0; j < 3; ++j) s = s + HE(g, m, i, j, gp, e) * g.dNgp[j + 3 * (a + n * gp)];
          gpcar[i + 3 * a] = s;
        }
      for (int i = 0; i < 3; ++i)
        for (int a = 0; a < n; ++a) {
          int p = ix.node(e, a);
          d[p] = d[p] + GV(g, m, gp, e) * gpcar[i + 3 * a] * gpcar[i + 3 * a];
        }
    }
}

// ---- eval_gradient (lumped), mod_operators.f90:212-288 --------------------
template <class R>
void eval_gradient(const Mesh &m, const Geo<R> &g, const R *x, R *gradX) {
  const long long N = m.npoin;
  const int n = m.nnode;
  for (long long i = 0; i < 3 * N; ++i) gradX[i] = 0;
  std::vector<R> buf((size_t)m.nelem * n * 3);
  Idx ix(m);
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < m.nelem; ++e) {
    std::vector<R> pl(n);
    for (int a = 0; a < n; ++a) pl[a] = x[ix.node(e, a)];
    for (int gp = 0; gp < n; ++gp) {
      int I = m.gI[gp] - 1, J = m.gJ[gp] - 1, K = m.gK[gp] - 1;
      R gi[3] = {0, 0, 0};
      for (int ii = 0; ii < m.np1; ++ii) {
        gi[0] = gi[0] + DL(g, m, gp, 0, ii) * pl[ix.inv(ii, J, K)];
        gi[1] = gi[1] + DL(g, m, gp, 1, ii) * pl[ix.inv(I, ii, K)];
        gi[2] = gi[2] + DL(g, m, gp, 2, ii) * pl[ix.inv(I, J, ii)];
      }
      for (int i = 0; i < 3; ++i) {
        R s = 0;
        for (int j = 0; j < 3; ++j) s = s + HE(g, m, i, j, gp, e) * gi[j];
        buf[((size_t)e * n + gp) * 3 + i] = GV(g, m, gp, e) * s;
      }
    }
  }
  R *dst[3] = {gradX, gradX + N, gradX + 2 * N};
  scatter(m, buf, 3, dst, R(1));
  lumped_solver(m, g, gradX, 3);
}

// ---- full_convec_ijk_incomp, src/lib_sod2d_incomp/sources/elem_convec_incomp.f90:19-125
template <class R>
void full_convec_ijk_incomp(const Mesh &m, const Geo<R> &g, const R *u, const R *q, R *Rmom) {
  const long long N = m.npoin;
  const int n = m.nnode;
  for (long long i = 0; i < 3 * N; ++i) Rmom[i] = 0;
  std::vector<R> buf((size_t)m.nelem * n * 3);
  Idx ix(m);
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < m.nelem; ++e) {
    std::vector<R> ul(n * 3), ql(n * 3);
    for (int a = 0; a < n; ++a) {
      int p = ix.node(e, a);
      for (int d = 0; d < 3; ++d) { ul[a * 3 + d] = u[p + N * d]; ql[a * 3 + d] = q[p + N * d]; }
    }
    for (int gp = 0; gp < n; ++gp) {
      int I = m.gI[gp] - 1, J = m.gJ[gp] - 1, K = m.gK[gp] - 1;
      R gQ[3][3] = {}, gF[3][3][3] = {};
      for (int ii = 0; ii < m.np1; ++ii) {
        int an[3] = {ix.inv(ii, J, K), ix.inv(I, ii, K), ix.inv(I, J, ii)};
        for (int i = 0; i < 3; ++i) {
          for (int d = 0; d < 3; ++d) gQ[i][d] = gQ[i][d] + DL(g, m, gp, d, ii) * ql[an[d] * 3 + i];
          for (int j = 0; j < 3; ++j)
            for (int d = 0; d < 3; ++d)
              gF[i][j][d] = gF[i][j][d] + DL(g, m, gp, d, ii) * ql[an[d] * 3 + i] * ul[an[d] * 3 + j];
        }
      }
      R gradQ[3][3] = {}, divF[3] = {0, 0, 0};
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          for (int k = 0; k < 3; ++k) {
            gradQ[i][j] = gradQ[i][j] + HE(g, m, j, k, gp, e) * gQ[i][k];
            divF[i] = divF[i] + HE(g, m, j, k, gp, e) * gF[i][j][k];
          }
      R divU = gradQ[0][0] + gradQ[1][1] + gradQ[2][2];
      for (int i = 0; i < 3; ++i) {
        R r = R(0.5) * (divF[i] + ul[gp * 3 + i] * divU);
        for (int j = 0; j < 3; ++j) r = r + R(0.5) * (ul[gp * 3 + j] * gradQ[i][j]);
        buf[((size_t)e * n + gp) * 3 + i] = GV(g, m, gp, e) * r;
      }
    }
  }
  R *dst[3] = {Rmom, Rmom + N, Rmom + 2 * N};
  scatter(m, buf, 3, dst, R(1));
}

// ---- conjGrad_pressure_incomp, src/lib_sod2d_incomp/sources/mod_solver_incomp.f90:253-506
// Jacobi-preconditioned CG on A x = R - A x0 with FP64 dot products and the
// Polak-Ribiere beta of the reference; vectors in R (FP32 in the reference),
// alpha and beta rounded to R.  Owned nodes = working nodes on one rank.
// Returns the iteration count; *res_rel = ||r|| / ||b|| at exit.
template <class R>
int conjGrad_pressure(const Mesh &m, const Geo<R> &g, const R *diag, const R *x0, const R *Rhs, int maxIter,
                      double tol, R *out, double *res_rel) {
  const long long N = m.npoin;
  std::vector<R> x(N, 0), r0(N, 0), p0(N, 0), qn(N, 0), b(N, 0), z0(N, 0), z1(N, 0);
  eval_laplacian_mult(m, g, x0, qn.data());
  for (int t = 0; t < m.npoin_w; ++t) { int p = m.lpoin_w[t] - 1; b[p] = Rhs[p] - qn[p]; }
  for (int t = 0; t < m.npoin_w; ++t) { int p = m.lpoin_w[t] - 1; r0[p] = b[p]; }
  for (int t = 0; t < m.npoin_w; ++t) { int p = m.lpoin_w[t] - 1; z0[p] = r0[p] / diag[p]; p0[p] = z0[p]; }
  double auxT1 = 0.0;
  for (int t = 0; t < m.npoin_w; ++t) { int p = m.lpoin_w[t] - 1; auxT1 += (double)(b[p] * b[p]); }
  const double auxB = std::sqrt(auxT1);
  int iter;
  double nrm = auxB;
  for (iter = 1; iter <= maxIter; ++iter) {
    eval_laplacian_mult(m, g, p0.data(), qn.data());
    double Q1 = 0.0, Q2 = 0.0;
    for (int t = 0; t < m.npoin_w; ++t) {
      int p = m.lpoin_w[t] - 1;
      Q1 += (double)(r0[p] * z0[p]);
      Q2 += (double)(p0[p] * qn[p]);
    }
    R alpha = (R)(Q1 / Q2);
    for (int t = 0; t < m.npoin_w; ++t) { int p = m.lpoin_w[t] - 1; x[p] = x[p] + alpha * p0[p]; }
    for (int t = 0; t < m.npoin_w; ++t) { int p = m.lpoin_w[t] - 1; r0[p] = r0[p] - alpha * qn[p]; }
    for (int t = 0; t < m.npoin_w; ++t) { int p = m.lpoin_w[t] - 1; z1[p] = z0[p]; z0[p] = r0[p] / diag[p]; }
    auxT1 = 0.0;
    for (int t = 0; t < m.npoin_w; ++t) { int p = m.lpoin_w[t] - 1; auxT1 += (double)(r0[p] * r0[p]); }
    nrm = std::sqrt(auxT1);
    if (nrm < tol * auxB) break;
    double T = 0.0;
    for (int t = 0; t < m.npoin_w; ++t) { int p = m.lpoin_w[t] - 1; T += (double)(r0[p] * (z0[p] - z1[p])); }
    R beta = (R)(T / Q1);
    for (int t = 0; t < m.npoin_w; ++t) { int p = m.lpoin_w[t] - 1; p0[p] = z0[p] + beta * p0[p]; }
  }
  for (long long p = 0; p < N; ++p) out[p] = x0[p] + x[p];
  *res_rel = auxB > 0 ? nrm / auxB : 0.0;
  return iter > maxIter ? maxIter : iter;
}

// ---- species_tau, src/lib_species/sources/elem_stab_species.f90:122-148
// tau_e = max over the element nodes of helem_k * (c_species_stab / p) * |u|.
template <class R>
void species_tau(const Mesh &m, const R *u, const R *helem_k, R *tau, R c_species_stab = R(0.5)) {
  const long long N = m.npoin;
  Idx ix(m);
  for (long long e = 0; e < m.nelem; ++e) {
    R taul = 0;
    for (int a = 0; a < m.nnode; ++a) {
      const int p = ix.node(e, a);
      const R uu = u[p] * u[p] + u[p + N] * u[p + N] + u[p + 2 * N] * u[p + 2 * N];
      const R aux1 = std::sqrt(uu);
      taul = std::max(taul, helem_k[e] * (c_species_stab / R(m.porder)) * aux1);
    }
    tau[e] = taul;
  }
}

// Velocity gradient at one Gauss point: gradU(i,j) = sum_k He(j,k) d_k u_i.
template <class R>
inline void grad_u(const Mesh &m, const Geo<R> &g, const Idx &ix, long long e, int gp, const R *ul, R gradU[3][3]) {
  const int I = m.gI[gp] - 1, J = m.gJ[gp] - 1, K = m.gK[gp] - 1;
  R gU[3][3] = {};
  for (int ii = 0; ii < m.np1; ++ii) {
    const int an[3] = {ix.inv(ii, J, K), ix.inv(I, ii, K), ix.inv(I, J, ii)};
    for (int i = 0; i < 3; ++i)
      for (int d = 0; d < 3; ++d) gU[i][d] = gU[i][d] + DL(g, m, gp, d, ii) * ul[an[d] * 3 + i];
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      gradU[i][j] = 0;
      for (int k = 0; k < 3; ++k) gradU[i][j] = gradU[i][j] + HE(g, m, j, k, gp, e) * gU[i][k];
    }
}

// ---- eval_tau_veloc, src/lib_sod2d_incomp/sources/mod_operators.f90:373-483
// GradX/Y/Z(:,d) = (sum_e gpvol (grad u + grad u^T)(row, d)) / Ml.
template <class R>
void eval_tau_veloc(const Mesh &m, const Geo<R> &g, const R *u, R *GX, R *GY, R *GZ) {
  const long long N = m.npoin;
  const int n = m.nnode;
  for (long long p = 0; p < 3 * N; ++p) { GX[p] = 0; GY[p] = 0; GZ[p] = 0; }
  std::vector<R> buf((size_t)m.nelem * n * 9);
  Idx ix(m);
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < m.nelem; ++e) {
    std::vector<R> ul(n * 3);
    for (int a = 0; a < n; ++a) {
      const int p = ix.node(e, a);
      for (int d = 0; d < 3; ++d) ul[a * 3 + d] = u[p + N * d];
    }
    for (int gp = 0; gp < n; ++gp) {
      R gradU[3][3];
      grad_u(m, g, ix, e, gp, ul.data(), gradU);
      R *b = &buf[((size_t)e * n + gp) * 9];
      const R gv = GV(g, m, gp, e);
      for (int d = 0; d < 3; ++d) {
        b[d] = gv * (gradU[0][d] + gradU[d][0]);
        b[3 + d] = gv * (gradU[1][d] + gradU[d][1]);
        b[6 + d] = gv * (gradU[2][d] + gradU[d][2]);
      }
    }
  }
  R *dst[9] = {GX, GX + N, GX + 2 * N, GY, GY + N, GY + 2 * N, GZ, GZ + N, GZ + 2 * N};
  scatter(m, buf, 9, dst, R(1));
  for (int t = 0; t < m.npoin_w; ++t) {  // lumped_solver_vect: R / Ml
    const int p = m.lpoin_w[t] - 1;
    for (int c = 0; c < 9; ++c) dst[c][p] = dst[c][p] / g.Ml[p];
  }
}

// ---- full_diff_stab_incomp, src/lib_sod2d_incomp/sources/elem_stab_incomp.f90:12-153
// Rmom = sum_e weak div of (mu_fluid + mu_sgs + tau_e)(grad u + grad u^T)
// - tau_e TauP (Rmom is zeroed first).
template <class R>
void full_diff_stab_incomp(const Mesh &m, const Geo<R> &g, const R *u, const R *mu_fluid, const R *mu_sgs,
                           const R *TPX, const R *TPY, const R *TPZ, const R *tau_stab, R *Rmom) {
  const long long N = m.npoin, NE = m.nelem;
  const int n = m.nnode;
  for (long long p = 0; p < 3 * N; ++p) Rmom[p] = 0;
  std::vector<R> buf((size_t)m.nelem * n * 3);
  Idx ix(m);
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < m.nelem; ++e) {
    std::vector<R> ul(n * 3), mufl(n), musgs(n), tpx(n * 3), tpy(n * 3), tpz(n * 3);
    std::vector<R> tauX(n * 3), tauY(n * 3), tauZ(n * 3);
    for (int a = 0; a < n; ++a) {
      const int p = ix.node(e, a);
      mufl[a] = mu_fluid[p];
      musgs[a] = mu_sgs[e + NE * a];
      for (int d = 0; d < 3; ++d) {
        ul[a * 3 + d] = u[p + N * d];
        tpx[a * 3 + d] = TPX[p + N * d]; tpy[a * 3 + d] = TPY[p + N * d]; tpz[a * 3 + d] = TPZ[p + N * d];
      }
    }
    const R ts = tau_stab[e];
    for (int gp = 0; gp < n; ++gp) {
      const R mu_fgp = mufl[gp] + musgs[gp] + ts;
      R gradU[3][3];
      grad_u(m, g, ix, e, gp, ul.data(), gradU);
      R tau[3][3];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) tau[i][j] = gradU[i][j] + gradU[j][i];
      for (int d = 0; d < 3; ++d) {
        tauX[gp * 3 + d] = mu_fgp * tau[0][d] - ts * tpx[gp * 3 + d];
        tauY[gp * 3 + d] = mu_fgp * tau[1][d] - ts * tpy[gp * 3 + d];
        tauZ[gp * 3 + d] = mu_fgp * tau[2][d] - ts * tpz[gp * 3 + d];
      }
    }
    for (int gp = 0; gp < n; ++gp) {
      R *b = &buf[((size_t)e * n + gp) * 3];
      b[0] = weak_div(m, g, ix, e, gp, tauX.data());
      b[1] = weak_div(m, g, ix, e, gp, tauY.data());
      b[2] = weak_div(m, g, ix, e, gp, tauZ.data());
    }
  }
  R *dst[3] = {Rmom, Rmom + N, Rmom + 2 * N};
  scatter(m, buf, 3, dst, R(1));
}

// ---- conjGrad_veloc_incomp (LPS path, periodic), src/lib_sod2d_incomp/sources/mod_solver_incomp.f90:27-251
// Preconditioned CG on Ml x + fact dt D(x) = b, D = full_diff_stab_incomp
// with the LPS projection of its argument, preconditioner Ml / dt, x0 = Rp0,
// tau from species_tau(x0); vectors in R, dots in FP64 (node-major order),
// alpha and beta rounded to R.  Rio: in b (npoin,3), out x.  Returns the
// iteration count; *res_rel = ||r|| / ||r0|| at exit.
template <class R>
int conjGrad_veloc(const Mesh &m, const Geo<R> &g, R fact, R dt, const R *helem_k, const R *mu_fluid,
                   const R *mu_sgs, const R *Rp0, R *Rio, int maxIter, double tol, double *res_rel) {
  const long long N = m.npoin;
  std::vector<R> x(Rp0, Rp0 + 3 * N), r0(3 * N, 0), p0(3 * N, 0), qn(3 * N, 0), b(Rio, Rio + 3 * N), z0(3 * N, 0),
      z1(3 * N, 0), Mu(3 * N, 0), tau(m.nelem), TX(3 * N), TY(3 * N), TZ(3 * N);
  for (long long p = 0; p < N; ++p)
    for (int d = 0; d < 3; ++d) Mu[p + N * d] = g.Ml[p] / dt;
  species_tau(m, x.data(), helem_k, tau.data());
  auto apply = [&](const R *v) {
    eval_tau_veloc(m, g, v, TX.data(), TY.data(), TZ.data());
    full_diff_stab_incomp(m, g, v, mu_fluid, mu_sgs, TX.data(), TY.data(), TZ.data(), tau.data(), qn.data());
    for (int t = 0; t < m.npoin_w; ++t) {
      const int p = m.lpoin_w[t] - 1;
      for (int d = 0; d < 3; ++d) qn[p + N * d] = v[p + N * d] * g.Ml[p] + qn[p + N * d] * fact * dt;
    }
  };
  apply(x.data());
  for (int t = 0; t < m.npoin_w; ++t) {
    const int p = m.lpoin_w[t] - 1;
    for (int d = 0; d < 3; ++d) r0[p + N * d] = b[p + N * d] - qn[p + N * d];
  }
  for (int t = 0; t < m.npoin_w; ++t) {
    const int p = m.lpoin_w[t] - 1;
    for (int d = 0; d < 3; ++d) { z0[p + N * d] = r0[p + N * d] / Mu[p + N * d]; p0[p + N * d] = z0[p + N * d]; }
  }
  auto dot = [&](auto f) {
    double s = 0.0;
    for (int t = 0; t < m.npoin_w; ++t) {
      const int p = m.lpoin_w[t] - 1;
      for (int d = 0; d < 3; ++d) s += f(p + N * d);
    }
    return s;
  };
  const double auxB = std::sqrt(dot([&](long long k) { return (double)(r0[k] * r0[k]); }));
  double nrm = auxB;
  int iter;
  for (iter = 1; iter <= maxIter; ++iter) {
    apply(p0.data());
    const double Q1 = dot([&](long long k) { return (double)(r0[k] * z0[k]); });
    const double Q2 = dot([&](long long k) { return (double)(p0[k] * qn[k]); });
    const R alpha = (R)(Q1 / Q2);
    for (int t = 0; t < m.npoin_w; ++t) {
      const int p = m.lpoin_w[t] - 1;
      for (int d = 0; d < 3; ++d) x[p + N * d] = x[p + N * d] + alpha * p0[p + N * d];
    }
    for (int t = 0; t < m.npoin_w; ++t) {
      const int p = m.lpoin_w[t] - 1;
      for (int d = 0; d < 3; ++d) r0[p + N * d] = r0[p + N * d] - alpha * qn[p + N * d];
    }
    for (int t = 0; t < m.npoin_w; ++t) {
      const int p = m.lpoin_w[t] - 1;
      for (int d = 0; d < 3; ++d) { z1[p + N * d] = z0[p + N * d]; z0[p + N * d] = r0[p + N * d] / Mu[p + N * d]; }
    }
    nrm = std::sqrt(dot([&](long long k) { return (double)(r0[k] * r0[k]); }));
    if (nrm < tol * auxB) break;
    const double T = dot([&](long long k) { return (double)(r0[k] * (z0[k] - z1[k])); });
    const R beta = (R)(T / Q1);
    for (int t = 0; t < m.npoin_w; ++t) {
      const int p = m.lpoin_w[t] - 1;
      for (int d = 0; d < 3; ++d) p0[p + N * d] = z0[p + N * d] + beta * p0[p + N * d];
    }
  }
  for (long long k = 0; k < 3 * N; ++k) Rio[k] = x[k];
  *res_rel = auxB > 0 ? nrm / auxB : 0.0;
  return iter > maxIter ? maxIter : iter;
}

// ---- conjGrad_imex (periodic), src/lib_sod2d/sources/mod_solver_imex.f90:25-342
// CG on the five conserved variables v = (mass, energy, momentum x, y, z):
// Ml x + fact dt D(x) = b, where D(v) = full_diffusion_ijk(init, fact 1) with
// rho_n = the iterate's density x_mass, the argument's density v_mass,
// velocity v_mom / x_mass and temperature from v_E, v_mom and x_mass
// (mod_solver_imex.f90:97-107, 310-320); preconditioner Ml / dt; x0 = the
// state at the start of the step; vectors in R, dots in FP64 (node-major,
// variable inner), alpha and beta rounded to R.  (rho, E, q): in b, out x
// on the working nodes.  Returns the iteration count.
template <class R>
int conjGrad_imex(const Mesh &m, const Geo<R> &g, R fact, R dt, R gamma, R Rgas, R Cp, R Prt, const R *mu_fluid,
                  const R *mu_e, const R *mu_sgs, const R *rho0, const R *E0, const R *q0, R *rho, R *E, R *q,
                  int maxIter, double tol, double *res_rel) {
  const long long N = m.npoin;
  constexpr int NV = 5;
  std::vector<R> x(NV * N, 0), r0(NV * N, 0), p0(NV * N, 0), qn(NV * N, 0), b(NV * N, 0), z0(NV * N, 0),
      z1(NV * N, 0), au(3 * N, 0), aT(N, 0);
  auto W = [&](auto f) {
    for (int t = 0; t < m.npoin_w; ++t) f((long long)m.lpoin_w[t] - 1);
  };
  W([&](long long p) {
    b[p] = rho[p]; x[p] = rho0[p];
    b[p + N] = E[p]; x[p + N] = E0[p];
    for (int d = 0; d < 3; ++d) { b[p + N * (2 + d)] = q[p + N * d]; x[p + N * (2 + d)] = q0[p + N * d]; }
  });
  // velocity and temperature of the argument v over the iterate's density
  auto prim = [&](const R *v) {
    W([&](long long p) {
      const R rhol = x[p], El = v[p + N];
      R umag = 0;
      for (int d = 0; d < 3; ++d) {
        au[p + N * d] = v[p + N * (2 + d)] / rhol;
        umag = umag + (au[p + N * d] * au[p + N * d]);
      }
      const R e_int_l = (El / rhol) - R(0.5) * umag;
      aT[p] = rhol * (gamma - R(1.0)) * e_int_l / (rhol * Rgas);
    });
  };
  auto apply = [&](const R *v) {  // qn = v Ml + D(v) fact dt
    full_diffusion_ijk(m, g, Cp, Prt, x.data(), v, au.data(), aT.data(), mu_fluid, mu_e, mu_sgs, qn.data(),
                       qn.data() + 2 * N, qn.data() + N, true, R(1));
    W([&](long long p) {
      for (int k = 0; k < NV; ++k) qn[p + N * k] = v[p + N * k] * g.Ml[p] + qn[p + N * k] * fact * dt;
    });
  };
  auto dot = [&](auto f) {
    double s = 0.0;
    W([&](long long p) {
      for (int k = 0; k < NV; ++k) s += f(p + N * k);
    });
    return s;
  };
  prim(x.data());
  apply(x.data());
  W([&](long long p) {
    for (int k = 0; k < NV; ++k) r0[p + N * k] = b[p + N * k] - qn[p + N * k];
  });
  W([&](long long p) {
    const R M = g.Ml[p] / dt;
    for (int k = 0; k < NV; ++k) { z0[p + N * k] = r0[p + N * k] / M; p0[p + N * k] = z0[p + N * k]; }
  });
  prim(p0.data());
  const double auxB = std::sqrt(dot([&](long long k) { return (double)(r0[k] * r0[k]); }));
  double nrm = auxB;
  int iter;
  for (iter = 1; iter <= maxIter; ++iter) {
    apply(p0.data());
    const double Q1 = dot([&](long long k) { return (double)(r0[k] * z0[k]); });
    const double Q2 = dot([&](long long k) { return (double)(p0[k] * qn[k]); });
    const R alpha = (R)(Q1 / Q2);
    W([&](long long p) {
      for (int k = 0; k < NV; ++k) {
        x[p + N * k] = x[p + N * k] + alpha * p0[p + N * k];
        r0[p + N * k] = r0[p + N * k] - alpha * qn[p + N * k];
      }
    });
    W([&](long long p) {
      const R M = g.Ml[p] / dt;
      for (int k = 0; k < NV; ++k) { z1[p + N * k] = z0[p + N * k]; z0[p + N * k] = r0[p + N * k] / M; }
    });
    nrm = std::sqrt(dot([&](long long k) { return (double)(r0[k] * r0[k]); }));
    if (nrm < tol * auxB) break;
    const double T = dot([&](long long k) { return (double)(r0[k] * (z0[k] - z1[k])); });
    const R beta = (R)(T / Q1);
    W([&](long long p) {
      for (int k = 0; k < NV; ++k) p0[p + N * k] = z0[p + N * k] + beta * p0[p + N * k];
    });
    prim(p0.data());
  }
  W([&](long long p) {
    rho[p] = x[p];
    E[p] = x[p + N];
    for (int d = 0; d < 3; ++d) q[p + N * d] = x[p + N * (2 + d)];
  });
  *res_rel = auxB > 0 ? nrm / auxB : 0.0;
  return iter > maxIter ? maxIter : iter;
}

}  // namespace oracle
