// ORACLE -- test infrastructure only (see oracle_ops.hpp).  C entry points
// over the CPU restatement, in FP32 (_f32) and FP64 (_f64), for the tests'
// ctypes bindings, plus the compressible Taylor-Green time loop that pins the
// restatement against the reference's regression histories.
#include "oracle_ops.hpp"

#include <cstdio>

using namespace oracle;

extern "C" {

// Mesh description shared by every entry point (reference Fortran layout).
typedef struct {
  int porder, nelem, npoin, npoin_w;
  const int *connec, *lpoin_w, *invAtoIJK, *gmshAtoI, *gmshAtoJ, *gmshAtoK, *lelpn, *atoIJK;
  const void *He, *gpvol, *dlxigp_ip, *dNgp, *Ngp, *Ml, *invMl, *helem, *helem_l;
  double volT;
} oracle_mesh_t;

// Physical and numerical constants of a compressible case.
typedef struct {
  double gamma, Rgas, Cp, Prt, rho_inf, p_inf, cfl_conv, cfl_diff, maxPhysTime;
  int stages, rk_n, lps, log_first, log_step;
  // 1: first-step entropy viscosity as the reference source computes it
  // (time_integ_ls.f90:270-293); 0: zero entropy viscosity during the first
  // step, the behaviour the CPU regression history
  // Tests/TGV_Compressible/CPU/LS_RK_5/Reference/analysis_cube-4.dat shows.
  int first_mue;
  // 1: IMEX integrator (imex_main, time_integ_imex.f90) with `stages` (3 or
  // 4) stages and the implicit solve's maxIter / tol; 0: SSP LS-RK
  int imex, imex_maxiter;
  double imex_tol;
} oracle_comp_params_t;

}  // extern "C"

namespace {

Mesh make_mesh(const oracle_mesh_t *c) {
  Mesh m;
  m.porder = c->porder; m.np1 = c->porder + 1; m.nnode = m.np1 * m.np1 * m.np1;
  m.nelem = c->nelem; m.npoin = c->npoin; m.npoin_w = c->npoin_w;
  m.connec = c->connec; m.lpoin_w = c->lpoin_w; m.invA = c->invAtoIJK;
  m.gI = c->gmshAtoI; m.gJ = c->gmshAtoJ; m.gK = c->gmshAtoK; m.lelpn = c->lelpn; m.atoIJK = c->atoIJK;
  return m;
}
template <class R>
Geo<R> make_geo(const oracle_mesh_t *c) {
  Geo<R> g;
  g.He = (const R *)c->He; g.gpvol = (const R *)c->gpvol; g.dl = (const R *)c->dlxigp_ip;
  g.dNgp = (const R *)c->dNgp; g.Ngp = (const R *)c->Ngp; g.Ml = (const R *)c->Ml;
  g.invMl = (const R *)c->invMl; g.helem = (const R *)c->helem; g.helem_l = (const R *)c->helem_l;
  g.volT = (R)c->volT;
  return g;
}

// SSP low-storage RK coefficients, time_integ_ls.f90:87-167.
template <class R>
int rk_coeffs(int S, int n, R lam[7][7], R gam[7][7]) {
  for (int i = 0; i < 7; ++i)
    for (int j = 0; j < 7; ++j) { lam[i][j] = 0; gam[i][j] = 0; }
  // 1-based (i,j) stored at [i][j].
  if (S == 3) {
    lam[2][1] = 1; lam[3][1] = R(3.0) / R(4.0); lam[3][2] = R(1.0) / R(4.0);
    lam[4][1] = R(1.0) / R(3.0); lam[4][3] = R(2.0) / R(3.0);
    gam[2][1] = 1; gam[3][2] = R(0.25); gam[4][3] = R(2.0) / R(3.0);
  } else if (S == 4) {
    lam[2][1] = 1; lam[3][2] = 1; lam[4][1] = R(2.0) / R(3.0); lam[4][3] = R(1.0) / R(3.0); lam[5][4] = 1;
    gam[2][1] = R(0.5); gam[3][2] = R(0.5); gam[4][3] = R(1.0) / R(6.0); gam[5][4] = R(0.5);
  } else if (S == 5) {
    lam[2][1] = 1; lam[3][2] = 1; lam[4][3] = 1; lam[5][4] = 1; lam[6][5] = 1;
    if (n == 1) {
      lam[5][1] = R(0.571403511494104); lam[5][4] = R(0.428596488505896);
      gam[2][1] = R(0.443568244942995); gam[3][2] = R(0.291111420073766);
      gam[4][3] = R(0.270612601278217); gam[5][4] = R(0.110577759392786);
      gam[6][5] = R(0.458557505351052);
    } else {
      return -1;
    }
  } else {
    return -1;
  }
  return 0;
}

// Compressible periodic solver state: the reference's 4-level arrays and the
// time_integ_ls module arrays.
template <class R>
struct CompSolver {
  Mesh m;
  Geo<R> g;
  oracle_comp_params_t prm;
  long long N, NE;
  int n;
  std::vector<R> rho, u, q, pr, E, Tem, e_int, eta, mu_fluid, csound, machno, mu_e, mu_sgs, mu_factor;
  std::vector<R> Rmass, Rener, Rmom, Reta, auxReta, f_eta, aux_h, divU, vorti, tau_stab;
  std::vector<R> PMass, PEner, PMX, PMY, PMZ;
  R lam[7][7], gam[7][7];
  // IMEX: Butcher tables (1-based) and per-stage explicit / implicit residuals
  R ae[5][5] = {}, ai[5][5] = {};
  std::vector<R> RmI, RqI, ReI, DmI, DqI, DeI, Rms, Rqs, Res, Pz;
  int cg_iters = 0;
  bool first = true;
  R dt = 0;
  double time = 0;

  R *lv(std::vector<R> &a, int lvl, int ncomp = 1) { return a.data() + (size_t)N * ncomp * (lvl - 1); }

  void updateF() {
    const R gm = (R)prm.gamma, Rgas = (R)prm.Rgas;
    R *rho2 = lv(rho, 2), *u2 = lv(u, 2, 3), *q2 = lv(q, 2, 3), *pr2 = lv(pr, 2), *E2 = lv(E, 2), *T2 = lv(Tem, 2, 1);
    R *ei2 = lv(e_int, 2);
    for (int t = 0; t < m.npoin_w; ++t) {
      long long p = m.lpoin_w[t] - 1;
      R umag = 0;
      for (int d = 0; d < 3; ++d) {
        u2[p + N * d] = q2[p + N * d] / rho2[p];
        umag = umag + (u2[p + N * d] * u2[p + N * d]);
      }
      ei2[p] = (E2[p] / rho2[p]) - R(0.5) * umag;
      pr2[p] = rho2[p] * (gm - R(1.0)) * ei2[p];
      aux_h[p] = (gm / (gm - R(1.0))) * pr2[p] / rho2[p];
      T2[p] = pr2[p] / (rho2[p] * Rgas);
    }
    sutherland<R>(N, T2, mu_factor.data(), mu_fluid.data());
    full_convec_ijk<R>(m, g, u2, q2, rho2, pr2, aux_h.data(), Rmass.data(), Rmom.data(), Rener.data(), true, R(-1));
    if (prm.lps) {
      full_proj_ijk<R>(m, g, rho2, u2, T2, PMass.data(), PEner.data(), PMX.data(), PMY.data(), PMZ.data());
      full_diff_stab_ijk<R>(m, g, (R)prm.Cp, (R)prm.Prt, rho2, rho2, u2, T2, mu_fluid.data(), mu_e.data(),
                            mu_sgs.data(), PMass.data(), PEner.data(), PMX.data(), PMY.data(), PMZ.data(),
                            tau_stab.data(), Rmass.data(), Rmom.data(), Rener.data(), false, R(-1));
    } else {
      full_diffusion_ijk<R>(m, g, (R)prm.Cp, (R)prm.Prt, rho2, rho2, u2, T2, mu_fluid.data(), mu_e.data(),
                            mu_sgs.data(), Rmass.data(), Rmom.data(), Rener.data(), false, R(-1));
    }
    halo_update<R>({Rmom.data(), Rmom.data() + N, Rmom.data() + 2 * N, Rmass.data(), Rener.data()}, N);
    lumped_solver<R>(m, g, Rmass.data(), 1);
    lumped_solver<R>(m, g, Rener.data(), 1);
    lumped_solver<R>(m, g, Rmom.data(), 3);
  }

  void stage_update(int istep) {  // istep 1-based; istep == 1: first (low-storage) stage
    R *rho1 = lv(rho, 1), *rho2 = lv(rho, 2), *E1 = lv(E, 1), *E2 = lv(E, 2), *q1 = lv(q, 1, 3), *q2 = lv(q, 2, 3);
    for (int t = 0; t < m.npoin_w; ++t) {
      long long p = m.lpoin_w[t] - 1;
      if (istep == 1) {
        rho2[p] = rho2[p] + gam[2][1] * dt * Rmass[p];
        E2[p] = E2[p] + gam[2][1] * dt * Rener[p];
        for (int d = 0; d < 3; ++d) q2[p + N * d] = q2[p + N * d] + gam[2][1] * dt * Rmom[p + N * d];
      } else {
        R l1 = lam[istep + 1][1], li = lam[istep + 1][istep], gi = gam[istep + 1][istep];
        rho2[p] = l1 * rho1[p] + li * rho2[p] + gi * dt * Rmass[p];
        E2[p] = l1 * E1[p] + li * E2[p] + gi * dt * Rener[p];
        for (int d = 0; d < 3; ++d) q2[p + N * d] = l1 * q1[p + N * d] + li * q2[p + N * d] + gi * dt * Rmom[p + N * d];
      }
    }
  }

  // rk_4_ls_main, time_integ_ls.f90:202-487 (periodic, no LES/BC/buffer).
  void rk_step() {
    const R gm = (R)prm.gamma, Rgas = (R)prm.Rgas;
    R *u1 = lv(u, 1, 3), *u2 = lv(u, 2, 3);
    R *rho1 = lv(rho, 1), *rho2 = lv(rho, 2), *eta1 = lv(eta, 1), *eta2 = lv(eta, 2);
    if (prm.lps) comp_tau<R>(m, g, csound.data(), u2, tau_stab.data());
    if (first) {
      first = false;
      for (int t = 0; t < m.npoin_w; ++t) {
        long long p = m.lpoin_w[t] - 1;
        for (int d = 0; d < 3; ++d) f_eta[p + N * d] = u1[p + N * d] * eta1[p];
      }
      generic_scalar_convec_ijk<R>(m, g, f_eta.data(), eta1, u1, Reta.data(), true, R(1));
      halo_update<R>({Reta.data()}, N);  // time_integ_ls.f90:287
      lumped_solver<R>(m, g, Reta.data(), 1);
      smart_visc_spectral_imex<R>(m, g, Reta.data(), rho1, u1, csound.data(), mu_e.data());
      if (!prm.first_mue) std::fill(mu_e.begin(), mu_e.end(), R(0));
      updateF();
    }
    stage_update(1);
    for (int istep = 2; istep <= prm.stages; ++istep) {
      updateF();
      stage_update(istep);
    }
    R *q2 = lv(q, 2, 3), *pr2 = lv(pr, 2), *E2 = lv(E, 2), *T2 = lv(Tem, 2), *ei2 = lv(e_int, 2);
    for (int t = 0; t < m.npoin_w; ++t) {
      long long p = m.lpoin_w[t] - 1;
      R umag = 0;
      for (int d = 0; d < 3; ++d) {
        u2[p + N * d] = q2[p + N * d] / rho2[p];
        umag = umag + u2[p + N * d] * u2[p + N * d];
      }
      ei2[p] = (E2[p] / rho2[p]) - R(0.5) * umag;
      pr2[p] = rho2[p] * (gm - R(1.0)) * ei2[p];
      csound[p] = std::sqrt(gm * pr2[p] / rho2[p]);
      umag = std::sqrt(umag);
      machno[p] = umag / csound[p];
      T2[p] = pr2[p] / (rho2[p] * Rgas);
    }
    thermo_entropy<R>(m, gm, (R)prm.p_inf, (R)prm.rho_inf, rho2, pr2, u1, eta.data(), f_eta.data());
    R *Reta1 = Reta.data(), *Reta2 = Reta.data() + N;
    generic_scalar_convec_ijk<R>(m, g, f_eta.data(), eta1, u1, Reta2, true, R(1));
    halo_update<R>({Reta2}, N);  // time_integ_ls.f90:431
    lumped_solver<R>(m, g, Reta2, 1);
    for (int t = 0; t < m.npoin_w; ++t) {
      long long p = m.lpoin_w[t] - 1;
      auxReta[p] = (R(1.5) * Reta2[p] - R(0.5) * Reta1[p]) + R(1.0) * (eta2[p] - eta1[p]) / dt;
      Reta1[p] = Reta2[p];
    }
    smart_visc_spectral_imex<R>(m, g, auxReta.data(), rho2, u2, csound.data(), mu_e.data());
    eval_divergence<R>(m, g, u2, divU.data());
    compute_vorticity<R>(m, g, u2, vorti.data());
    ducros_visc_limit<R>(m, g, rho2, u2, divU.data(), vorti.data(), csound.data(), mu_e.data());
    sutherland<R>(N, T2, mu_factor.data(), mu_fluid.data());
  }

  // Butcher tables of init_imex_solver, time_integ_imex.f90:42-158
  int imex_coeffs(int S) {
    if (S == 4) {
      const R bi[5] = {0, R(4.0 / 15.0), R(1.0 / 3.0), R(7.0 / 30.0), R(1.0 / 6.0)};
      const R be[5] = {0, R(1.0 / 4.0), R(0.0), R(3.0 / 4.0), R(0.0)};
      ai[2][1] = bi[1]; ai[2][2] = bi[1];
      ai[3][1] = bi[1]; ai[3][2] = bi[2]; ai[3][3] = R(1.0 / 15.0);
      ai[4][1] = bi[1]; ai[4][2] = bi[2]; ai[4][3] = bi[3]; ai[4][4] = bi[4];
      ae[2][1] = R(8.0 / 15.0);
      ae[3][1] = be[1]; ae[3][2] = R(5.0 / 12.0);
      ae[4][1] = be[1]; ae[4][2] = be[2]; ae[4][3] = be[3]; ae[4][4] = be[4];
      return 0;
    }
    if (S == 3) {
      ai[2][1] = R(0.353842865099275); ai[2][2] = R(0.353842865099275);
      ai[3][1] = R(0.398930808264689); ai[3][2] = R(0.345755244189622); ai[3][3] = R(0.255313947545689);
      ae[2][1] = R(0.711664700366941);
      ae[3][1] = R(0.077338168947683); ae[3][2] = R(0.917273367886007);
      return 0;
    }
    return -1;
  }

  // EOS of a stage, time_integ_imex.f90:424-438 (also csound, Mach)
  void eos2() {
    const R gm = (R)prm.gamma, Rgas = (R)prm.Rgas;
    R *rho2 = lv(rho, 2), *u2 = lv(u, 2, 3), *q2 = lv(q, 2, 3), *pr2 = lv(pr, 2), *E2 = lv(E, 2), *T2 = lv(Tem, 2);
    R *ei2 = lv(e_int, 2);
    for (int t = 0; t < m.npoin_w; ++t) {
      long long p = m.lpoin_w[t] - 1;
      R umag = 0;
      for (int d = 0; d < 3; ++d) {
        u2[p + N * d] = q2[p + N * d] / rho2[p];
        umag = umag + u2[p + N * d] * u2[p + N * d];
      }
      ei2[p] = (E2[p] / rho2[p]) - R(0.5) * umag;
      pr2[p] = rho2[p] * (gm - R(1.0)) * ei2[p];
      aux_h[p] = (gm / (gm - R(1.0))) * pr2[p] / rho2[p];
      csound[p] = std::sqrt(gm * pr2[p] / rho2[p]);
      umag = std::sqrt(umag);
      machno[p] = umag / csound[p];
      T2[p] = pr2[p] / (rho2[p] * Rgas);
    }
  }

  // imex_main, time_integ_imex.f90:181-525 (periodic, no wall model, source
  // or LES; flag_use_ducros and flag_total_enthalpy off).  Convection and
  // diffusion residuals carry the subroutines' default fact +1 (their saved
  // aux_fact is never set otherwise on this path).  full_stab_ijk (fact -1)
  // is taken as full_diff_stab_ijk with zero viscosities and fact +1: the
  // same terms with the sign moved inside, equal in every bit.
  void imex_step() {
    const int S = prm.stages;
    const R gm = (R)prm.gamma;
    R *u1 = lv(u, 1, 3), *u2 = lv(u, 2, 3), *q1 = lv(q, 1, 3), *q2 = lv(q, 2, 3);
    R *rho1 = lv(rho, 1), *rho2 = lv(rho, 2), *eta1 = lv(eta, 1), *eta2 = lv(eta, 2);
    R *E1 = lv(E, 1), *E2 = lv(E, 2), *pr1 = lv(pr, 1), *T1 = lv(Tem, 1);
    auto st = [&](std::vector<R> &a, int k, int nc = 1) { return a.data() + (size_t)N * nc * (k - 1); };
    if (first) {
      first = false;
      for (int t = 0; t < m.npoin_w; ++t) {
        long long p = m.lpoin_w[t] - 1;
        for (int d = 0; d < 3; ++d) f_eta[p + N * d] = u1[p + N * d] * eta1[p];
      }
      generic_scalar_convec_ijk<R>(m, g, f_eta.data(), eta1, u1, Reta.data(), true, R(1));
      lumped_solver<R>(m, g, Reta.data(), 1);
      smart_visc_spectral_imex<R>(m, g, Reta.data(), rho1, u1, csound.data(), mu_e.data());
      if (!prm.first_mue) std::fill(mu_e.begin(), mu_e.end(), R(0));
      for (int t = 0; t < m.npoin_w; ++t) {
        long long p = m.lpoin_w[t] - 1;
        aux_h[p] = (gm / (gm - R(1.0))) * pr1[p] / rho1[p];
      }
      full_convec_ijk<R>(m, g, u1, q1, rho1, pr1, aux_h.data(), st(RmI, 1), st(RqI, 1, 3), st(ReI, 1), true, R(1));
      full_diffusion_ijk<R>(m, g, (R)prm.Cp, (R)prm.Prt, rho1, rho1, u1, T1, mu_fluid.data(), mu_e.data(),
                            mu_sgs.data(), st(DmI, 1), st(DqI, 1, 3), st(DeI, 1), true, R(1));
    } else {
      std::copy(st(RmI, S), st(RmI, S) + N, st(RmI, 1));
      std::copy(st(DmI, S), st(DmI, S) + N, st(DmI, 1));
      std::copy(st(ReI, S), st(ReI, S) + N, st(ReI, 1));
      std::copy(st(DeI, S), st(DeI, S) + N, st(DeI, 1));
      std::copy(st(RqI, S, 3), st(RqI, S, 3) + 3 * N, st(RqI, 1, 3));
      std::copy(st(DqI, S, 3), st(DqI, S, 3) + 3 * N, st(DqI, 1, 3));
    }
    if (prm.lps) {
      comp_tau<R>(m, g, csound.data(), u2, tau_stab.data());
      full_proj_ijk<R>(m, g, rho1, u1, T1, PMass.data(), PEner.data(), PMX.data(), PMY.data(), PMZ.data());
      full_diff_stab_ijk<R>(m, g, (R)prm.Cp, (R)prm.Prt, rho1, rho1, u1, T1, Pz.data(), Pz.data(), Pz.data(),
                            PMass.data(), PEner.data(), PMX.data(), PMY.data(), PMZ.data(), tau_stab.data(),
                            Rms.data(), Rqs.data(), Res.data(), true, R(1));
    }
    for (int is = 2; is <= S; ++is) {
      for (long long p = 0; p < N; ++p) {
        rho2[p] = -dt * Rms[p];
        E2[p] = -dt * Res[p];
        for (int d = 0; d < 3; ++d) q2[p + N * d] = -dt * Rqs[p + N * d];
        for (int js = 1; js < is; ++js) {
          rho2[p] = rho2[p] - dt * ae[is][js] * st(RmI, js)[p] - dt * ai[is][js] * st(DmI, js)[p];
          E2[p] = E2[p] - dt * ae[is][js] * st(ReI, js)[p] - dt * ai[is][js] * st(DeI, js)[p];
          for (int d = 0; d < 3; ++d)
            q2[p + N * d] = q2[p + N * d] - dt * ae[is][js] * st(RqI, js, 3)[p + N * d] -
                            dt * ai[is][js] * st(DqI, js, 3)[p + N * d];
        }
      }
      for (long long p = 0; p < N; ++p) {
        rho2[p] = rho2[p] + rho1[p] * g.Ml[p];
        E2[p] = E2[p] + E1[p] * g.Ml[p];
        for (int d = 0; d < 3; ++d) q2[p + N * d] = q2[p + N * d] + q1[p + N * d] * g.Ml[p];
      }
      double res = 0.0;
      cg_iters = conjGrad_imex<R>(m, g, ai[is][is], dt, gm, (R)prm.Rgas, (R)prm.Cp, (R)prm.Prt, mu_fluid.data(),
                                  mu_e.data(), mu_sgs.data(), rho1, E1, q1, rho2, E2, q2, prm.imex_maxiter,
                                  prm.imex_tol, &res);
      eos2();
      full_convec_ijk<R>(m, g, u2, q2, rho2, lv(pr, 2), aux_h.data(), st(RmI, is), st(RqI, is, 3), st(ReI, is), true,
                         R(1));
      full_diffusion_ijk<R>(m, g, (R)prm.Cp, (R)prm.Prt, rho2, rho2, u2, lv(Tem, 2), mu_fluid.data(), mu_e.data(),
                            mu_sgs.data(), st(DmI, is), st(DqI, is, 3), st(DeI, is), true, R(1));
    }
    R *pr2 = lv(pr, 2), *T2 = lv(Tem, 2);
    thermo_entropy<R>(m, gm, (R)prm.p_inf, (R)prm.rho_inf, rho2, pr2, u1, eta.data(), f_eta.data());
    R *Reta1 = Reta.data(), *Reta2 = Reta.data() + N;
    generic_scalar_convec_ijk<R>(m, g, f_eta.data(), eta1, u1, Reta2, true, R(1));
    lumped_solver<R>(m, g, Reta2, 1);
    for (int t = 0; t < m.npoin_w; ++t) {
      long long p = m.lpoin_w[t] - 1;
      auxReta[p] = (R(1.5) * Reta2[p] - R(0.5) * Reta1[p]) + R(1.0) * (eta2[p] - eta1[p]) / dt;
      Reta1[p] = Reta2[p];
    }
    smart_visc_spectral_imex<R>(m, g, auxReta.data(), rho2, u2, csound.data(), mu_e.data());
    eval_divergence<R>(m, g, u2, divU.data());
    compute_vorticity<R>(m, g, u2, vorti.data());
    ducros_visc_limit<R>(m, g, rho2, u2, divU.data(), vorti.data(), csound.data(), mu_e.data());
    sutherland<R>(N, T2, mu_factor.data(), mu_fluid.data());
  }

  void analysis(double *row) {
    R *rho2 = lv(rho, 2), *u2 = lv(u, 2, 3);
    double EK = volAvg_EK<R>(m, g, (R)prm.rho_inf, rho2, u2);
    double eS, eD, eT;
    visc_dissipationRate<R>(m, g, (R)prm.rho_inf, mu_fluid.data(), mu_e.data(), u2, g.volT, &eS, &eD, &eT);
    R mx = 0;
    for (int t = 0; t < m.npoin_w; ++t) mx = std::max(mx, machno[m.lpoin_w[t] - 1]);
    double mxd = (double)mx;
    reduce_all(&mxd, 1, 1);  // MPI_Allreduce MAX, mod_analysis.f90:166
    mx = (R)mxd;
    row[0] = (double)(R)time; row[1] = (double)(R)EK; row[2] = eS; row[3] = eD; row[4] = eT; row[5] = (double)mx;
  }

  R eval_dt() {
    return adapt_dt_cfl<R>(m, g, lv(u, 2, 3), csound.data(), (R)prm.cfl_conv, (R)prm.cfl_diff, mu_fluid.data(),
                           mu_sgs.data(), mu_e.data(), lv(rho, 2));
  }
};

// Compressible TGV driver: CFDSolverBase_run / evalTimeIteration
// (CFDSolverBase.f90:2601-2747, :1929-2164) for a periodic case.
template <class R>
int tgv_comp_run(const oracle_mesh_t *cm, const oracle_comp_params_t *prm, const R *init /*10 fields*/,
                 R mu_factor_v, int nsteps, double *hist, int max_rows, int *nrows, R *final_state) {
  CompSolver<R> s;
  s.m = make_mesh(cm);
  s.g = make_geo<R>(cm);
  s.prm = *prm;
  s.N = s.m.npoin; s.NE = s.m.nelem; s.n = s.m.nnode;
  const long long N = s.N;
  if (prm->imex ? s.imex_coeffs(prm->stages) : rk_coeffs<R>(prm->stages, prm->rk_n, s.lam, s.gam)) return -1;
  s.rho.assign(N * 4, 0); s.u.assign(N * 12, 0); s.q.assign(N * 12, 0); s.pr.assign(N * 4, 0); s.E.assign(N * 4, 0);
  s.Tem.assign(N * 2, 0); s.e_int.assign(N * 2, 0); s.eta.assign(N * 4, 0); s.mu_fluid.assign(N, 0);
  s.csound.assign(N, 0); s.machno.assign(N, 0); s.mu_e.assign(s.NE * s.n, 0); s.mu_sgs.assign(s.NE * s.n, 0);
  s.mu_factor.assign(N, mu_factor_v);
  s.Rmass.assign(N, 0); s.Rener.assign(N, 0); s.Rmom.assign(N * 3, 0); s.Reta.assign(N * 2, 0);
  s.auxReta.assign(N, 0); s.f_eta.assign(N * 3, 0); s.aux_h.assign(N, 0); s.divU.assign(N, 0);
  s.vorti.assign(N * 3, 0); s.tau_stab.assign(s.NE, 0);
  s.PMass.assign(N * 3, 0); s.PEner.assign(N * 3, 0); s.PMX.assign(N * 3, 0); s.PMY.assign(N * 3, 0); s.PMZ.assign(N * 3, 0);
  if (prm->imex) {
    const int S = prm->stages;
    s.RmI.assign(N * S, 0); s.ReI.assign(N * S, 0); s.DmI.assign(N * S, 0); s.DeI.assign(N * S, 0);
    s.RqI.assign(N * 3 * S, 0); s.DqI.assign(N * 3 * S, 0);
    s.Rms.assign(N, 0); s.Res.assign(N, 0); s.Rqs.assign(N * 3, 0); s.Pz.assign((size_t)s.NE * s.n + N, 0);
  }
  // init layout: rho, u(3), q(3), pr, E, Tem, e_int, csound, machno, eta -> 14 N values
  const R *I = init;
  std::copy(I, I + N, s.lv(s.rho, 2)); I += N;
  std::copy(I, I + 3 * N, s.lv(s.u, 2, 3)); I += 3 * N;
  std::copy(I, I + 3 * N, s.lv(s.q, 2, 3)); I += 3 * N;
  std::copy(I, I + N, s.lv(s.pr, 2)); I += N;
  std::copy(I, I + N, s.lv(s.E, 2)); I += N;
  std::copy(I, I + N, s.lv(s.Tem, 2)); I += N;
  std::copy(I, I + N, s.lv(s.e_int, 2)); I += N;
  std::copy(I, I + N, s.csound.data()); I += N;
  std::copy(I, I + N, s.machno.data()); I += N;
  std::copy(I, I + N, s.lv(s.eta, 2)); I += N;
  sutherland<R>(N, s.lv(s.Tem, 2), s.mu_factor.data(), s.mu_fluid.data());
  int rows = 0;
  if (rows < max_rows) s.analysis(hist + 6 * rows++);
  s.dt = s.eval_dt();
  int log_next = prm->log_first;
  for (int istep = 1; istep <= nsteps; ++istep) {
    std::copy(s.lv(s.rho, 2), s.lv(s.rho, 2) + N, s.lv(s.rho, 1));
    std::copy(s.lv(s.u, 2, 3), s.lv(s.u, 2, 3) + 3 * N, s.lv(s.u, 1, 3));
    std::copy(s.lv(s.q, 2, 3), s.lv(s.q, 2, 3) + 3 * N, s.lv(s.q, 1, 3));
    std::copy(s.lv(s.pr, 2), s.lv(s.pr, 2) + N, s.lv(s.pr, 1));
    std::copy(s.lv(s.E, 2), s.lv(s.E, 2) + N, s.lv(s.E, 1));
    std::copy(s.lv(s.Tem, 2), s.lv(s.Tem, 2) + N, s.lv(s.Tem, 1));
    std::copy(s.lv(s.e_int, 2), s.lv(s.e_int, 2) + N, s.lv(s.e_int, 1));
    std::copy(s.lv(s.eta, 2), s.lv(s.eta, 2) + N, s.lv(s.eta, 1));
    if (prm->imex) s.imex_step();
    else s.rk_step();
    s.time = (double)((R)s.time + s.dt);
    if (log_next == istep) {
      if (rows < max_rows) s.analysis(hist + 6 * rows++);
      log_next += prm->log_step;
    }
    s.dt = s.eval_dt();
    if (prm->maxPhysTime > 0 && (R)s.time >= (R)prm->maxPhysTime) break;
  }
  *nrows = rows;
  if (final_state) {
    R *F = final_state;
    std::copy(s.lv(s.rho, 2), s.lv(s.rho, 2) + N, F); F += N;
    std::copy(s.lv(s.q, 2, 3), s.lv(s.q, 2, 3) + 3 * N, F); F += 3 * N;
    std::copy(s.lv(s.E, 2), s.lv(s.E, 2) + N, F); F += N;
    std::copy(s.mu_e.begin(), s.mu_e.end(), F);
  }
  return 0;
}

// One RHS evaluation (updateF body) at a given state: EOS + Sutherland +
// convection + LPS projection + stabilised diffusion + lumped inversion.
template <class R>
int rhs_eval(const oracle_mesh_t *cm, const oracle_comp_params_t *prm, const R *rho, const R *q, const R *E,
             const R *mu_e, const R *mu_factor, const R *tau_stab, R *Rmass, R *Rmom, R *Rener, R *proj15) {
  CompSolver<R> s;
  s.m = make_mesh(cm);
  s.g = make_geo<R>(cm);
  s.prm = *prm;
  s.N = s.m.npoin; s.NE = s.m.nelem; s.n = s.m.nnode;
  const long long N = s.N;
  s.rho.assign(N * 4, 0); s.u.assign(N * 12, 0); s.q.assign(N * 12, 0); s.pr.assign(N * 4, 0); s.E.assign(N * 4, 0);
  s.Tem.assign(N * 2, 0); s.e_int.assign(N * 2, 0); s.mu_fluid.assign(N, 0);
  s.mu_e.assign(mu_e, mu_e + s.NE * s.n); s.mu_sgs.assign(s.NE * s.n, 0);
  s.mu_factor.assign(mu_factor, mu_factor + N);
  s.Rmass.assign(N, 0); s.Rener.assign(N, 0); s.Rmom.assign(N * 3, 0); s.aux_h.assign(N, 0);
  s.tau_stab.assign(tau_stab, tau_stab + s.NE);
  s.PMass.assign(N * 3, 0); s.PEner.assign(N * 3, 0); s.PMX.assign(N * 3, 0); s.PMY.assign(N * 3, 0); s.PMZ.assign(N * 3, 0);
  std::copy(rho, rho + N, s.lv(s.rho, 2));
  std::copy(q, q + 3 * N, s.lv(s.q, 2, 3));
  std::copy(E, E + N, s.lv(s.E, 2));
  s.updateF();
  std::copy(s.Rmass.begin(), s.Rmass.end(), Rmass);
  std::copy(s.Rmom.begin(), s.Rmom.end(), Rmom);
  std::copy(s.Rener.begin(), s.Rener.end(), Rener);
  if (proj15) {
    // order: ProjMass, ProjEner, ProjMX, ProjMY, ProjMZ, each (N,3)
    R *P = proj15;
    for (auto *v : {&s.PMass, &s.PEner, &s.PMX, &s.PMY, &s.PMZ}) { std::copy(v->begin(), v->end(), P); P += 3 * N; }
  }
  return 0;
}

// Entropy-viscosity chain at the end of a step, time_integ_ls.f90:409-463,
// for a given old/new level: returns mu_e(E,n) after the Ducros limiter.
template <class R>
int entropy_visc(const oracle_mesh_t *cm, const oracle_comp_params_t *prm, const R *rho1, const R *u1,
                 const R *eta1, const R *Reta1, const R *rho2, const R *u2, const R *pr2, const R *csound, R dt,
                 R *mu_e, R *eta2_out, R *Reta2_out) {
  Mesh m = make_mesh(cm);
  Geo<R> g = make_geo<R>(cm);
  const long long N = m.npoin;
  std::vector<R> eta(N * 2), feta(N * 3, 0), Reta2(N), aux(N), divU(N), vorti(3 * N);
  std::copy(eta1, eta1 + N, eta.data() + N);  // thermo_entropy shifts level 2 into level 1
  thermo_entropy<R>(m, (R)prm->gamma, (R)prm->p_inf, (R)prm->rho_inf, rho2, pr2, u1, eta.data(), feta.data());
  generic_scalar_convec_ijk<R>(m, g, feta.data(), eta.data(), u1, Reta2.data(), true, R(1));
  lumped_solver<R>(m, g, Reta2.data(), 1);
  for (int t = 0; t < m.npoin_w; ++t) {
    long long p = m.lpoin_w[t] - 1;
    aux[p] = (R(1.5) * Reta2[p] - R(0.5) * Reta1[p]) + R(1.0) * (eta[p + N] - eta[p]) / dt;
  }
  smart_visc_spectral_imex<R>(m, g, aux.data(), rho2, u2, csound, mu_e);
  eval_divergence<R>(m, g, u2, divU.data());
  compute_vorticity<R>(m, g, u2, vorti.data());
  ducros_visc_limit<R>(m, g, rho2, u2, divU.data(), vorti.data(), csound, mu_e);
  if (eta2_out) std::copy(eta.data() + N, eta.data() + 2 * N, eta2_out);
  if (Reta2_out) std::copy(Reta2.begin(), Reta2.end(), Reta2_out);
  return 0;
}

// Jacobian restatement in precision R (jacobian_oper.f90:7-139), used to
// build FP64 geometry and to cross-check the product's FP32 set-up.
template <class R>
int elem_jacobian(int porder, int nelem, int npoin, const int *connec, const R *coord, const R *dNgp,
                  const R *wgp, R *gpvol, R *He) {
  const int np1 = porder + 1, nnode = np1 * np1 * np1;
  const long long ne = nelem, nn = npoin;
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < ne; ++e)
    for (int gp = 0; gp < nnode; ++gp) {
      double Je[3][3];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          double dot = 0.0;
          for (int a = 0; a < nnode; ++a) {
            R prod = dNgp[i + 3 * (a + (long long)nnode * gp)] * coord[(connec[e + ne * a] - 1) + nn * j];
            dot = dot + (double)prod;
          }
          Je[i][j] = dot;
        }
      double det = (Je[0][0] * Je[1][1] * Je[2][2] + Je[0][1] * Je[1][2] * Je[2][0] + Je[0][2] * Je[1][0] * Je[2][1] -
                    Je[2][0] * Je[1][1] * Je[0][2] - Je[2][1] * Je[1][2] * Je[0][0] - Je[2][2] * Je[1][0] * Je[0][1]);
      R gv = (R)det;
      double a[9];
      a[0] = Je[1][1] * Je[2][2] - Je[2][1] * Je[1][2];
      a[1] = Je[1][0] * Je[2][2] - Je[2][0] * Je[1][2];
      a[2] = Je[1][0] * Je[2][1] - Je[2][0] * Je[1][1];
      a[3] = Je[0][1] * Je[2][2] - Je[2][1] * Je[0][2];
      a[4] = Je[0][0] * Je[2][2] - Je[2][0] * Je[0][2];
      a[5] = Je[0][0] * Je[2][1] - Je[2][0] * Je[0][1];
      a[6] = Je[0][1] * Je[1][2] - Je[1][1] * Je[0][2];
      a[7] = Je[0][0] * Je[1][2] - Je[1][0] * Je[0][2];
      a[8] = Je[0][0] * Je[1][1] - Je[1][0] * Je[0][1];
      a[1] = -a[1]; a[3] = -a[3]; a[5] = -a[5]; a[7] = -a[7];
      double b[9];
      for (int t = 0; t < 9; ++t) b[t] = a[t];
      b[1] = a[3]; b[2] = a[6]; b[3] = a[1]; b[5] = a[7]; b[6] = a[2]; b[7] = a[5];
      for (int t = 0; t < 9; ++t) b[t] = (double)(R(1.0) / gv) * b[t];
      R *he = He + 9 * ((long long)gp + (long long)nnode * e);
      he[0 + 3 * 0] = (R)b[0]; he[0 + 3 * 1] = (R)b[1]; he[0 + 3 * 2] = (R)b[2];
      he[1 + 3 * 0] = (R)b[3]; he[1 + 3 * 1] = (R)b[4]; he[1 + 3 * 2] = (R)b[5];
      he[2 + 3 * 0] = (R)b[6]; he[2 + 3 * 1] = (R)b[7]; he[2 + 3 * 2] = (R)b[8];
      gpvol[gp + (long long)nnode * e] = wgp[gp] * gv;
    }
  return 0;
}

// First-step entropy viscosity (time_integ_ls.f90:270-293): residual of the
// entropy flux at level 1, lumped, then smart_visc_spectral_imex.
template <class R>
int first_mue(const oracle_mesh_t *cm, const R *rho1, const R *u1, const R *eta1, const R *csound, R *mu_e,
              R *Reta_out) {
  Mesh m = make_mesh(cm);
  Geo<R> g = make_geo<R>(cm);
  const long long N = m.npoin;
  std::vector<R> feta(3 * N, 0), Reta(N);
  for (int t = 0; t < m.npoin_w; ++t) {
    long long p = m.lpoin_w[t] - 1;
    for (int d = 0; d < 3; ++d) feta[p + N * d] = u1[p + N * d] * eta1[p];
  }
  generic_scalar_convec_ijk<R>(m, g, feta.data(), eta1, u1, Reta.data(), true, R(1));
  lumped_solver<R>(m, g, Reta.data(), 1);
  smart_visc_spectral_imex<R>(m, g, Reta.data(), rho1, u1, csound, mu_e);
  if (Reta_out) std::copy(Reta.begin(), Reta.end(), Reta_out);
  return 0;
}

}  // namespace

#define ORACLE_BOTH(X) X(float, f32) X(double, f64)

extern "C" {

#define DEF_RUN(R, S)                                                                                    \
  int oracle_tgv_comp_run_##S(const oracle_mesh_t *m, const oracle_comp_params_t *p, const R *init,     \
                              double mu_factor, int nsteps, double *hist, int max_rows, int *nrows,     \
                              R *final_state) {                                                         \
    return tgv_comp_run<R>(m, p, init, (R)mu_factor, nsteps, hist, max_rows, nrows, final_state);      \
  }                                                                                                      \
  int oracle_rhs_##S(const oracle_mesh_t *m, const oracle_comp_params_t *p, const R *rho, const R *q,   \
                     const R *E, const R *mu_e, const R *mu_factor, const R *tau_stab, R *Rmass,         \
                     R *Rmom, R *Rener, R *proj15) {                                                     \
    return rhs_eval<R>(m, p, rho, q, E, mu_e, mu_factor, tau_stab, Rmass, Rmom, Rener, proj15);        \
  }                                                                                                      \
  int oracle_entropy_visc_##S(const oracle_mesh_t *m, const oracle_comp_params_t *p, const R *rho1,     \
                              const R *u1, const R *eta1, const R *Reta1, const R *rho2, const R *u2,   \
                              const R *pr2, const R *csound, double dt, R *mu_e, R *eta2, R *Reta2) {   \
    return entropy_visc<R>(m, p, rho1, u1, eta1, Reta1, rho2, u2, pr2, csound, (R)dt, mu_e, eta2, Reta2); \
  }                                                                                                      \
  int oracle_elem_jacobian_##S(int porder, int nelem, int npoin, const int *connec, const R *coord,     \
                               const R *dNgp, const R *wgp, R *gpvol, R *He) {                          \
    return elem_jacobian<R>(porder, nelem, npoin, connec, coord, dNgp, wgp, gpvol, He);                 \
  }                                                                                                      \
  int oracle_convec_##S(const oracle_mesh_t *cm, const R *u, const R *q, const R *rho, const R *pr,     \
                        const R *E, R *Rmass, R *Rmom, R *Rener, int init, double fact) {               \
    Mesh m = make_mesh(cm);                                                                              \
    Geo<R> g = make_geo<R>(cm);                                                                          \
    full_convec_ijk<R>(m, g, u, q, rho, pr, E, Rmass, Rmom, Rener, init != 0, (R)fact);                 \
    return 0;                                                                                            \
  }                                                                                                      \
  int oracle_comp_tau_##S(const oracle_mesh_t *cm, const R *csound, const R *u, R *tau) {               \
    Mesh m = make_mesh(cm);                                                                              \
    Geo<R> g = make_geo<R>(cm);                                                                          \
    comp_tau<R>(m, g, csound, u, tau);                                                                   \
    return 0;                                                                                            \
  }                                                                                                      \
  int oracle_dt_##S(const oracle_mesh_t *cm, const R *u, const R *csound, double cfl_conv,              \
                    double cfl_diff, const R *mu_fluid, const R *mu_sgs, const R *mu_e, const R *rho,   \
                    double *dt) {                                                                        \
    Mesh m = make_mesh(cm);                                                                              \
    Geo<R> g = make_geo<R>(cm);                                                                          \
    *dt = (double)adapt_dt_cfl<R>(m, g, u, csound, (R)cfl_conv, (R)cfl_diff, mu_fluid, mu_sgs, mu_e, rho); \
    return 0;                                                                                            \
  }                                                                                                      \
  int oracle_analysis_##S(const oracle_mesh_t *cm, double rho0, const R *rho, const R *u,               \
                          const R *mu_fluid, const R *mu_e, double *out4) {                              \
    Mesh m = make_mesh(cm);                                                                              \
    Geo<R> g = make_geo<R>(cm);                                                                          \
    out4[0] = volAvg_EK<R>(m, g, (R)rho0, rho, u);                                                       \
    visc_dissipationRate<R>(m, g, (R)rho0, mu_fluid, mu_e, u, g.volT, out4 + 1, out4 + 2, out4 + 3);    \
    return 0;                                                                                            \
  }
ORACLE_BOTH(DEF_RUN)

#define DEF_FIRST(R, S)                                                                                \
  int oracle_first_mue_##S(const oracle_mesh_t *m, const R *rho1, const R *u1, const R *eta1,          \
                           const R *csound, R *mu_e, R *Reta) {                                        \
    return first_mue<R>(m, rho1, u1, eta1, csound, mu_e, Reta);                                        \
  }
ORACLE_BOTH(DEF_FIRST)

#define DEF_INCOMP(R, S)                                                                               \
  int oracle_laplacian_##S(const oracle_mesh_t *cm, const R *p, R *out) {                              \
    Mesh m = make_mesh(cm);                                                                            \
    Geo<R> g = make_geo<R>(cm);                                                                        \
    eval_laplacian_mult<R>(m, g, p, out);                                                              \
    return 0;                                                                                          \
  }                                                                                                    \
  int oracle_laplacian_diag_##S(const oracle_mesh_t *cm, R *out) {                                     \
    Mesh m = make_mesh(cm);                                                                            \
    Geo<R> g = make_geo<R>(cm);                                                                        \
    eval_laplacian_diag<R>(m, g, out);                                                                 \
    return 0;                                                                                          \
  }                                                                                                    \
  int oracle_gradient_##S(const oracle_mesh_t *cm, const R *x, R *out) {                               \
    Mesh m = make_mesh(cm);                                                                            \
    Geo<R> g = make_geo<R>(cm);                                                                        \
    eval_gradient<R>(m, g, x, out);                                                                    \
    return 0;                                                                                          \
  }                                                                                                    \
  int oracle_divergence_##S(const oracle_mesh_t *cm, const R *u, R *out) {                             \
    Mesh m = make_mesh(cm);                                                                            \
    Geo<R> g = make_geo<R>(cm);                                                                        \
    eval_divergence<R>(m, g, u, out);                                                                  \
    return 0;                                                                                          \
  }                                                                                                    \
  int oracle_convec_incomp_##S(const oracle_mesh_t *cm, const R *u, const R *q, R *out) {              \
    Mesh m = make_mesh(cm);                                                                            \
    Geo<R> g = make_geo<R>(cm);                                                                        \
    full_convec_ijk_incomp<R>(m, g, u, q, out);                                                        \
    return 0;                                                                                          \
  }                                                                                                    \
  int oracle_cg_pressure_##S(const oracle_mesh_t *cm, const R *diag, const R *x0, const R *rhs,        \
                             int maxIter, double tol, R *out, double *res) {                           \
    Mesh m = make_mesh(cm);                                                                            \
    Geo<R> g = make_geo<R>(cm);                                                                        \
    return conjGrad_pressure<R>(m, g, diag, x0, rhs, maxIter, tol, out, res);                          \
  }
ORACLE_BOTH(DEF_INCOMP)

#define DEF_VELOC(R, S)                                                                                \
  int oracle_species_tau_##S(const oracle_mesh_t *cm, const R *u, R *tau) {                            \
    Mesh m = make_mesh(cm);                                                                            \
    Geo<R> g = make_geo<R>(cm);                                                                        \
    species_tau<R>(m, u, g.helem, tau);                                                                \
    return 0;                                                                                          \
  }                                                                                                    \
  int oracle_eval_tau_veloc_##S(const oracle_mesh_t *cm, const R *u, R *out) {                         \
    Mesh m = make_mesh(cm);                                                                            \
    Geo<R> g = make_geo<R>(cm);                                                                        \
    const long long N = m.npoin;                                                                       \
    eval_tau_veloc<R>(m, g, u, out, out + 3 * N, out + 6 * N);                                         \
    return 0;                                                                                          \
  }                                                                                                    \
  int oracle_full_diff_stab_incomp_##S(const oracle_mesh_t *cm, const R *u, const R *mu_fluid,         \
                                       const R *mu_sgs, const R *tauP, const R *tau_stab, R *out) {    \
    Mesh m = make_mesh(cm);                                                                            \
    Geo<R> g = make_geo<R>(cm);                                                                        \
    const long long N = m.npoin;                                                                       \
    full_diff_stab_incomp<R>(m, g, u, mu_fluid, mu_sgs, tauP, tauP + 3 * N, tauP + 6 * N, tau_stab,    \
                             out);                                                                     \
    return 0;                                                                                          \
  }                                                                                                    \
  int oracle_cg_veloc_##S(const oracle_mesh_t *cm, R fact, R dt, const R *mu_fluid, const R *mu_sgs,   \
                          const R *Rp0, R *Rio, int maxIter, double tol, double *res) {                \
    Mesh m = make_mesh(cm);                                                                            \
    Geo<R> g = make_geo<R>(cm);                                                                        \
    return conjGrad_veloc<R>(m, g, fact, dt, g.helem, mu_fluid, mu_sgs, Rp0, Rio, maxIter, tol, res);  \
  }
ORACLE_BOTH(DEF_VELOC)

}  // extern "C"

// Entropy-viscosity pieces, individually (generic_scalar_convec_ijk,
// smart_visc_spectral_imex, ducros_visc_limit, compute_vorticity).
#define DEF_ENTROPY(R, S)                                                                              \
  int oracle_scalar_convec_##S(const oracle_mesh_t *cm, const R *q, const R *eta, const R *u, R *Rout, \
                               int init, double fact) {                                                \
    Mesh m = make_mesh(cm);                                                                            \
    Geo<R> g = make_geo<R>(cm);                                                                        \
    generic_scalar_convec_ijk<R>(m, g, q, eta, u, Rout, init != 0, (R)fact);                           \
    return 0;                                                                                          \
  }                                                                                                    \
  int oracle_smart_visc_##S(const oracle_mesh_t *cm, const R *Reta, const R *rho, const R *u,          \
                            const R *csound, R *mu_e) {                                                \
    Mesh m = make_mesh(cm);                                                                            \
    Geo<R> g = make_geo<R>(cm);                                                                        \
    smart_visc_spectral_imex<R>(m, g, Reta, rho, u, csound, mu_e);                                     \
    return 0;                                                                                          \
  }                                                                                                    \
  int oracle_ducros_##S(const oracle_mesh_t *cm, const R *rho, const R *u, const R *divU,              \
                        const R *vorti, const R *csound, R *mu_e) {                                    \
    Mesh m = make_mesh(cm);                                                                            \
    Geo<R> g = make_geo<R>(cm);                                                                        \
    ducros_visc_limit<R>(m, g, rho, u, divU, vorti, csound, mu_e);                                     \
    return 0;                                                                                          \
  }                                                                                                    \
  int oracle_vorticity_##S(const oracle_mesh_t *cm, const R *u, R *vorti) {                            \
    Mesh m = make_mesh(cm);                                                                            \
    Geo<R> g = make_geo<R>(cm);                                                                        \
    compute_vorticity<R>(m, g, u, vorti);                                                              \
    return 0;                                                                                          \
  }
extern "C" int oracle_set_reduce(void (*fn)(void *, double *, int, int), void *user) {
  ReduceHook::fn = fn;
  ReduceHook::user = user;
  return 0;
}

#define DEF_HALO(R, S)                                                                                 \
  int oracle_set_halo_##S(void (*fn)(void *, R *const *, int, long long), void *user) {                \
    HaloHook<R>::fn = fn;                                                                                \
    HaloHook<R>::user = user;                                                                            \
    return 0;                                                                                            \
  }

extern "C" {
ORACLE_BOTH(DEF_HALO)
ORACLE_BOTH(DEF_ENTROPY)
}
