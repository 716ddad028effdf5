// C-ABI entry points of the compressible time integration: the low-storage
// SSP RK step with the entropy-viscosity chain, the IMEX step, the CFL
// time step and the analysis integrals (declarations: include/sod2d_gpu.h).
#include "cg_common.cuh"

// ---- compressible time integration --------------------------------------

namespace {

int rk_coeffs(int S, int n, double lam[7][7], double gam[7][7]) {
  for (int i = 0; i < 7; ++i)
    for (int j = 0; j < 7; ++j) { lam[i][j] = 0.0; gam[i][j] = 0.0; }
  // time_integ_ls.f90:87-167, 1-based indices
  if (S == 3) {
    lam[2][1] = 1.0; lam[3][1] = 3.0 / 4.0; lam[3][2] = 1.0 / 4.0; lam[4][1] = 1.0 / 3.0; lam[4][3] = 2.0 / 3.0;
    gam[2][1] = 1.0; gam[3][2] = 0.25; gam[4][3] = 2.0 / 3.0;
  } else if (S == 4) {
    lam[2][1] = 1.0; lam[3][2] = 1.0; lam[4][1] = 2.0 / 3.0; lam[4][3] = 1.0 / 3.0; lam[5][4] = 1.0;
    gam[2][1] = 0.5; gam[3][2] = 0.5; gam[4][3] = 1.0 / 6.0; gam[5][4] = 0.5;
  } else if (S == 5) {
    lam[2][1] = lam[3][2] = lam[4][3] = lam[5][4] = lam[6][5] = 1.0;
    if (n == 1) {
      lam[5][1] = 0.571403511494104; lam[5][4] = 0.428596488505896;
      gam[2][1] = 0.443568244942995; gam[3][2] = 0.291111420073766; gam[4][3] = 0.270612601278217;
      gam[5][4] = 0.110577759392786; gam[6][5] = 0.458557505351052;
    } else if (n == 2) {
      lam[4][1] = 0.682342861037239; lam[4][3] = 0.317657138962761; lam[6][1] = 0.045230974482400;
      lam[6][5] = 0.954769025517600;
      gam[2][1] = 0.465388589249323; gam[3][2] = 0.465388589249323; gam[4][3] = 0.124745797313998;
      gam[5][4] = 0.465388589249323; gam[6][5] = 0.154263303748666;
    } else if (n == 3) {
      lam[5][1] = 0.592032910942121; lam[5][4] = 1.0 - lam[5][1];
      gam[2][1] = 0.266541020678955; gam[3][2] = 0.548560709048532; gam[4][3] = 0.289517014154401;
      gam[5][4] = 0.086408328057923; gam[6][5] = 0.462943578481813;
    } else if (n == 4) {
      lam[4][1] = 0.707858560931430; lam[4][3] = 1.0 - lam[4][1]; lam[6][1] = 0.222853615080669;
      lam[6][5] = 1.0 - lam[6][1];
      gam[2][1] = 0.292845746913355; gam[3][2] = 0.339532793976408; gam[4][3] = 0.200532330324672;
      gam[5][4] = 0.701676169006879; gam[6][5] = 0.155278812461877;
    } else {
      return -1;
    }
  } else {
    return -1;
  }
  return 0;
}

// The FP32 reference rounds its RK coefficients to real(rp): mirror that.
inline double as_rp(double v, bool fp64) { return fp64 ? v : (double)(float)v; }

template <class T>
void launch_stage(sod_gpu_ctx *c, double l1, double li, double gdt, int first) {
  auto &S = c->comp;
  State5<T> U1, U2;
  for (int f = 0; f < 5; ++f) { U1.f[f] = (T *)S.U1[f]; U2.f[f] = (T *)S.U2[f]; }
  k_stage<T><<<nblk(c->npoin_w, 256), 256, 0, c->stream>>>(c->npoin_w, c->npoin, c->lpoin_w, U1, U2, S.Rmass,
                                                           S.Rmom, S.Rener, (T)l1, (T)li, (T)gdt, first, S.rho32,
                                                           S.q32, S.E32);
}

// RHS at the current FP32 shadow state into comp.R* (updateF body).
int comp_updateF(sod_gpu_ctx *c) {
  auto &S = c->comp;
  RhsArgs A{};
  A.rho = S.rho32; A.q = S.q32; A.E = S.E32; A.mu_factor = S.mu_factor;
  A.mue_t = c->mue_t; A.tau_stab = S.tau; A.proj12 = c->proj12;
  A.fact_c = -1.0f; A.fact_d = -1.0f;
  int rc = dispatch(c, [&](auto L) {
    L.proj(c, false, S.rho32, S.q32, S.E32);
    gather_proj_aos(c);
    int hrc = halo_sum(c, halo_proj_view(c));
    if (hrc) return hrc;
    L.template rhs<MODE_CONV | MODE_DIFF, IN_CONS>(c, A);
    return 0;
  });
  if (rc) return rc;
  gather_res(c, S.Rmass, S.Rmom, S.Rener, 0, 1);
  return halo_sum(c, halo_res_view(c, S.Rmass, S.Rmom, S.Rener));
}

// Entropy residual (+ divergence and vorticity when dc) of (feta, eta1, u1[, u2]).
int comp_entropy_pass(sod_gpu_ctx *c, float *Reta_out, bool dc) {
  auto &S = c->comp;
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    constexpr int P = LL::P_;
    if (dc)
      k_entropy_elem<P, LL::EPB, true><<<LL::grid(c->nelem), LL::TPB, 0, c->stream>>>(c->md(), S.feta, S.eta1, S.u1,
                                                                                     S.u2, c->slotsB);
    else
      k_entropy_elem<P, LL::EPB, false><<<LL::grid(c->nelem), LL::TPB, 0, c->stream>>>(c->md(), S.feta, S.eta1, S.u1,
                                                                                      S.u2, c->slotsB);
    return 0;
  });
  k_gather_entropy<<<nblk(c->npoin, 256), 256, 0, c->stream>>>(c->md(), c->slotsB, c->lelpn, c->is_work, Reta_out,
                                                               S.divU, S.vort, dc ? 1 : 0);
  // halo sums of the lumped entropy residual (time_integ_ls.f90:287, :431),
  // the divergence and the vorticity (mod_operators.f90:566, :759)
  HaloView v{};
  const long long N = c->npoin;
  v.nstride = 1;
  v.width = dc ? 5 : 1;
  v.comp[0] = Reta_out;
  if (dc) { v.comp[1] = S.divU; v.comp[2] = S.vort; v.comp[3] = S.vort + N; v.comp[4] = S.vort + 2 * N; }
  return halo_sum(c, v);
}

int comp_visc(sod_gpu_ctx *c, const float *Reta, const float *rho, const float *u, bool ducros) {
  auto &S = c->comp;
  const unsigned init_bits = 0x47C35000u;  // 100000.0f
  CUDA_TRY(cudaMemcpyAsync(S.bits, &init_bits, sizeof(unsigned), cudaMemcpyHostToDevice, c->stream));
  k_min_rho<<<MINMAX_BLOCKS, 256, 0, c->stream>>>(c->npoin_w, c->lpoin_w, rho, S.bits);
  // the bits of a positive float order like the float: reduce as float
  int rc = allreduce(c, S.bits, 1, SOD_REDUCE_MIN_F32);
  if (rc) return rc;
  ViscArgs V{};
  V.Reta = Reta; V.rho = rho; V.u = u; V.csound = S.csound; V.divU = S.divU; V.vort = S.vort; V.Ml = c->Ml;
  V.helem = c->helem; V.helem_l_t = c->helem_l_t; V.min_rho_bits = S.bits;
  V.ce = c->phys.ce; V.cmax = c->phys.cmax; V.cglob = c->phys.cglob; V.ducros_min = c->phys.ducros_min_val;
  V.inv_p = 1.0f / (float)c->P; V.ducros = ducros ? 1 : 0;
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    k_visc<LL::P_><<<nblk(c->nelem, 8), 256, 0, c->stream>>>(c->md(), V, c->a_of_t, c->mue_t, nullptr);
    return 0;
  });
  return 0;
}

}  // namespace

extern "C" {

int sod_gpu_generic_scalar_convec_ijk(sod_gpu_ctx *c, const float *q, const float *eta, const float *u, float *R,
                                      int initialze, float fact) {
  if (!c || !q || !eta || !u || !R) return fail(SOD_GPU_EINVAL, "bad argument");
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    k_entropy_elem<LL::P_, LL::EPB, false><<<LL::grid(c->nelem), LL::TPB, 0, c->stream>>>(c->md(), q, eta, u,
                                                                                        nullptr, c->slotsB, fact);
    return 0;
  });
  OutPtrs o{};
  o.p[0] = R;
  k_gather<8, 1, false><<<nblk(c->npoin, 256), 256, 0, c->stream>>>(c->md(), c->slotsB, nullptr, o,
                                                                     initialze ? 0 : 1, 0);
  return c->finish();
}

int sod_gpu_smart_visc_spectral_imex(sod_gpu_ctx *c, const float *Reta, const float *rho, const float *u,
                                     const float *csound, float *mu_e) {
  if (!c || !Reta || !rho || !u || !csound || !mu_e) return fail(SOD_GPU_EINVAL, "bad argument");
  if (!c->helem) return fail(SOD_GPU_EINVAL, "smart_visc_spectral_imex needs helem at init");
  int rc;
  if (!c->vbits && (rc = c->alloc(&c->vbits, 4))) return rc;
  const unsigned init_bits = 0x47C35000u;  // 100000.0f, the reference's initial minimum
  CUDA_TRY(cudaMemcpyAsync(c->vbits, &init_bits, sizeof(unsigned), cudaMemcpyHostToDevice, c->stream));
  k_min_rho<<<MINMAX_BLOCKS, 256, 0, c->stream>>>(c->npoin_w, c->lpoin_w, rho, c->vbits);
  if ((rc = allreduce(c, c->vbits, 1, SOD_REDUCE_MIN_F32))) return rc;
  ViscArgs V{};
  V.Reta = Reta; V.rho = rho; V.u = u; V.csound = csound; V.Ml = c->Ml;
  V.helem = c->helem; V.helem_l_t = c->helem_l_t; V.min_rho_bits = c->vbits;
  V.ce = c->phys.ce; V.cmax = c->phys.cmax; V.cglob = c->phys.cglob; V.ducros_min = c->phys.ducros_min_val;
  V.inv_p = 1.0f / (float)c->P; V.ducros = 0;
  // the element-layout copy goes to scratch: the context's own mu_e is left alone
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    k_visc<LL::P_><<<nblk(c->nelem, 8), 256, 0, c->stream>>>(c->md(), V, c->a_of_t, c->slotsA, mu_e);
    return 0;
  });
  return c->finish();
}

int sod_gpu_ducros_visc_limit(sod_gpu_ctx *c, const float *rho, const float *u, const float *divU,
                              const float *vorti, const float *csound, float *mu_e) {
  if (!c || !rho || !u || !divU || !vorti || !csound || !mu_e) return fail(SOD_GPU_EINVAL, "bad argument");
  if (!c->helem_l_t) return fail(SOD_GPU_EINVAL, "ducros_visc_limit needs helem_l at init");
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    k_ducros<LL::P_><<<nblk(c->nelem, 8), 256, 0, c->stream>>>(c->md(), u, divU, vorti, c->Ml, c->helem_l_t,
                                                               c->phys.ducros_min_val, c->a_of_t, mu_e);
    return 0;
  });
  return c->finish();
}

int sod_gpu_rk_ls_stage(sod_gpu_ctx *c, int first, float lam1, float lami, float gam, float dt, const float *rho1,
                        const float *q1, const float *E1, float *rho2, float *q2, float *E2, const float *Rmass,
                        const float *Rmom, const float *Rener) {
  if (!c || !rho2 || !q2 || !E2 || !Rmass || !Rmom || !Rener || (!first && (!rho1 || !q1 || !E1)))
    return fail(SOD_GPU_EINVAL, "bad argument");
  k_ls_stage_ref<<<nblk(c->npoin_w, 256), 256, 0, c->stream>>>(c->npoin_w, c->npoin, c->lpoin_w, first ? 1 : 0, lam1,
                                                               lami, gam, dt, rho1, q1, E1, rho2, q2, E2, Rmass,
                                                               Rmom, Rener);
  return c->finish();
}

int sod_gpu_comp_init_state(sod_gpu_ctx *c, const sod_rk_cfg_t *cfg, const float *rho, const float *u,
                            const float *q, const float *pr, const float *E, const float *Tem, const float *csound,
                            const float *machno, const float *eta) {
  if (!c || !cfg || !rho || !u || !q || !pr || !E || !Tem || !csound || !machno || !eta)
    return fail(SOD_GPU_EINVAL, "bad argument");
  if (!c->helem || !c->helem_l_t || !c->lelpn) return fail(SOD_GPU_EINVAL, "time integration needs helem, helem_l and lelpn at init");
  auto &S = c->comp;
  if (rk_coeffs(cfg->stages, cfg->rk_n, S.lam, S.gam)) return fail(SOD_GPU_EINVAL, "unsupported RK scheme");
  const size_t N = c->npoin, NE = (size_t)c->nelem;
  int rc = 0;
  if (!S.ready) {
    const size_t tb = cfg->fp64_state ? sizeof(double) : sizeof(float);
    for (int f = 0; f < 5; ++f) {
      char *p1, *p2;
      if ((rc = c->alloc(&p1, N * tb)) || (rc = c->alloc(&p2, N * tb))) return rc;
      S.U1[f] = p1; S.U2[f] = p2;
    }
    float **f1[] = {&S.rho32, &S.E32, &S.eint, &S.pr, &S.csound, &S.machno, &S.Tem, &S.eta1, &S.eta2,
                    &S.Reta1, &S.Reta2, &S.aux, &S.divU, &S.mu_fluid, &S.Rmass, &S.Rener};
    for (auto pp : f1)
      if ((rc = c->alloc(pp, N))) return rc;
    float **f3[] = {&S.q32, &S.u1, &S.u2, &S.feta, &S.vort, &S.Rmom};
    for (auto pp : f3)
      if ((rc = c->alloc(pp, 3 * N))) return rc;
    if ((rc = c->alloc(&S.tau, NE)) || (rc = c->alloc(&S.part, 3 * NE)) || (rc = c->alloc(&S.bits, 4)) ||
        (rc = c->alloc(&S.sums, 4)))
      return rc;
    S.ready = true;
    S.fp64 = cfg->fp64_state != 0;
  } else if ((cfg->fp64_state != 0) != S.fp64) {
    return fail(SOD_GPU_EINVAL, "state precision cannot change after the first init");
  }
  S.stages = cfg->stages;
  S.mu_factor = cfg->mu_factor;
  S.first = true;
  const cudaStream_t st = c->stream;
  CUDA_TRY(cudaMemcpyAsync(S.rho32, rho, N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(S.q32, q, 3 * N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(S.E32, E, N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(S.u2, u, 3 * N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(S.pr, pr, N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(S.Tem, Tem, N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(S.csound, csound, N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(S.machno, machno, N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(S.eta2, eta, N * 4, cudaMemcpyDeviceToDevice, st));
  for (float *z : {S.Reta1, S.Reta2, S.Rmass, S.Rener, S.divU, S.aux})
    CUDA_TRY(cudaMemsetAsync(z, 0, N * 4, st));
  CUDA_TRY(cudaMemsetAsync(S.Rmom, 0, 3 * N * 4, st));
  CUDA_TRY(cudaMemsetAsync(S.vort, 0, 3 * N * 4, st));
  CUDA_TRY(cudaMemsetAsync(c->mue_t, 0, NE * c->N * 4, st));
  c->mue_set = true;
  // FP64 (or FP32) master state from the FP32 initial arrays
  {
    const float *src[5] = {rho, q, q + N, q + 2 * N, E};
    std::vector<float> h(N);
    for (int f = 0; f < 5; ++f) {
      CUDA_TRY(cudaMemcpyAsync(h.data(), src[f], N * 4, cudaMemcpyDeviceToHost, st));
      CUDA_TRY(cudaStreamSynchronize(st));
      if (S.fp64) {
        std::vector<double> d(h.begin(), h.end());
        CUDA_TRY(cudaMemcpy(S.U2[f], d.data(), N * 8, cudaMemcpyHostToDevice));
      } else {
        CUDA_TRY(cudaMemcpy(S.U2[f], h.data(), N * 4, cudaMemcpyHostToDevice));
      }
    }
  }
  k_sutherland<<<nblk(c->npoin_w, 256), 256, 0, st>>>(c->npoin_w, c->lpoin_w, S.mu_factor, S.Tem, S.mu_fluid);
  return c->finish();
}

int sod_gpu_comp_rk_ls_step(sod_gpu_ctx *c, float dt) {
  if (!c || !c->comp.ready) return fail(SOD_GPU_EINVAL, "state not initialised");
  if (!(dt > 0.f)) return fail(SOD_GPU_EINVAL, "dt must be positive");
  auto &S = c->comp;
  const cudaStream_t st = c->stream;
  const size_t N = c->npoin;
  const size_t tb = S.fp64 ? 8 : 4;
  // level 1 <- level 2 (CFDSolverBase.f90:1951-1960)
  for (int f = 0; f < 5; ++f) CUDA_TRY(cudaMemcpyAsync(S.U1[f], S.U2[f], N * tb, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(S.u1, S.u2, 3 * N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(S.eta1, S.eta2, N * 4, cudaMemcpyDeviceToDevice, st));
  // tau from level 2 (comp_tau)
  k_comp_tau<<<nblk(c->nelem, 8), 256, 0, st>>>(c->nelem, c->N, c->conn, c->helem, S.csound, S.u2, c->npoin,
                                                c->phys.c_species_stab / (float)c->P, S.tau);
  if (S.first) {
    S.first = false;
    k_feta<<<nblk(c->npoin_w, 256), 256, 0, st>>>(c->npoin_w, c->npoin, c->lpoin_w, S.u1, S.eta1, S.feta);
    int rc;
    if ((rc = comp_entropy_pass(c, S.Reta1, false)) || (rc = comp_visc(c, S.Reta1, S.rho32, S.u1, false)) ||
        (rc = comp_updateF(c)))
      return rc;
  }
  const double dtd = (double)dt;
  auto stage = [&](double l1, double li, double g, int first) {
    const double gdt = S.fp64 ? g * dtd : (double)((float)g * dt);
    if (S.fp64)
      launch_stage<double>(c, l1, li, gdt, first);
    else
      launch_stage<float>(c, as_rp(l1, false), as_rp(li, false), gdt, first);
  };
  stage(0.0, 0.0, as_rp(S.gam[2][1], S.fp64), 1);
  for (int i = 2; i <= S.stages; ++i) {
    int rc = comp_updateF(c);
    if (rc) return rc;
    stage(as_rp(S.lam[i + 1][1], S.fp64), as_rp(S.lam[i + 1][i], S.fp64), as_rp(S.gam[i + 1][i], S.fp64), 0);
  }
  const float gm = c->phys.gamma_gas;
  k_eos_end<<<nblk(c->npoin_w, 256), 256, 0, st>>>(c->npoin_w, c->npoin, c->lpoin_w, gm - 1.0f, gm, c->phys.Rgas,
                                                   S.rho32, S.q32, S.E32, S.u2, S.eint, S.pr, S.csound, S.machno,
                                                   S.Tem);
  k_thermo_entropy<<<nblk(c->npoin_w, 256), 256, 0, st>>>(c->npoin_w, c->npoin, c->lpoin_w, gm, c->phys.p_inf,
                                                          c->phys.rho_inf, S.rho32, S.pr, S.u1, S.eta1, S.eta2,
                                                          S.feta);
  int rc = comp_entropy_pass(c, S.Reta2, true);
  if (rc) return rc;
  k_aux_reta<<<nblk(c->npoin_w, 256), 256, 0, st>>>(c->npoin_w, c->lpoin_w, dt, S.Reta1, S.Reta2, S.eta1, S.eta2,
                                                    S.aux);
  if ((rc = comp_visc(c, S.aux, S.rho32, S.u2, true))) return rc;
  k_sutherland<<<nblk(c->npoin_w, 256), 256, 0, st>>>(c->npoin_w, c->lpoin_w, S.mu_factor, S.Tem, S.mu_fluid);
  return c->finish();
}

}  // extern "C"

// ---- IMEX time step (imex_main) ------------------------------------------

namespace {

int ensure_imex(sod_gpu_ctx *c) {
  auto &X = c->imex;
  if (X.R) return 0;
  const size_t N = c->npoin, EN = (size_t)c->nelem * c->N;
  int rc;
  if ((rc = c->alloc(&X.R, 4 * 5 * N)) || (rc = c->alloc(&X.D, 4 * 5 * N)) || (rc = c->alloc(&X.stab, 5 * N)) ||
      (rc = c->alloc(&X.lvl1, 5 * N)) || (rc = c->alloc(&X.aux_h, N)) || (rc = c->alloc(&X.x, 5 * N)) ||
      (rc = c->alloc(&X.r, 5 * N)) || (rc = c->alloc(&X.p, 5 * N)) || (rc = c->alloc(&X.qn, 5 * N)) ||
      (rc = c->alloc(&X.b, 5 * N)) || (rc = c->alloc(&X.z, 5 * N)) || (rc = c->alloc(&X.z1, 5 * N)) ||
      (rc = c->alloc(&X.au, 3 * N)) || (rc = c->alloc(&X.aT, N)) || (rc = c->alloc(&X.zmu, N)) ||
      (rc = c->alloc(&X.zmue, EN)))
    return rc;
  if (!c->cg.part && ((rc = c->alloc(&c->cg.part, 8 * DOT_BLOCKS)) || (rc = c->alloc(&c->cg.dots, 16)))) return rc;
  for (float *v : {X.R, X.D}) CUDA_TRY(cudaMemsetAsync(v, 0, 4 * 5 * N * 4, c->stream));
  for (float *v : {X.stab, X.x, X.r, X.p, X.qn, X.b, X.z, X.z1}) CUDA_TRY(cudaMemsetAsync(v, 0, 5 * N * 4, c->stream));
  CUDA_TRY(cudaMemsetAsync(X.au, 0, 3 * N * 4, c->stream));
  for (float *v : {X.aT, X.zmu, X.aux_h}) CUDA_TRY(cudaMemsetAsync(v, 0, N * 4, c->stream));
  CUDA_TRY(cudaMemsetAsync(X.zmue, 0, EN * 4, c->stream));
  return 0;
}

// Butcher tables of init_imex_solver, time_integ_imex.f90:42-158, rounded
// to FP32 as the reference's real(rp) constants
ImexCoef imex_coef(int S) {
  ImexCoef k{};
  if (S == 4) {
    const float bi1 = 4.0f / 15.0f, bi2 = 1.0f / 3.0f, bi3 = 7.0f / 30.0f, bi4 = 1.0f / 6.0f;
    const float be1 = 1.0f / 4.0f, be2 = 0.0f, be3 = 3.0f / 4.0f, be4 = 0.0f;
    k.ai[2][1] = bi1; k.ai[2][2] = bi1;
    k.ai[3][1] = bi1; k.ai[3][2] = bi2; k.ai[3][3] = 1.0f / 15.0f;
    k.ai[4][1] = bi1; k.ai[4][2] = bi2; k.ai[4][3] = bi3; k.ai[4][4] = bi4;
    k.ae[2][1] = 8.0f / 15.0f;
    k.ae[3][1] = be1; k.ae[3][2] = 5.0f / 12.0f;
    k.ae[4][1] = be1; k.ae[4][2] = be2; k.ae[4][3] = be3; k.ae[4][4] = be4;
  } else {
    k.ai[2][1] = (float)0.353842865099275; k.ai[2][2] = (float)0.353842865099275;
    k.ai[3][1] = (float)0.398930808264689; k.ai[3][2] = (float)0.345755244189622;
    k.ai[3][3] = (float)0.255313947545689;
    k.ae[2][1] = (float)0.711664700366941;
    k.ae[3][1] = (float)0.077338168947683; k.ae[3][2] = (float)0.917273367886007;
  }
  return k;
}

// explicit convection (fact +1) of a stage state into a five-variable block
// Halo sum of a five-variable block [mass][energy][mom x][mom y][mom z].
int halo_block5(sod_gpu_ctx *c, float *out) {
  HaloView v{};
  const long long N = c->npoin;
  v.width = 5;
  v.nstride = 1;
  for (int k = 0; k < 5; ++k) v.comp[k] = out + k * N;
  return halo_sum(c, v);
}

int imex_convec(sod_gpu_ctx *c, const float *rho, const float *u, const float *q, const float *pr, const float *h,
                float *out) {
  RhsArgs A{};
  A.rho = rho; A.u = u; A.q = q; A.pr = pr; A.E = h; A.fact_c = 1.0f;
  dispatch(c, [&](auto L) {
    L.template rhs<MODE_CONV, IN_PRIM>(c, A);
    return 0;
  });
  const long long N = c->npoin;
  gather_res(c, out, out + 2 * N, out + N, 0, 0);
  return halo_block5(c, out);
}

// diffusion without LPS (fact +1) into a five-variable block; rho_n null: rho
int imex_diffusion(sod_gpu_ctx *c, const float *rho_n, const float *rho, const float *u, const float *Tem,
                    float *out) {
  auto &S = c->comp;
  RhsArgs A{};
  A.rho = rho; A.rho_n = rho_n; A.u = u; A.Tem = Tem; A.mu_fluid = S.mu_fluid; A.mue_t = c->mue_t;
  A.musgs_t = nullptr; A.fact_d = 1.0f;
  dispatch(c, [&](auto L) {
    L.template rhs<MODE_DIFF | MODE_NOLPS, IN_DIFF>(c, A);
    return 0;
  });
  const long long N = c->npoin;
  gather_res(c, out, out + 2 * N, out + N, 0, 0);
  return halo_block5(c, out);  // mod_solver_imex.f90:123, :196 (operator); time_integ_imex.f90:382 (stages)
}

// FP64 sum over the working nodes and the five variables of a (b - c)
double imex_dot(sod_gpu_ctx *c, const float *a, const float *b, const float *cc, int *rc) {
  const long long N = c->npoin;
  DotArgs<float, 5> A{};
  for (int k = 0; k < 5; ++k) {
    A.a[k] = a + N * k; A.b[k] = b + N * k; A.c[k] = cc ? cc + N * k : nullptr;
  }
  dots<float, 5>(c, A, c->cg.dots + 8);
  if ((*rc = allreduce(c, c->cg.dots + 8, 5, SOD_REDUCE_SUM_F64))) return 0.0;  // mod_solver_imex.f90:181, 225
  double t[5] = {0, 0, 0, 0, 0};
  if (cudaMemcpyAsync(t, c->cg.dots + 8, 40, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess) {
    *rc = fail(SOD_GPU_ECUDA, "dot product of the IMEX solve failed");
    return 0.0;
  }
  return (((t[0] + t[1]) + t[2]) + t[3]) + t[4];
}

// conjGrad_imex, mod_solver_imex.f90:25-342 (periodic): x0 = the step's
// initial state (X.lvl1), right-hand side the stage state in (rho32, E32,
// q32), which receives the solution on the working nodes.
int imex_cg(sod_gpu_ctx *c, float fact, float dt, int maxIter, double tol) {
  auto &S = c->comp;
  auto &X = c->imex;
  const long long N = c->npoin;
  const int nw = c->npoin_w;
  const unsigned nb = nblk(nw, 256);
  const float gm1 = c->phys.gamma_gas - 1.0f;
  CUDA_TRY(cudaMemcpyAsync(X.x, X.lvl1, 5 * N * 4, cudaMemcpyDeviceToDevice, c->stream));
  CUDA_TRY(cudaMemcpyAsync(X.b, S.rho32, N * 4, cudaMemcpyDeviceToDevice, c->stream));
  CUDA_TRY(cudaMemcpyAsync(X.b + N, S.E32, N * 4, cudaMemcpyDeviceToDevice, c->stream));
  CUDA_TRY(cudaMemcpyAsync(X.b + 2 * N, S.q32, 3 * N * 4, cudaMemcpyDeviceToDevice, c->stream));
  auto apply = [&](const float *v) {  // qn = v Ml + fact dt D(v)
    k_imex_prim<<<nb, 256, 0, c->stream>>>(nw, N, c->lpoin_w, gm1, c->phys.Rgas, X.x, v, X.au, X.aT);
    int arc = imex_diffusion(c, X.x, v, X.au, X.aT, X.qn);
    k_imex_op<<<nb, 256, 0, c->stream>>>(nw, N, c->lpoin_w, c->Ml, v, fact, dt, X.qn);
    return arc;
  };
  int rc = apply(X.x);
  if (rc) return rc;
  k_imex_vec<<<nb, 256, 0, c->stream>>>(0, nw, N, c->lpoin_w, c->Ml, dt, 0.f, 0.f, X.b, X.x, X.r, X.p, X.qn, X.z,
                                        X.z1);
  const double auxB = std::sqrt(imex_dot(c, X.r, X.r, nullptr, &rc));
  if (rc) return rc;
  double nrm = auxB;
  int it;
  for (it = 1; it <= maxIter; ++it) {
    if ((rc = apply(X.p))) return rc;
    const double Q1 = imex_dot(c, X.r, X.z, nullptr, &rc);
    const double Q2 = imex_dot(c, X.p, X.qn, nullptr, &rc);
    if (rc) return rc;
    const float alpha = (float)(Q1 / Q2);
    k_imex_vec<<<nb, 256, 0, c->stream>>>(1, nw, N, c->lpoin_w, c->Ml, dt, alpha, 0.f, X.b, X.x, X.r, X.p, X.qn,
                                          X.z, X.z1);
    nrm = std::sqrt(imex_dot(c, X.r, X.r, nullptr, &rc));
    if (rc) return rc;
    if (!std::isfinite(nrm)) return fail(SOD_GPU_ENONFINITE, "non-finite residual in the IMEX solve");
    if (nrm < tol * auxB) break;
    const double T = imex_dot(c, X.r, X.z, X.z1, &rc);
    if (rc) return rc;
    const float beta = (float)(T / Q1);
    k_imex_vec<<<nb, 256, 0, c->stream>>>(2, nw, N, c->lpoin_w, c->Ml, dt, 0.f, beta, X.b, X.x, X.r, X.p, X.qn,
                                          X.z, X.z1);
  }
  k_imex_out<<<nb, 256, 0, c->stream>>>(nw, N, c->lpoin_w, X.x, S.rho32, S.E32, S.q32);
  X.cg_iters = it > maxIter ? maxIter : it;
  X.cg_res = auxB > 0 ? nrm / auxB : 0.0;
  return 0;
}

}  // namespace

extern "C" {

int sod_gpu_comp_imex_step(sod_gpu_ctx *c, float dt, int maxIter, double tol) {
  if (!c || !c->comp.ready) return fail(SOD_GPU_EINVAL, "state not initialised");
  if (!(dt > 0.f) || maxIter < 1 || !(tol > 0.0)) return fail(SOD_GPU_EINVAL, "bad argument");
  auto &S = c->comp;
  if (S.stages != 3 && S.stages != 4) return fail(SOD_GPU_EINVAL, "the IMEX integrator has 3 or 4 stages");
  if (S.fp64) return fail(SOD_GPU_EINVAL, "the IMEX integrator runs on the FP32 state (fp64_state = 0)");
  int rc;
  if ((rc = ensure_imex(c))) return rc;
  auto &X = c->imex;
  const cudaStream_t st = c->stream;
  const long long N = c->npoin;
  const int nw = c->npoin_w;
  const unsigned nb = nblk(nw, 256);
  const float gm = c->phys.gamma_gas;
  const ImexCoef K = imex_coef(S.stages);
  const bool was_async = c->async;
  c->async = true;
  // level 1 <- level 2 (CFDSolverBase.f90:1951-1960)
  CUDA_TRY(cudaMemcpyAsync(S.u1, S.u2, 3 * N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(S.eta1, S.eta2, N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(X.lvl1, S.rho32, N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(X.lvl1 + N, S.E32, N * 4, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(X.lvl1 + 2 * N, S.q32, 3 * N * 4, cudaMemcpyDeviceToDevice, st));
  const long long B = 5 * N;
  if (S.first) {  // time_integ_imex.f90:240-273
    S.first = false;
    k_feta<<<nb, 256, 0, st>>>(nw, N, c->lpoin_w, S.u1, S.eta1, S.feta);
    k_aux_h<<<nb, 256, 0, st>>>(nw, c->lpoin_w, gm / (gm - 1.0f), S.rho32, S.pr, X.aux_h);
    if ((rc = comp_entropy_pass(c, S.Reta1, false)) || (rc = comp_visc(c, S.Reta1, S.rho32, S.u1, false)) ||
        (rc = imex_convec(c, S.rho32, S.u2, S.q32, S.pr, X.aux_h, X.R)) ||
        (rc = imex_diffusion(c, nullptr, S.rho32, S.u2, S.Tem, X.D))) {
      c->async = was_async;
      return rc;
    }
  } else {  // the last stage's residuals open the step
    CUDA_TRY(cudaMemcpyAsync(X.R, X.R + (S.stages - 1) * B, B * 4, cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(X.D, X.D + (S.stages - 1) * B, B * 4, cudaMemcpyDeviceToDevice, st));
  }
  // LPS stabilisation of the step's initial state (comp_tau, full_proj_ijk,
  // full_stab_ijk with fact -1 = the LPS part of full_diff_stab_ijk with zero
  // viscosities and fact +1)
  k_comp_tau<<<nblk(c->nelem, 8), 256, 0, st>>>(c->nelem, c->N, c->conn, c->helem, S.csound, S.u2, c->npoin,
                                                c->phys.c_species_stab / (float)c->P, S.tau);
  {
    RhsArgs A{};
    A.rho = S.rho32; A.u = S.u2; A.Tem = S.Tem; A.mu_fluid = X.zmu; A.mue_t = X.zmue; A.musgs_t = nullptr;
    A.tau_stab = S.tau; A.proj12 = c->proj12; A.fact_d = 1.0f;
    rc = dispatch(c, [&](auto L) {
      L.proj(c, true, S.rho32, S.u2, S.Tem);
      gather_proj_aos(c);
      int hrc = halo_sum(c, halo_proj_view(c));
      if (hrc) return hrc;
      L.template rhs<MODE_DIFF, IN_DIFF>(c, A);
      return 0;
    });
    if (!rc) {
      gather_res(c, X.stab, X.stab + 2 * N, X.stab + N, 0, 0);
      rc = halo_block5(c, X.stab);
    }
    if (rc) {
      c->async = was_async;
      return rc;
    }
  }
  int iters = 0;
  for (int is = 2; is <= S.stages; ++is) {
    k_imex_comb<<<nblk(N, 256), 256, 0, st>>>(N, is, K, dt, c->Ml, X.R, X.D, X.stab, X.lvl1, S.rho32, S.E32, S.q32);
    if ((rc = imex_cg(c, K.ai[is][is], dt, maxIter, tol))) { c->async = was_async; return rc; }
    iters += X.cg_iters;
    k_eos_end<<<nb, 256, 0, st>>>(nw, N, c->lpoin_w, gm - 1.0f, gm, c->phys.Rgas, S.rho32, S.q32, S.E32, S.u2, S.eint,
                                  S.pr, S.csound, S.machno, S.Tem);
    k_aux_h<<<nb, 256, 0, st>>>(nw, c->lpoin_w, gm / (gm - 1.0f), S.rho32, S.pr, X.aux_h);
    if ((rc = imex_convec(c, S.rho32, S.u2, S.q32, S.pr, X.aux_h, X.R + (is - 1) * B)) ||
        (rc = imex_diffusion(c, nullptr, S.rho32, S.u2, S.Tem, X.D + (is - 1) * B))) {
      c->async = was_async;
      return rc;
    }
  }
  X.cg_iters = iters;
  // entropy viscosity of the new state (time_integ_imex.f90:454-505)
  k_thermo_entropy<<<nb, 256, 0, st>>>(nw, N, c->lpoin_w, gm, c->phys.p_inf, c->phys.rho_inf, S.rho32, S.pr, S.u1,
                                       S.eta1, S.eta2, S.feta);
  if ((rc = comp_entropy_pass(c, S.Reta2, true))) {
    c->async = was_async;
    return rc;
  }
  k_aux_reta<<<nb, 256, 0, st>>>(nw, c->lpoin_w, dt, S.Reta1, S.Reta2, S.eta1, S.eta2, S.aux);
  if ((rc = comp_visc(c, S.aux, S.rho32, S.u2, true))) {
    c->async = was_async;
    return rc;
  }
  k_sutherland<<<nb, 256, 0, st>>>(nw, c->lpoin_w, S.mu_factor, S.Tem, S.mu_fluid);
  c->async = was_async;
  return c->finish();
}

int sod_gpu_comp_imex_stats(sod_gpu_ctx *c, int *cg_iters, double *cg_res) {
  if (!c || !c->comp.ready) return fail(SOD_GPU_EINVAL, "state not initialised");
  if (cg_iters) *cg_iters = c->imex.cg_iters;
  if (cg_res) *cg_res = c->imex.cg_res;
  return 0;
}

int sod_gpu_comp_adapt_dt(sod_gpu_ctx *c, float cfl_conv, float cfl_diff, float *dt) {
  if (!c || !c->comp.ready || !dt) return fail(SOD_GPU_EINVAL, "bad argument");
  auto &S = c->comp;
  const unsigned init_bits = 0x56B5E621u;  // 1e14f
  CUDA_TRY(cudaMemcpyAsync(S.bits + 1, &init_bits, 4, cudaMemcpyHostToDevice, c->stream));
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    k_dt<LL::P_><<<nblk(c->nelem, 8), 256, 0, c->stream>>>(c->md(), c->helem, S.u2, S.csound, S.mu_fluid,
                                                            c->mue_t, S.rho32, cfl_conv, cfl_diff, S.bits + 1);
    return 0;
  });
  int rc = allreduce(c, S.bits + 1, 1, SOD_REDUCE_MIN_F32);
  if (rc) return rc;
  unsigned b = 0;
  CUDA_TRY(cudaMemcpyAsync(&b, S.bits + 1, 4, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  float v;
  std::memcpy(&v, &b, 4);
  *dt = v;
  return 0;
}

int sod_gpu_comp_analysis(sod_gpu_ctx *c, float rho0, double *out) {
  if (!c || !c->comp.ready || !out) return fail(SOD_GPU_EINVAL, "bad argument");
  auto &S = c->comp;
  dispatch(c, [&](auto L) {
    using LL = decltype(L);
    k_analysis_elem<LL::P_, LL::EPB><<<LL::grid(c->nelem), LL::TPB, 0, c->stream>>>(
        c->md(), S.rho32, S.u2, S.mu_fluid, c->mue_t, c->Ngp_t, S.part);
    return 0;
  });
  k_sum_parts<<<1, 1024, 0, c->stream>>>(c->nelem, S.part, S.sums);
  const unsigned zero = 0u;
  CUDA_TRY(cudaMemcpyAsync(S.bits + 2, &zero, 4, cudaMemcpyHostToDevice, c->stream));
  k_max_mach<<<MINMAX_BLOCKS, 256, 0, c->stream>>>(c->npoin_w, c->lpoin_w, S.machno, S.bits + 2);
  int rc;
  if ((rc = allreduce(c, S.sums, 3, SOD_REDUCE_SUM_F64)) || (rc = allreduce(c, S.bits + 2, 1, SOD_REDUCE_MAX_F32)))
    return rc;
  double sums[3];
  unsigned mb = 0;
  CUDA_TRY(cudaMemcpyAsync(sums, S.sums, 24, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaMemcpyAsync(&mb, S.bits + 2, 4, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  const float twopi = 2.0f * 3.14159f;
  double EK = sums[0] / (double)(rho0 * powf(twopi, 3.0f));
  const float alpha = 1.0f / (rho0 * c->volT);
  double eS = sums[1] * (double)alpha;
  double eD = (double)(4.0f / 3.0f) * sums[2] * (double)alpha;
  float mach;
  std::memcpy(&mach, &mb, 4);
  out[0] = (double)(float)EK;
  out[1] = (double)(float)eS;
  out[2] = (double)(float)eD;
  out[3] = (double)(float)(eS + eD);
  out[4] = (double)mach;
  return 0;
}

int sod_gpu_comp_get_state(sod_gpu_ctx *c, float *rho, float *q, float *E, float *mu_e) {
  if (!c || !c->comp.ready) return fail(SOD_GPU_EINVAL, "state not initialised");
  auto &S = c->comp;
  const size_t N = c->npoin;
  if (rho) CUDA_TRY(cudaMemcpyAsync(rho, S.rho32, N * 4, cudaMemcpyDeviceToDevice, c->stream));
  if (q) CUDA_TRY(cudaMemcpyAsync(q, S.q32, 3 * N * 4, cudaMemcpyDeviceToDevice, c->stream));
  if (E) CUDA_TRY(cudaMemcpyAsync(E, S.E32, N * 4, cudaMemcpyDeviceToDevice, c->stream));
  if (mu_e) {
    const long long EN = (long long)c->nelem * c->N;
    k_t_to_elem<<<nblk(EN, 256), 256, 0, c->stream>>>(c->nelem, c->N, c->a_of_t, c->mue_t, mu_e);
  }
  return c->finish();
}

}  // extern "C"
