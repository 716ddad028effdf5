"""ORACLE -- test infrastructure only.

ctypes binding of ``_build/liboracle.so``, the CPU restatement of the SOD2D
reference arithmetic (``oracle_ops.hpp``).  Imported only by tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg, as the reference
arithmetic the CUDA results are compared with.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_lib = None


def build(force: bool = False) -> Path:
    out = HERE / "_build" / "liboracle.so"
    if force or not out.exists() or any(
            (HERE / s).stat().st_mtime > out.stat().st_mtime for s in ("oracle_capi.cpp", "oracle_ops.hpp")):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return out


class MeshT(C.Structure):
    _fields_ = [("porder", C.c_int), ("nelem", C.c_int), ("npoin", C.c_int), ("npoin_w", C.c_int),
                ("connec", C.c_void_p), ("lpoin_w", C.c_void_p), ("invAtoIJK", C.c_void_p),
                ("gmshAtoI", C.c_void_p), ("gmshAtoJ", C.c_void_p), ("gmshAtoK", C.c_void_p),
                ("lelpn", C.c_void_p), ("atoIJK", C.c_void_p),
                ("He", C.c_void_p), ("gpvol", C.c_void_p), ("dlxigp_ip", C.c_void_p), ("dNgp", C.c_void_p),
                ("Ngp", C.c_void_p), ("Ml", C.c_void_p), ("invMl", C.c_void_p), ("helem", C.c_void_p),
                ("helem_l", C.c_void_p), ("volT", C.c_double)]


class CompParams(C.Structure):
    _fields_ = [("gamma", C.c_double), ("Rgas", C.c_double), ("Cp", C.c_double), ("Prt", C.c_double),
                ("rho_inf", C.c_double), ("p_inf", C.c_double), ("cfl_conv", C.c_double),
                ("cfl_diff", C.c_double), ("maxPhysTime", C.c_double), ("stages", C.c_int),
                ("rk_n", C.c_int), ("lps", C.c_int), ("log_first", C.c_int), ("log_step", C.c_int),
                ("first_mue", C.c_int), ("imex", C.c_int), ("imex_maxiter", C.c_int), ("imex_tol", C.c_double)]


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        _lib = C.CDLL(str(build()))
        for s in ("f32", "f64"):
            for name in ("tgv_comp_run", "rhs", "entropy_visc", "elem_jacobian", "convec", "comp_tau",
                         "dt", "analysis"):
                f = getattr(_lib, f"oracle_{name}_{s}")
                f.restype = C.c_int
            getattr(_lib, f"oracle_tgv_comp_run_{s}").argtypes = [
                C.POINTER(MeshT), C.POINTER(CompParams), C.c_void_p, C.c_double, C.c_int, C.c_void_p,
                C.c_int, C.POINTER(C.c_int), C.c_void_p]
            getattr(_lib, f"oracle_rhs_{s}").argtypes = [C.POINTER(MeshT), C.POINTER(CompParams)] + [C.c_void_p] * 10
            getattr(_lib, f"oracle_entropy_visc_{s}").argtypes = (
                [C.POINTER(MeshT), C.POINTER(CompParams)] + [C.c_void_p] * 8 + [C.c_double] + [C.c_void_p] * 3)
            getattr(_lib, f"oracle_elem_jacobian_{s}").argtypes = [C.c_int] * 3 + [C.c_void_p] * 6
            getattr(_lib, f"oracle_convec_{s}").argtypes = [C.POINTER(MeshT)] + [C.c_void_p] * 8 + [C.c_int, C.c_double]
            getattr(_lib, f"oracle_comp_tau_{s}").argtypes = [C.POINTER(MeshT)] + [C.c_void_p] * 3
            getattr(_lib, f"oracle_dt_{s}").argtypes = ([C.POINTER(MeshT)] + [C.c_void_p] * 2 + [C.c_double] * 2 +
                                                        [C.c_void_p] * 5)
            getattr(_lib, f"oracle_first_mue_{s}").argtypes = [C.POINTER(MeshT)] + [C.c_void_p] * 6
            getattr(_lib, f"oracle_first_mue_{s}").restype = C.c_int
            for nm, na in (("laplacian", 2), ("laplacian_diag", 1), ("gradient", 2), ("divergence", 2),
                           ("convec_incomp", 3)):
                getattr(_lib, f"oracle_{nm}_{s}").argtypes = [C.POINTER(MeshT)] + [C.c_void_p] * na
                getattr(_lib, f"oracle_{nm}_{s}").restype = C.c_int
            getattr(_lib, f"oracle_cg_pressure_{s}").argtypes = ([C.POINTER(MeshT)] + [C.c_void_p] * 3 +
                                                                 [C.c_int, C.c_double, C.c_void_p, C.c_void_p])
            getattr(_lib, f"oracle_cg_pressure_{s}").restype = C.c_int
            getattr(_lib, f"oracle_analysis_{s}").argtypes = ([C.POINTER(MeshT), C.c_double] + [C.c_void_p] * 5)
            real = C.c_float if s == "f32" else C.c_double
            for nm, na in (("species_tau", 2), ("eval_tau_veloc", 2), ("full_diff_stab_incomp", 6)):
                getattr(_lib, f"oracle_{nm}_{s}").argtypes = [C.POINTER(MeshT)] + [C.c_void_p] * na
                getattr(_lib, f"oracle_{nm}_{s}").restype = C.c_int
            getattr(_lib, f"oracle_cg_veloc_{s}").argtypes = ([C.POINTER(MeshT), real, real] + [C.c_void_p] * 4 +
                                                              [C.c_int, C.c_double, C.c_void_p])
            getattr(_lib, f"oracle_cg_veloc_{s}").restype = C.c_int
            getattr(_lib, f"oracle_scalar_convec_{s}").argtypes = ([C.POINTER(MeshT)] + [C.c_void_p] * 4 +
                                                                   [C.c_int, C.c_double])
            for nm, na in (("smart_visc", 5), ("ducros", 6), ("vorticity", 2)):
                getattr(_lib, f"oracle_{nm}_{s}").argtypes = [C.POINTER(MeshT)] + [C.c_void_p] * na
            for nm in ("scalar_convec", "smart_visc", "ducros", "vorticity"):
                getattr(_lib, f"oracle_{nm}_{s}").restype = C.c_int
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class OracleMesh:
    """Holds the oracle's view of a host.Mesh in precision ``dtype``."""

    def __init__(self, mesh, dtype=np.float32, geometry64=None):
        self.mesh = mesh
        self.dtype = np.dtype(dtype)
        self.suffix = "f32" if self.dtype == np.float32 else "f64"
        cast = lambda a: np.ascontiguousarray(a, dtype=self.dtype)
        geo = dict(He=mesh.He, gpvol=mesh.gpvol, dlxigp_ip=mesh.dlxigp_ip, dNgp=mesh.dNgp, Ngp=mesh.Ngp,
                   Ml=mesh.Ml, invMl=mesh.invMl, helem=mesh.helem, helem_l=mesh.helem_l)
        if geometry64 is not None:
            geo.update(geometry64)
        self.arr = {k: cast(v) for k, v in geo.items()}
        self.ints = {k: np.ascontiguousarray(getattr(mesh, k), np.int32)
                     for k in ("connecWork", "lpoin_w", "invAtoIJK", "gmshAtoI", "gmshAtoJ", "gmshAtoK",
                               "lelpn", "atoIJK")}
        self.volT = float(self.dtype.type(mesh.vol_total if geometry64 is None else geometry64.get(
            "vol_total", mesh.vol_total)))
        self.s = MeshT(mesh.porder, mesh.nelem, mesh.npoin, mesh.npoin_w,
                       _p(self.ints["connecWork"]), _p(self.ints["lpoin_w"]), _p(self.ints["invAtoIJK"]),
                       _p(self.ints["gmshAtoI"]), _p(self.ints["gmshAtoJ"]), _p(self.ints["gmshAtoK"]),
                       _p(self.ints["lelpn"]), _p(self.ints["atoIJK"]),
                       *(_p(self.arr[k]) for k in ("He", "gpvol", "dlxigp_ip", "dNgp", "Ngp", "Ml", "invMl",
                                                   "helem", "helem_l")), self.volT)

    def fn(self, name):
        return getattr(lib(), f"oracle_{name}_{self.suffix}")


def comp_params(ic, cfl_conv=0.5, cfl_diff=0.5, stages=5, rk_n=1, lps=True, maxPhysTime=0.0,
                log_first=1, log_step=10, first_mue=True, imex=False, imex_maxiter=200,
                imex_tol=1e-3) -> CompParams:
    """imex: the IMEX integrator (imex_main) with `stages` = 3 or 4 and the
    implicit solve's maxIter / tol (TGVCompSolver.f90:90-93 defaults)."""
    return CompParams(ic.gamma, ic.Rgas, ic.Cp, ic.Prt, ic.rho0, ic.P0, cfl_conv, cfl_diff, maxPhysTime,
                      stages, rk_n, int(lps), log_first, log_step, int(first_mue), int(imex), imex_maxiter,
                      imex_tol)


def tgv_comp_run(om: OracleMesh, ic, prm: CompParams, nsteps: int, max_rows: int = 4096):
    """Run the compressible TGV time loop; returns (history[rows,6], final)
    where history columns are time, EK, eps_S, eps_D, eps_T, max Mach and
    final = dict(rho, q, E, mu_e)."""
    N, n = om.mesh.npoin, om.mesh.nnode
    dt = om.dtype
    init = np.concatenate([ic.rho, ic.u, ic.q, ic.pr, ic.E, ic.Tem, ic.e_int, ic.csound, ic.machno,
                           ic.eta]).astype(dt)
    hist = np.zeros((max_rows, 6))
    nrows = C.c_int()
    final = np.zeros(5 * N + om.mesh.nelem * n, dt)
    rc = om.fn("tgv_comp_run")(C.byref(om.s), C.byref(prm), _p(init), ic.mu_factor, nsteps, _p(hist),
                               max_rows, C.byref(nrows), _p(final))
    if rc:
        raise RuntimeError(f"oracle tgv run failed {rc}")
    out = dict(rho=final[:N], q=final[N:4 * N], E=final[4 * N:5 * N], mu_e=final[5 * N:])
    return hist[: nrows.value], out


def rhs(om: OracleMesh, prm: CompParams, rho, q, E, mu_e, mu_factor, tau_stab, want_proj=False):
    """One RHS evaluation (updateF body).  Returns Rmass, Rmom(N*3), Rener
    (and the 15 mass-inverted projections if want_proj)."""
    N = om.mesh.npoin
    dt = om.dtype
    c = lambda a: np.ascontiguousarray(a, dt)
    Rm, Rq, Re = np.zeros(N, dt), np.zeros(3 * N, dt), np.zeros(N, dt)
    proj = np.zeros(15 * N, dt) if want_proj else None
    mf = np.full(N, mu_factor, dt) if np.isscalar(mu_factor) else c(mu_factor)
    rc = om.fn("rhs")(C.byref(om.s), C.byref(prm), _p(c(rho)), _p(c(q)), _p(c(E)), _p(c(mu_e)), _p(mf),
                      _p(c(tau_stab)), _p(Rm), _p(Rq), _p(Re), _p(proj))
    if rc:
        raise RuntimeError("oracle rhs failed")
    return (Rm, Rq, Re, proj) if want_proj else (Rm, Rq, Re)


def convec(om: OracleMesh, u, q, rho, pr, E, init=True, fact=-1.0, R=None):
    """full_convec_ijk on the oracle (returns Rmass, Rmom(N*3), Rener)."""
    N = om.mesh.npoin
    c = lambda a: np.ascontiguousarray(a, om.dtype)
    Rm, Rq, Re = (np.zeros(N, om.dtype), np.zeros(3 * N, om.dtype), np.zeros(N, om.dtype)) if R is None else R
    om.fn("convec")(C.byref(om.s), _p(c(u)), _p(c(q)), _p(c(rho)), _p(c(pr)), _p(c(E)), _p(Rm), _p(Rq), _p(Re),
                    int(init), float(fact))
    return Rm, Rq, Re


def _op(om, name, ncomp_out, *inputs):
    c = lambda a: np.ascontiguousarray(a, om.dtype)
    out = np.zeros(ncomp_out * om.mesh.npoin, om.dtype)
    keep = [c(a) for a in inputs]
    om.fn(name)(C.byref(om.s), *(_p(a) for a in keep), _p(out))
    return out


def laplacian(om, p):
    """eval_laplacian_mult (assembled, not mass-inverted)."""
    return _op(om, "laplacian", 1, p)


def laplacian_diag(om):
    return _op(om, "laplacian_diag", 1)


def gradient(om, x):
    """eval_gradient with lumped inversion: (N,3)."""
    return _op(om, "gradient", 3, x)


def divergence(om, u):
    """eval_divergence (assembled int N div u)."""
    return _op(om, "divergence", 1, u)


def convec_incomp(om, u, q):
    return _op(om, "convec_incomp", 3, u, q)


def cg_pressure(om, diag, x0, rhs, maxIter=20, tol=1e-2):
    """conjGrad_pressure_incomp: returns (x0 + x, iterations, ||r||/||b||)."""
    c = lambda a: np.ascontiguousarray(a, om.dtype)
    out = np.zeros(om.mesh.npoin, om.dtype)
    res = C.c_double()
    keep = [c(diag), c(x0), c(rhs)]
    it = om.fn("cg_pressure")(C.byref(om.s), *(_p(a) for a in keep), maxIter, tol, _p(out), C.byref(res))
    return out, it, res.value


def species_tau(om, u):
    """species_tau: element stabilisation time tau (nelem,) from u (N,3)."""
    c = lambda a: np.ascontiguousarray(a, om.dtype)
    out = np.zeros(om.mesh.nelem, om.dtype)
    keep = c(u)
    om.fn("species_tau")(C.byref(om.s), _p(keep), _p(out))
    return out


def eval_tau_veloc(om, u):
    """eval_tau_veloc: (GradX, GradY, GradZ), each (N,3) flattened, mass-inverted."""
    out = _op(om, "eval_tau_veloc", 9, u)
    N = om.mesh.npoin
    return out[:3 * N], out[3 * N:6 * N], out[6 * N:]


def full_diff_stab_incomp(om, u, mu_fluid, mu_sgs, tauP, tau_stab):
    """full_diff_stab_incomp: Rmom (N,3) flattened; tauP = GradX|GradY|GradZ."""
    c = lambda a: np.ascontiguousarray(a, om.dtype)
    out = np.zeros(3 * om.mesh.npoin, om.dtype)
    keep = [c(u), c(mu_fluid), c(mu_sgs), c(tauP), c(tau_stab)]
    om.fn("full_diff_stab_incomp")(C.byref(om.s), *(_p(a) for a in keep), _p(out))
    return out


def cg_veloc(om, fact, dt, mu_fluid, mu_sgs, Rp0, b, maxIter=20, tol=1e-2):
    """conjGrad_veloc_incomp (LPS path): returns (x, iterations, ||r||/||r0||)."""
    c = lambda a: np.ascontiguousarray(a, om.dtype)
    rio = c(b).copy()
    res = C.c_double()
    keep = [c(mu_fluid), c(mu_sgs), c(Rp0)]
    it = om.fn("cg_veloc")(C.byref(om.s), float(fact), float(dt), *(_p(a) for a in keep), _p(rio), maxIter, tol,
                           C.byref(res))
    return rio, it, res.value


def _pressure_fp64(om64, b, x0, tol=1e-11, maxIter=5000):
    """Jacobi-preconditioned CG in FP64 on the assembled Laplacian over the
    working nodes.  The periodic system is singular (constants) and, with
    single-precision geometry, its rows sum to ~1e-8 instead of 0, so the
    right-hand side and every residual are projected to zero mean; without
    that the iterate drifts along the near-constant null vector once the
    residual reaches the inconsistency floor (~1e-10)."""
    w = om64.mesh.lpoin_w - 1
    A = lambda v: laplacian(om64, v)
    d = laplacian_diag(om64)
    b = np.asarray(b, np.float64).copy()
    b[w] -= b[w].mean()
    x = np.asarray(x0, np.float64).copy()
    r = np.zeros_like(b)
    r[w] = (b - A(x))[w]
    r[w] -= r[w].mean()
    z = np.zeros_like(b)
    z[w] = r[w] / d[w]
    p = z.copy()
    rz = float(r[w] @ z[w])
    bn = float(np.linalg.norm(b[w]))
    for _ in range(maxIter):
        if np.linalg.norm(r[w]) <= tol * bn:
            break
        q = A(p)
        a = rz / float(p[w] @ q[w])
        x[w] += a * p[w]
        r[w] -= a * q[w]
        r[w] -= r[w].mean()
        z[w] = r[w] / d[w]
        rz_new = float(r[w] @ z[w])
        p[w] = z[w] + (rz_new / rz) * p[w]
        rz = rz_new
    return x


class IncompState:
    """Time levels of bdfext3_main_incomp: u(:,:,1..4), Rmom(:,:,1..3), pr."""

    def __init__(self, u0):
        u0 = np.asarray(u0, np.float32)
        self.u1, self.u3, self.u4 = u0.copy(), u0.copy(), u0.copy()
        self.Rm1 = np.zeros_like(u0)
        self.Rm3 = np.zeros_like(u0)
        self.p = np.zeros(u0.size // 3)
        self.iltime = 1


def bdfext3_step(om, om64, st: IncompState, dt, nu, maxIter=20, tol=1e-4, pressure="fp64", p_maxIter=20,
                 p_tol=1e-2, diag=None):
    """One bdfext3_main_incomp step (periodic mesh, no wall model, source term
    or LES; rho = 1, mu_fluid = nu), time_integ_incomp.f90:88-433, composed
    of the oracle operators above.  pressure="fp64": the pressure system is
    solved in FP64 to a 1e-11 residual; pressure="reference": the FP32
    right-hand side -gamma0 div(u)/dt and conjGrad_pressure_incomp with
    p_maxIter / p_tol from the previous pressure (diag: its Jacobi
    diagonal), as the reference runs.  Updates st in place and returns the
    velocity solve's (iterations, ||r||/||r0||)."""
    N = om.mesh.npoin
    w = om.mesh.lpoin_w - 1
    f32 = np.float32
    it = st.iltime
    if it == 1:
        g0, a, b = 1.0, (1.0, 0.0, 0.0), (1.0, 0.0, 0.0)
    elif it == 2:
        g0, a, b = 1.5, (2.0, -0.5, 0.0), (2.0, -1.0, 0.0)
    else:
        g0, a, b = 11.0 / 6.0, (3.0, -1.5, 1.0 / 3.0), (3.0, -3.0, 1.0)
    g0, a, b = f32(g0), [f32(v) for v in a], [f32(v) for v in b]
    dt = f32(dt)
    Rm2 = convec_incomp(om, st.u1, st.u1)
    Ml = np.tile(np.asarray(om.mesh.Ml, f32), 3)
    W = np.concatenate([w + N * d for d in range(3)])
    u2 = np.zeros(3 * N, f32)
    e = b[0] * Rm2[W] + b[1] * st.Rm1[W] + b[2] * st.Rm3[W]
    u2[W] = (dt * (-e) / Ml[W] + a[0] * st.u1[W] + a[1] * st.u3[W] + a[2] * st.u4[W]) / g0
    st.Rm3, st.Rm1 = st.Rm1, Rm2
    if pressure == "reference":
        rhs = (f32(-g0) * divergence(om, u2)) / dt
        p, _, _ = cg_pressure(om, diag, np.asarray(st.p, f32), rhs.astype(f32), maxIter=p_maxIter, tol=p_tol)
    else:
        rhs = -np.float64(g0) * divergence(om, u2).astype(np.float64) / np.float64(dt)
        p = _pressure_fp64(om64, rhs, st.p)
    gp = gradient(om, p.astype(f32))
    u2[W] = (u2[W] - dt * gp[W] / g0) * Ml[W]
    mu = np.full(N, nu, f32)
    musgs = np.zeros(om.mesh.nelem * om.mesh.nnode, f32)
    u2, vit, vres = cg_veloc(om, 1.0 / g0, dt, mu, musgs, st.u1, u2, maxIter=maxIter, tol=tol)
    st.u4, st.u3, st.u1 = st.u3, st.u1, u2
    st.p = p
    st.iltime += 1
    return vit, vres


def adapt_dt(om, u, csound, cfl_conv, cfl_diff=1e30, mu_fluid=None, mu_sgs=None, mu_e=None, rho=None):
    """adapt_dt_cfl, mod_time_ops.f90:7-48; without viscosities (the
    incompressible solvers' call) only the convective limit acts."""
    N, EN = om.mesh.npoin, om.mesh.nelem * om.mesh.nnode
    c = lambda a, n: np.ascontiguousarray(np.zeros(n) if a is None else a, om.dtype)
    keep = [c(u, 3 * N), c(csound, N), c(mu_fluid, N), c(mu_sgs, EN), c(mu_e, EN),
            c(np.ones(N) if rho is None else rho, N)]
    out = C.c_double()
    om.fn("dt")(C.byref(om.s), _p(keep[0]), _p(keep[1]), float(cfl_conv), float(cfl_diff), _p(keep[2]), _p(keep[3]),
                _p(keep[4]), _p(keep[5]), C.byref(out))
    return om.dtype.type(out.value)


def analysis(om, rho0, rho, u, mu_fluid, mu_e=None):
    """volAvg_EK and visc_dissipationRate, mod_analysis.f90:10-144:
    (EK, eps_S, eps_D, eps_T)."""
    N, EN = om.mesh.npoin, om.mesh.nelem * om.mesh.nnode
    c = lambda a, n: np.ascontiguousarray(np.zeros(n) if a is None else a, om.dtype)
    keep = [c(rho, N), c(u, 3 * N), c(mu_fluid, N), c(mu_e, EN)]
    out = np.zeros(4)
    om.fn("analysis")(C.byref(om.s), float(rho0), *(_p(a) for a in keep), _p(out))
    return out


def tgv_incomp_run(om, nsteps, Re=1600.0, cfl_conv=0.5, maxIter=20, tol=1e-2, log_first=1, log_step=10,
                   max_time=None):
    """Incompressible Taylor-Green time loop as the reference runs it
    (TGVSolverIncomp.f90:103-174 initial state, CFDSolverPeriodicIncomp
    evalDt :119-128 (convective CFL, zero sound speed), bdfext3_main_incomp
    with conjGrad_pressure_incomp and conjGrad_veloc_incomp sharing maxIter
    / tol): rows (time, EK, eps_S, eps_D, eps_T, 0) at t = 0, after step
    log_first and every log_step steps."""
    f32 = np.float32
    m = om.mesh
    N = m.npoin
    X = m.coord.reshape(3, N).astype(f32)
    x, y, z = X
    u0 = np.concatenate([np.sin(x) * np.cos(y) * np.cos(z), -np.cos(x) * np.sin(y) * np.cos(z),
                         np.zeros(N, f32)]).astype(f32)
    p0 = (f32(1.0 / 16.0) * (np.cos(f32(2) * x) + np.cos(f32(2) * y)) * (np.cos(f32(2) * z) + f32(2))).astype(f32)
    nu = f32(1.0) / f32(Re)
    mu = np.full(N, nu, f32)
    rho = np.ones(N, f32)
    st = IncompState(u0)
    st.p = p0
    diag = laplacian_diag(om)
    zero = np.zeros(N, f32)

    def row(t):
        a = analysis(om, 1.0, rho, st.u1, mu)
        return [float(t), a[0], a[1], a[2], a[3], 0.0]

    t = f32(0.0)
    hist = [row(t)]
    dt = adapt_dt(om, st.u1, zero, cfl_conv)
    log_next = log_first
    for istep in range(1, nsteps + 1):
        bdfext3_step(om, None, st, dt, nu, maxIter=maxIter, tol=tol, pressure="reference", p_maxIter=maxIter,
                     p_tol=tol, diag=diag)
        t = f32(t + dt)
        if istep == log_next:
            hist.append(row(t))
            log_next += log_step
        dt = adapt_dt(om, st.u1, zero, cfl_conv)
        if max_time is not None and t >= f32(max_time):
            break
    return np.array(hist), st


def scalar_convec(om, q, eta, u, R=None, init=True, fact=1.0):
    """generic_scalar_convec_ijk, elem_convec.f90:472-594 (not mass-inverted)."""
    c = lambda a: np.ascontiguousarray(a, om.dtype)
    out = np.zeros(om.mesh.npoin, om.dtype) if R is None else c(R).copy()
    keep = [c(q), c(eta), c(u)]
    om.fn("scalar_convec")(C.byref(om.s), *(_p(a) for a in keep), _p(out), int(init), float(fact))
    return out


def smart_visc(om, Reta, rho, u, csound):
    """smart_visc_spectral_imex, mod_entropy_viscosity.f90:113-227: mu_e (nelem*ngaus)."""
    c = lambda a: np.ascontiguousarray(a, om.dtype)
    out = np.zeros(om.mesh.nelem * om.mesh.nnode, om.dtype)
    keep = [c(Reta), c(rho), c(u), c(csound)]
    om.fn("smart_visc")(C.byref(om.s), *(_p(a) for a in keep), _p(out))
    return out


def ducros(om, rho, u, divU, vorti, csound, mu_e):
    """ducros_visc_limit, mod_entropy_viscosity.f90:277-314: limited copy of mu_e."""
    c = lambda a: np.ascontiguousarray(a, om.dtype)
    out = c(mu_e).copy()
    keep = [c(rho), c(u), c(divU), c(vorti), c(csound)]
    om.fn("ducros")(C.byref(om.s), *(_p(a) for a in keep), _p(out))
    return out


def vorticity(om, u):
    """compute_vorticity with the per-node averaging, mod_operators.f90:684-775."""
    return _op(om, "vorticity", 3, u)


def comp_tau(om: OracleMesh, csound, u):
    out = np.zeros(om.mesh.nelem, om.dtype)
    om.fn("comp_tau")(C.byref(om.s), _p(np.ascontiguousarray(csound, om.dtype)),
                      _p(np.ascontiguousarray(u, om.dtype)), _p(out))
    return out


def first_mue(om: OracleMesh, rho1, u1, eta1, csound):
    """First-step entropy viscosity and lumped entropy residual."""
    c = lambda a: np.ascontiguousarray(a, om.dtype)
    mu_e = np.zeros(om.mesh.nelem * om.mesh.nnode, om.dtype)
    Reta = np.zeros(om.mesh.npoin, om.dtype)
    om.fn("first_mue")(C.byref(om.s), _p(c(rho1)), _p(c(u1)), _p(c(eta1)), _p(c(csound)), _p(mu_e), _p(Reta))
    return mu_e, Reta


def elem_jacobian(porder, nelem, npoin, connec, coord, dNgp, wgp, dtype=np.float64):
    dt = np.dtype(dtype)
    n = (porder + 1) ** 3
    gpvol = np.zeros(n * nelem, dt)
    He = np.zeros(9 * n * nelem, dt)
    s = "f32" if dt == np.float32 else "f64"
    c = lambda a: np.ascontiguousarray(a, dt)
    rc = getattr(lib(), f"oracle_elem_jacobian_{s}")(porder, nelem, npoin, _p(np.ascontiguousarray(connec, np.int32)),
                                                    _p(c(coord)), _p(c(dNgp)), _p(c(wgp)), _p(gpvol), _p(He))
    if rc:
        raise RuntimeError("oracle elem_jacobian failed")
    return gpvol, He


def load_history(path) -> np.ndarray:
    return np.loadtxt(path, ndmin=2)


_HALO_CB = {np.float32: C.CFUNCTYPE(None, C.c_void_p, C.POINTER(C.POINTER(C.c_float)), C.c_int, C.c_longlong),
            np.float64: C.CFUNCTYPE(None, C.c_void_p, C.POINTER(C.POINTER(C.c_double)), C.c_int, C.c_longlong)}
_halo_keep = {}


def set_halo(fn, dtype=np.float32):
    """Install fn(list of ncomp numpy views of npoin values) at the oracle's
    halo points (the reference's mpi_halo_atomic_update_* calls inside
    full_proj_ijk and updateF); None removes it."""
    dt = np.dtype(dtype).type
    suffix = "f32" if dt is np.float32 else "f64"
    setter = getattr(lib(), f"oracle_set_halo_{suffix}")
    if fn is None:
        setter(None, None)
        _halo_keep.pop(suffix, None)
        return

    def cb(user, comp, ncomp, npoin):
        fn([np.ctypeslib.as_array(comp[k], shape=(npoin,)) for k in range(ncomp)])

    c = _HALO_CB[dt](cb)
    _halo_keep[suffix] = c
    setter(c, None)


def halo_exchange_add(plan, comps, transport):
    """The reference's halo sum on one rank (mod_comms.f90:467-627 around
    the transport): fill_sendBuffer_arrays_real packs node i of
    nodesToComm, array k at (i-1)*W + k; the transport exchanges the
    neighbour ranges; copy_from_rcvBuffer_arrays_real adds the received
    values to the local ones, entry by entry in nodesToComm order."""
    import torch
    W = len(comps)
    nodes = plan.nodesToComm.astype(np.int64) - 1
    send = np.zeros(nodes.size * W, comps[0].dtype)
    for k, a in enumerate(comps):
        send[k::W] = a[nodes]
    recv = np.zeros_like(send)
    transport.exchange(plan, torch.from_numpy(send), torch.from_numpy(recv), W)
    for i, p in enumerate(nodes):
        for k, a in enumerate(comps):
            a[p] = a[p] + recv[i * W + k]


_REDUCE_CB = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(C.c_double), C.c_int, C.c_int)


def set_reduce(fn):
    """Install fn(values: float64 numpy view, kind) at the oracle's global
    reductions (the reference's MPI_Allreduce calls: kind 0 min, 1 max,
    2 sum, in place); None removes it."""
    setter = lib().oracle_set_reduce
    if fn is None:
        setter(None, None)
        _halo_keep.pop("reduce", None)
        return
    c = _REDUCE_CB(lambda user, vals, count, kind: fn(np.ctypeslib.as_array(vals, shape=(count,)), kind))
    _halo_keep["reduce"] = c
    setter(c, None)
