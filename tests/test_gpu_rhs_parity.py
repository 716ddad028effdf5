"""GPU parity of the RHS operators against the CPU oracle (FP32, same inputs).

Bar (SOD2D RHS hot path): relative L2 error <= 1e-5 per RHS evaluation
against the oracle's FP32 restatement of the reference.  Every call goes
through the C-ABI with device pointers, as a Fortran caller would make it.
Meshes use jittered (curved) elements, a shuffled element order and a
shuffled element-local node numbering to exercise the general path.
"""
import numpy as np
import pytest

import oracle as O
from sod2d_b200 import host

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-5  # relative L2 per RHS evaluation


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def zeros(n):
    return torch.zeros(n, dtype=torch.float32, device="cuda")


@pytest.fixture(scope="module")
def gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_b200 import gpu as g
    return g


def make_case(porder, n, seed=3):
    m = host.periodic_cube(porder, n, jitter=0.05, seed=seed, elem_shuffle=True, ordering=1)
    rho, q, E = host.random_comp_state(m, seed=seed + 1)
    ic = host.tgv_comp_init(m, Ma=0.1)  # gas constants of the Ma=0.1 TGV
    N = m.npoin
    u = (q.reshape(3, N) / rho).astype(np.float32)
    eint = E / rho - 0.5 * (u.astype(np.float64) ** 2).sum(0)
    pr = (rho * (ic.gamma - 1.0) * eint).astype(np.float32)
    csound = np.sqrt(ic.gamma * pr / rho).astype(np.float32)
    return m, ic, rho, q, E, u.reshape(-1), pr, csound


def run_updateF(gpu, ctx, ic, d, N):
    out = dict(Rm=zeros(N), Rq=zeros(3 * N), Re=zeros(N))
    ctx.call("sod_gpu_updateF", gpu.dptr(d["rho"]), gpu.dptr(d["q"]), gpu.dptr(d["E"]), gpu.dptr(d["mu_e"]),
             float(ic.mu_factor), gpu.dptr(d["tau"]), gpu.dptr(out["Rm"]), gpu.dptr(out["Rq"]),
             gpu.dptr(out["Re"]), None, None, None, None)
    return out


@pytest.mark.parametrize("porder,n", [(3, 4), (4, 3)])
def test_updateF_matches_oracle(gpu, porder, n):
    m, ic, rho, q, E, u, pr, csound = make_case(porder, n)
    om = O.OracleMesh(m)
    mu_e = np.random.default_rng(5).uniform(0.0, 2e-3, m.nelem * m.nnode).astype(np.float32)
    tau = O.comp_tau(om, csound, u)
    Rm, Rq, Re = O.rhs(om, O.comp_params(ic), rho, q, E, mu_e, ic.mu_factor, tau)
    ctx = gpu.Context(m, gpu.phys_from_ic(ic))
    N = m.npoin
    d = {k: dev(v) for k, v in dict(rho=rho, q=q, E=E, mu_e=mu_e, tau=tau).items()}
    out = run_updateF(gpu, ctx, ic, d, N)
    g = {k: v.cpu().numpy() for k, v in out.items()}
    for name, a, b in (("mass", g["Rm"], Rm), ("mom", g["Rq"], Rq), ("ener", g["Re"], Re)):
        err = rel_l2(a, b)
        print(f"P={porder} updateF {name}: rel L2 vs FP32 oracle = {err:.3e}")
        assert err < TOL, (name, err)
    out2 = run_updateF(gpu, ctx, ic, d, N)  # deterministic assembly
    for k in out:
        assert torch.equal(out[k], out2[k])
    ctx.close()


def test_convec_op_matches_oracle(gpu):
    m, ic, rho, q, E, u, pr, csound = make_case(3, 4)
    N = m.npoin
    om = O.OracleMesh(m)
    h = (ic.gamma / (ic.gamma - 1.0) * pr / rho).astype(np.float32)
    Rm, Rq, Re = O.convec(om, u, q, rho, pr, h, init=True, fact=-1.0)
    ctx = gpu.Context(m, gpu.phys_from_ic(ic))
    d = {k: dev(v) for k, v in dict(u=u, q=q, rho=rho, pr=pr, h=h).items()}
    g = dict(Rm=zeros(N), Rq=zeros(3 * N), Re=zeros(N))
    ctx.call("sod_gpu_full_convec_ijk", *(gpu.dptr(d[k]) for k in ("u", "q", "rho", "pr", "h")),
             gpu.dptr(g["Rm"]), gpu.dptr(g["Rq"]), gpu.dptr(g["Re"]), 1, -1.0)
    for name, a, b in (("mass", g["Rm"], Rm), ("mom", g["Rq"], Rq), ("ener", g["Re"], Re)):
        err = rel_l2(a.cpu().numpy(), b)
        print(f"convec {name}: rel L2 = {err:.3e}")
        assert err < TOL, (name, err)
    ctx.close()


def test_comp_tau_matches_oracle(gpu):
    m, ic, rho, q, E, u, pr, csound = make_case(3, 4)
    om = O.OracleMesh(m)
    ref = O.comp_tau(om, csound, u)
    ctx = gpu.Context(m, gpu.phys_from_ic(ic))
    out = zeros(m.nelem)
    dc, du = dev(csound), dev(u)  # keep the device buffers alive across the call
    ctx.call("sod_gpu_comp_tau", gpu.dptr(dc), gpu.dptr(du), gpu.dptr(out))
    assert rel_l2(out.cpu().numpy(), ref) < 1e-6
    ctx.close()


def test_op_level_entry_points_compose_to_updateF(gpu):
    """full_convec_ijk + full_proj_ijk + full_diff_stab_ijk + lumped_solver,
    called as updateF calls them (time_integ_ls.f90:605-686), equal the
    oracle's updateF."""
    m, ic, rho, q, E, u, pr, csound = make_case(3, 4, seed=9)
    om = O.OracleMesh(m)
    N = m.npoin
    mu_e = np.random.default_rng(2).uniform(0.0, 2e-3, m.nelem * m.nnode).astype(np.float32)
    tau = O.comp_tau(om, csound, u)
    Rm, Rq, Re, proj = O.rhs(om, O.comp_params(ic), rho, q, E, mu_e, ic.mu_factor, tau, want_proj=True)
    ctx = gpu.Context(m, gpu.phys_from_ic(ic))
    d = {k: dev(v) for k, v in dict(rho=rho, q=q, E=E, mu_e=mu_e, tau=tau).items()}
    prim = dict(u=zeros(3 * N), pr=zeros(N), Tem=zeros(N), mu=zeros(N))
    tmp = dict(Rm=zeros(N), Rq=zeros(3 * N), Re=zeros(N))
    # primitive fields from the library's EOS (updateF's optional outputs)
    ctx.call("sod_gpu_updateF", gpu.dptr(d["rho"]), gpu.dptr(d["q"]), gpu.dptr(d["E"]), gpu.dptr(d["mu_e"]),
             float(ic.mu_factor), gpu.dptr(d["tau"]), gpu.dptr(tmp["Rm"]), gpu.dptr(tmp["Rq"]), gpu.dptr(tmp["Re"]),
             gpu.dptr(prim["u"]), gpu.dptr(prim["pr"]), gpu.dptr(prim["Tem"]), gpu.dptr(prim["mu"]))
    h = (prim["pr"] * float(ic.gamma / (ic.gamma - 1.0)) / d["rho"]).contiguous()
    P5 = [zeros(3 * N) for _ in range(5)]  # ProjMass, ProjEner, ProjMX, ProjMY, ProjMZ
    ctx.call("sod_gpu_full_proj_ijk", gpu.dptr(d["rho"]), gpu.dptr(prim["u"]), gpu.dptr(prim["Tem"]),
             *(gpu.dptr(x) for x in P5))
    w = m.lpoin_w - 1
    refP = proj.reshape(5, 3, N)
    for k in range(5):
        err = rel_l2(P5[k].cpu().numpy().reshape(3, N)[:, w], refP[k][:, w])
        print("proj", k, err)
        assert err < TOL
    R = dict(Rm=zeros(N), Rq=zeros(3 * N), Re=zeros(N))
    ctx.call("sod_gpu_full_convec_ijk", gpu.dptr(prim["u"]), gpu.dptr(d["q"]), gpu.dptr(d["rho"]),
             gpu.dptr(prim["pr"]), gpu.dptr(h), gpu.dptr(R["Rm"]), gpu.dptr(R["Rq"]), gpu.dptr(R["Re"]), 1, -1.0)
    ctx.call("sod_gpu_full_diff_stab_ijk", float(ic.Cp), float(ic.Prt), gpu.dptr(d["rho"]), gpu.dptr(d["rho"]),
             gpu.dptr(prim["u"]), gpu.dptr(prim["Tem"]), gpu.dptr(prim["mu"]), gpu.dptr(d["mu_e"]), None,
             *(gpu.dptr(x) for x in P5), gpu.dptr(d["tau"]), gpu.dptr(R["Rm"]), gpu.dptr(R["Rq"]),
             gpu.dptr(R["Re"]), 0, -1.0)
    for k, nc in (("Rm", 1), ("Re", 1), ("Rq", 3)):
        ctx.call("sod_gpu_lumped_solver", gpu.dptr(R[k]), nc)
    for name, a, b in (("mass", R["Rm"], Rm), ("mom", R["Rq"], Rq), ("ener", R["Re"], Re)):
        err = rel_l2(a.cpu().numpy(), b)
        print(f"composed {name}: rel L2 = {err:.3e}")
        assert err < TOL, (name, err)
    ctx.close()


@pytest.mark.parametrize("porder", [3, 4])
def test_plain_diffusion_without_lps(gpu, porder):
    """full_convec_ijk + full_diffusion_ijk (the flag_lps_stab = .false. path
    of updateF, time_integ_ls.f90:621-626) + lumped_solver equal the oracle's
    updateF with LPS off."""
    m, ic, rho, q, E, u, pr, csound = make_case(porder, 4, seed=13)
    om = O.OracleMesh(m)
    N = m.npoin
    mu_e = np.random.default_rng(5).uniform(0.0, 2e-3, m.nelem * m.nnode).astype(np.float32)
    tau = O.comp_tau(om, csound, u)
    Rm, Rq, Re = O.rhs(om, O.comp_params(ic, lps=False), rho, q, E, mu_e, ic.mu_factor, tau)
    ctx = gpu.Context(m, gpu.phys_from_ic(ic))
    d = {k: dev(v) for k, v in dict(rho=rho, q=q, E=E, mu_e=mu_e, tau=tau).items()}
    prim = dict(u=zeros(3 * N), pr=zeros(N), Tem=zeros(N), mu=zeros(N))
    tmp = dict(Rm=zeros(N), Rq=zeros(3 * N), Re=zeros(N))
    ctx.call("sod_gpu_updateF", gpu.dptr(d["rho"]), gpu.dptr(d["q"]), gpu.dptr(d["E"]), gpu.dptr(d["mu_e"]),
             float(ic.mu_factor), gpu.dptr(d["tau"]), gpu.dptr(tmp["Rm"]), gpu.dptr(tmp["Rq"]), gpu.dptr(tmp["Re"]),
             gpu.dptr(prim["u"]), gpu.dptr(prim["pr"]), gpu.dptr(prim["Tem"]), gpu.dptr(prim["mu"]))
    h = (prim["pr"] * float(ic.gamma / (ic.gamma - 1.0)) / d["rho"]).contiguous()
    R = dict(Rm=zeros(N), Rq=zeros(3 * N), Re=zeros(N))
    ctx.call("sod_gpu_full_convec_ijk", gpu.dptr(prim["u"]), gpu.dptr(d["q"]), gpu.dptr(d["rho"]),
             gpu.dptr(prim["pr"]), gpu.dptr(h), gpu.dptr(R["Rm"]), gpu.dptr(R["Rq"]), gpu.dptr(R["Re"]), 1, -1.0)
    ctx.call("sod_gpu_full_diffusion_ijk", float(ic.Cp), float(ic.Prt), gpu.dptr(d["rho"]), gpu.dptr(d["rho"]),
             gpu.dptr(prim["u"]), gpu.dptr(prim["Tem"]), gpu.dptr(prim["mu"]), gpu.dptr(d["mu_e"]), None,
             gpu.dptr(R["Rm"]), gpu.dptr(R["Rq"]), gpu.dptr(R["Re"]), 0, -1.0)
    for k, nc in (("Rm", 1), ("Re", 1), ("Rq", 3)):
        ctx.call("sod_gpu_lumped_solver", gpu.dptr(R[k]), nc)
    for name, a, b in (("mass", R["Rm"], Rm), ("mom", R["Rq"], Rq), ("ener", R["Re"], Re)):
        err = rel_l2(a.cpu().numpy(), b)
        print(f"no-LPS {name}: rel L2 = {err:.3e}")
        assert err < TOL, (name, err)
    ctx.close()
