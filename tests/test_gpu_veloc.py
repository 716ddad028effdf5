"""Implicit velocity solve of the incompressible step on the GPU against the
oracle: species_tau, the LPS projection of the velocity gradient
(eval_tau_veloc), the stabilised viscous operator (full_diff_stab_incomp)
and the preconditioned CG (conjGrad_veloc_incomp), P=3 and P=4, jittered
and shuffled meshes, the reference's FP32 arithmetic."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from sod2d_b200 import host

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.fixture(scope="module")
def gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_b200 import gpu as g
    return g


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def case(porder, seed=11):
    m = host.periodic_cube(porder, 4, jitter=0.05, seed=seed, elem_shuffle=True, ordering=1)
    N = m.npoin
    x, y, z = (m.coord[i * N:(i + 1) * N].astype(np.float64) for i in range(3))
    rng = np.random.default_rng(seed)
    u = np.concatenate([np.sin(x) * np.cos(y) * np.cos(z), -np.cos(x) * np.sin(y) * np.cos(z),
                        0.1 * np.sin(z)]) + 0.02 * rng.normal(size=3 * N)
    mu = np.full(N, 1.0 / 1600.0)
    musgs = rng.uniform(0, 1e-4, m.nelem * m.nnode)
    return m, u.astype(np.float32), mu.astype(np.float32), musgs.astype(np.float32)


@pytest.mark.parametrize("porder", [3, 4])
def test_operators_match_oracle(gpu, porder):
    m, u, mu, musgs = case(porder)
    om = O.OracleMesh(m)
    N = m.npoin
    w = m.lpoin_w - 1
    ctx = gpu.Context(m, gpu.default_phys())
    dv = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    du, dmu, dsgs = dv(u), dv(mu), dv(musgs)
    tau = torch.zeros(m.nelem, device="cuda")
    ctx.call("sod_gpu_species_tau", gpu.dptr(du), gpu.dptr(tau))
    tref = O.species_tau(om, u)
    assert np.abs(tau.cpu().numpy() - tref).max() <= 1e-6 * np.abs(tref).max()
    G = [torch.zeros(3 * N, device="cuda") for _ in range(3)]
    ctx.call("sod_gpu_eval_tau_veloc", gpu.dptr(du), *(gpu.dptr(g) for g in G))
    Gref = O.eval_tau_veloc(om, u)
    for g, r in zip(G, Gref):
        err = rel_l2(g.cpu().numpy().reshape(3, N)[:, w], r.reshape(3, N)[:, w])
        print("tau_veloc", err)
        assert err < TOL
    Rm = torch.zeros(3 * N, device="cuda")
    ctx.call("sod_gpu_full_diff_stab_incomp", gpu.dptr(du), gpu.dptr(dmu), gpu.dptr(dsgs), *(gpu.dptr(g) for g in G),
             gpu.dptr(tau), gpu.dptr(Rm))
    Rref = O.full_diff_stab_incomp(om, u, mu, musgs, np.concatenate(Gref), tref)
    err = rel_l2(Rm.cpu().numpy().reshape(3, N)[:, w], Rref.reshape(3, N)[:, w])
    print("diff_stab_incomp", err)
    assert err < TOL
    ctx.close()


@pytest.mark.parametrize("porder", [3, 4])
def test_velocity_cg_matches_oracle(gpu, porder):
    m, u, mu, musgs = case(porder, seed=12)
    om = O.OracleMesh(m)
    N = m.npoin
    w = m.lpoin_w - 1
    dt, fact = 0.01, 1.0 / (11.0 / 6.0)
    # right-hand side as the BDF/EXT3 step builds it: (u** - dt grad p / gamma0) * Ml
    rng = np.random.default_rng(13)
    ustar = u + 0.01 * rng.normal(size=3 * N).astype(np.float32)
    b = (ustar.reshape(3, N) * m.Ml.astype(np.float32)).reshape(-1).astype(np.float32)
    for maxIter, tol in ((20, 1e-2), (50, 1e-6)):
        xr, itr, rr = O.cg_veloc(om, fact, dt, mu, musgs, u, b, maxIter=maxIter, tol=tol)
        ctx = gpu.Context(m, gpu.default_phys())
        dv = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        R = dv(b).clone()
        dmu, dsgs, du = dv(mu), dv(musgs), dv(u)  # keep the device copies alive across the call
        its, res = C.c_int(), C.c_double()
        ctx.call("sod_gpu_conjgrad_veloc", float(fact), float(dt), gpu.dptr(dmu), gpu.dptr(dsgs), gpu.dptr(du),
                 gpu.dptr(R), maxIter, tol, C.byref(its), C.byref(res))
        x = R.cpu().numpy()
        err = rel_l2(x.reshape(3, N)[:, w], xr.reshape(3, N)[:, w])
        print(f"tol {tol}: iterations gpu {its.value} oracle {itr}, residual {res.value:.3e} / {rr:.3e}, rel L2 {err:.2e}")
        assert abs(its.value - itr) <= 1
        assert res.value < tol or its.value == maxIter
        assert err < TOL
        ctx.close()
