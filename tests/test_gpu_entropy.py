"""The entropy-viscosity pieces as individual C-ABI calls against the
oracle: generic_scalar_convec_ijk (with initialze and fact),
smart_visc_spectral_imex and ducros_visc_limit, P=3 and P=4, jittered and
shuffled meshes, a random compressible state."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from sod2d_b200 import host

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_b200 import gpu as g
    return g


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


@pytest.mark.parametrize("porder", [3, 4])
def test_entropy_pieces_match_oracle(gpu, porder):
    m = host.periodic_cube(porder, 4, jitter=0.05, seed=31, elem_shuffle=True, ordering=1)
    ic = host.tgv_comp_init(m, Ma=0.5)
    rho, q, E = host.random_comp_state(m, seed=32)
    N = m.npoin
    w = m.lpoin_w - 1
    u = (q.reshape(3, N) / rho).astype(np.float32)
    eint = E / rho - 0.5 * (u.astype(np.float64) ** 2).sum(0)
    csound = np.sqrt(ic.gamma * rho * (ic.gamma - 1.0) * eint / rho).astype(np.float32)
    u = u.reshape(-1)
    rng = np.random.default_rng(33)
    eta = rng.uniform(0.5, 1.5, N).astype(np.float32)
    feta = (u.reshape(3, N) * eta).astype(np.float32).reshape(-1)
    om = O.OracleMesh(m)
    ctx = gpu.Context(m, gpu.phys_from_ic(ic))
    dv = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    d = {k: dv(v) for k, v in dict(rho=rho, u=u, csound=csound, eta=eta, feta=feta).items()}

    # generic_scalar_convec_ijk: zeroed and scaled, then accumulated
    R = torch.zeros(N, device="cuda")
    ctx.call("sod_gpu_generic_scalar_convec_ijk", gpu.dptr(d["feta"]), gpu.dptr(d["eta"]), gpu.dptr(d["u"]),
             gpu.dptr(R), 1, -1.0)
    ref = O.scalar_convec(om, feta, eta, u, init=True, fact=-1.0)
    err = rel_l2(R.cpu().numpy()[w], ref[w])
    print("scalar convection", err)
    assert err < 1e-5
    R0 = rng.normal(size=N).astype(np.float32)
    R = dv(R0)
    ctx.call("sod_gpu_generic_scalar_convec_ijk", gpu.dptr(d["feta"]), gpu.dptr(d["eta"]), gpu.dptr(d["u"]),
             gpu.dptr(R), 0, 0.5)
    ref = O.scalar_convec(om, feta, eta, u, R=R0, init=False, fact=0.5)
    assert rel_l2(R.cpu().numpy()[w], ref[w]) < 1e-5

    # smart_visc_spectral_imex on the lumped residual
    Reta = (O.scalar_convec(om, feta, eta, u) * m.invMl).astype(np.float32)
    dR = dv(Reta)
    mu = torch.zeros(m.nelem * m.nnode, device="cuda")
    ctx.call("sod_gpu_smart_visc_spectral_imex", gpu.dptr(dR), gpu.dptr(d["rho"]), gpu.dptr(d["u"]),
             gpu.dptr(d["csound"]), gpu.dptr(mu))
    mu_ref = O.smart_visc(om, Reta, rho, u, csound)
    err = rel_l2(mu.cpu().numpy(), mu_ref)
    print("smart viscosity", err)
    assert err < 1e-5

    # ducros_visc_limit on the oracle's mu_e
    divU = O.divergence(om, u)
    vort = O.vorticity(om, u)
    dmu = dv(mu_ref)
    ddiv, dvort = dv(divU), dv(vort)
    ctx.call("sod_gpu_ducros_visc_limit", gpu.dptr(d["rho"]), gpu.dptr(d["u"]), gpu.dptr(ddiv), gpu.dptr(dvort),
             gpu.dptr(d["csound"]), gpu.dptr(dmu))
    lim_ref = O.ducros(om, rho, u, divU, vort, csound, mu_ref)
    err = rel_l2(dmu.cpu().numpy(), lim_ref)
    print("Ducros limit", err)
    assert err < 1e-5
    assert not np.allclose(lim_ref, mu_ref)  # the limiter acted
    ctx.close()


def test_rk_ls_stage_bitwise(gpu):
    """The stage update of rk_4_ls_main as its own call: bit-identical to the
    FP32 arithmetic of time_integ_ls.f90:325-329 (first stage) and :352-356
    (later stages) on the working nodes; other nodes untouched."""
    m = host.periodic_cube(3, 3, seed=41)
    N = m.npoin
    w = m.lpoin_w - 1
    rng = np.random.default_rng(42)
    f32 = np.float32
    U1 = [rng.normal(size=k * N).astype(f32) for k in (1, 3, 1)]
    U2 = [rng.normal(size=k * N).astype(f32) for k in (1, 3, 1)]
    R = [rng.normal(size=k * N).astype(f32) for k in (1, 3, 1)]
    lam1, lami, gam, dt = f32(0.571403511494104), f32(0.428596488505896), f32(0.110577759392786), f32(3.7e-3)
    ctx = gpu.Context(m, gpu.default_phys())
    dv = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    gdt = gam * dt
    W3 = np.concatenate([w + N * d for d in range(3)])
    for first in (1, 0):
        d1, d2, dr = [dv(a) for a in U1], [dv(a) for a in U2], [dv(a) for a in R]
        ctx.call("sod_gpu_rk_ls_stage", first, float(lam1), float(lami), float(gam), float(dt),
                 *(gpu.dptr(x) for x in d1), *(gpu.dptr(x) for x in d2), *(gpu.dptr(x) for x in dr))
        for k, idx in ((0, w), (1, W3), (2, w)):
            got = d2[k].cpu().numpy()
            if first:
                exp = U2[k][idx] + gdt * R[k][idx]
            else:
                exp = (lam1 * U1[k][idx] + lami * U2[k][idx]) + gdt * R[k][idx]
            assert np.array_equal(got[idx].view(np.uint32), exp.astype(f32).view(np.uint32))
            other = np.setdiff1d(np.arange(got.size), idx)
            assert np.array_equal(got[other], U2[k][other])
    ctx.close()
