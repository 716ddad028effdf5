"""The known-answer properties of tests/test_oracle_kat.py on the GPU,
through the C-ABI: zero RHS of a uniform state (sod_gpu_updateF),
telescoping residual sums on an affine mesh, and the exact gradient of
x^P (sod_gpu_eval_gradient)."""
import numpy as np
import pytest

from sod2d_b200 import host
from test_oracle_kat import polynomial_gradient_error, uniform_state

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_b200 import gpu as g
    return g


def gpu_rhs(gpu, m, ic, rho, q, E, mu_e):
    N = m.npoin
    ctx = gpu.Context(m, gpu.phys_from_ic(ic))
    dv = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    u = (q.reshape(3, N) / rho).astype(np.float32).reshape(-1)
    d = [dv(a) for a in (rho, q, E, mu_e, u, np.full(N, 2.0, np.float32))]
    tau = torch.zeros(m.nelem, device="cuda")
    ctx.call("sod_gpu_comp_tau", gpu.dptr(d[5]), gpu.dptr(d[4]), gpu.dptr(tau))
    out = [torch.zeros(k * N, device="cuda") for k in (1, 3, 1)]
    ctx.call("sod_gpu_updateF", *(gpu.dptr(x) for x in d[:4]), float(ic.mu_factor), gpu.dptr(tau),
             *(gpu.dptr(x) for x in out), None, None, None, None)
    res = [x.cpu().numpy() for x in out]
    ctx.close()
    return res


@pytest.mark.parametrize("porder", [3, 4])
def test_uniform_flow_has_zero_rhs(gpu, porder):
    m = host.periodic_cube(porder, 3, jitter=0.05, seed=81, elem_shuffle=True, ordering=1)
    ic = host.tgv_comp_init(m, Ma=0.5)
    mu_e = np.full(m.nelem * m.nnode, 1e-3, np.float32)
    R0 = gpu_rhs(gpu, m, ic, *uniform_state(m, ic)[:3], mu_e)
    Rr = gpu_rhs(gpu, m, ic, *host.random_comp_state(m, seed=82), mu_e)
    w = m.lpoin_w - 1
    for r0, rr, k in zip(R0, Rr, (1, 3, 1)):
        r0 = r0.reshape(k, -1)[:, w]
        rr = rr.reshape(k, -1)[:, w]
        assert np.abs(r0).max() <= 1e-6 * np.abs(rr).max()


@pytest.mark.parametrize("porder", [3, 4])
def test_residuals_telescope_on_affine_mesh(gpu, porder):
    m = host.periodic_cube(porder, 3, jitter=0.0, seed=83, elem_shuffle=True, ordering=1)
    ic = host.tgv_comp_init(m, Ma=0.5)
    mu_e = np.random.default_rng(84).uniform(0, 1e-3, m.nelem * m.nnode).astype(np.float32)
    R = gpu_rhs(gpu, m, ic, *host.random_comp_state(m, seed=85), mu_e)
    w = m.lpoin_w - 1
    Ml = m.Ml.astype(np.float64)[w]
    for r, k in zip(R, (1, 3, 1)):
        r = r.astype(np.float64).reshape(k, -1)[:, w]
        ratio = np.abs((r * Ml).sum(axis=1)) / (np.abs(r) * Ml).sum(axis=1)
        assert np.all(ratio < 2e-6), ratio


@pytest.mark.parametrize("porder", [3, 4])
def test_gradient_of_degree_p_polynomial_is_exact(gpu, porder):
    m = host.periodic_cube(porder, 4, jitter=0.0, seed=86, elem_shuffle=True, ordering=1)
    ctx = gpu.Context(m, gpu.default_phys())

    def grad(f):
        x = torch.from_numpy(f).cuda()
        g = torch.zeros(3 * m.npoin, device="cuda")
        ctx.call("sod_gpu_eval_gradient", gpu.dptr(x), gpu.dptr(g))
        return g.cpu().numpy()

    err, cross = polynomial_gradient_error(m, grad)
    ctx.close()
    assert err < 2e-6 and cross < 2e-6, (err, cross)
