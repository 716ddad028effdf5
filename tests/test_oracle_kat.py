"""Known-answer properties of the discretisation, checked on the oracle
(CPU).  tests/test_gpu_kat.py checks the same properties through the C-ABI.

- GLL nodes and weights of order 3 and 4 against their closed forms
  (ZELEGL / WELEGL, src/lib_sod2d/sources/mod_maths.f90:41-106).
- A uniform state (constant rho, u, p; constant mu_e) has a zero RHS on a
  jittered, shuffled periodic mesh: every term is a derivative of a
  constant or a product with one.
- On an affine periodic mesh the lumped-mass-weighted sums of the mass,
  energy and momentum residuals vanish for any state: the split-form
  convection and the weak-form diffusion telescope between elements.
- The gradient operator differentiates x^P exactly on affine elements of
  order P (collocation at the GLL points), on every working node away from
  the periodic seam.
"""
import numpy as np
import pytest

import oracle as O
from sod2d_b200 import host

CLOSED = {
    3: ([-1.0, -1 / np.sqrt(5), 1 / np.sqrt(5), 1.0], [1 / 6, 5 / 6, 5 / 6, 1 / 6]),
    4: ([-1.0, -np.sqrt(3 / 7), 0.0, np.sqrt(3 / 7), 1.0], [1 / 10, 49 / 90, 32 / 45, 49 / 90, 1 / 10]),
}


@pytest.mark.parametrize("porder", [3, 4])
def test_gll_closed_form(porder):
    x, w = host.gll(porder)
    xe, we = CLOSED[porder]
    assert np.allclose(x, xe, rtol=0, atol=1e-14)
    assert np.allclose(w, we, rtol=0, atol=1e-14)
    assert abs(w.sum() - 2.0) < 1e-14


def uniform_state(m, ic, rho0=1.2, u=(0.3, -0.2, 0.1), p0=5.0):
    N = m.npoin
    u = np.asarray(u, np.float32)
    rho = np.full(N, rho0, np.float32)
    q = (np.repeat(u, N) * np.float32(rho0)).astype(np.float32)
    E = np.full(N, p0 / (ic.gamma - 1) + 0.5 * rho0 * float((u.astype(np.float64) ** 2).sum()), np.float32)
    return rho, q, E, np.repeat(u, N).astype(np.float32)


def rhs_of(m, ic, rho, q, E, mu_e):
    N = m.npoin
    om = O.OracleMesh(m)
    u = (q.reshape(3, N) / rho).astype(np.float32).reshape(-1)
    tau = O.comp_tau(om, np.full(N, 2.0, np.float32), u)
    return O.rhs(om, O.comp_params(ic), rho, q, E, mu_e, ic.mu_factor, tau)


@pytest.mark.parametrize("porder", [3, 4])
def test_uniform_flow_has_zero_rhs(porder):
    m = host.periodic_cube(porder, 3, jitter=0.05, seed=81, elem_shuffle=True, ordering=1)
    ic = host.tgv_comp_init(m, Ma=0.5)
    mu_e = np.full(m.nelem * m.nnode, 1e-3, np.float32)
    R0 = rhs_of(m, ic, *uniform_state(m, ic)[:3], mu_e)
    Rr = rhs_of(m, ic, *host.random_comp_state(m, seed=82), mu_e)
    w = m.lpoin_w - 1
    for r0, rr, k in zip(R0, Rr, (1, 3, 1)):
        r0 = np.asarray(r0).reshape(k, -1)[:, w]
        rr = np.asarray(rr).reshape(k, -1)[:, w]
        assert np.abs(r0).max() <= 1e-6 * np.abs(rr).max()


@pytest.mark.parametrize("porder", [3, 4])
def test_residuals_telescope_on_affine_mesh(porder):
    m = host.periodic_cube(porder, 3, jitter=0.0, seed=83, elem_shuffle=True, ordering=1)
    ic = host.tgv_comp_init(m, Ma=0.5)
    mu_e = np.random.default_rng(84).uniform(0, 1e-3, m.nelem * m.nnode).astype(np.float32)
    R = rhs_of(m, ic, *host.random_comp_state(m, seed=85), mu_e)
    w = m.lpoin_w - 1
    Ml = m.Ml.astype(np.float64)[w]
    for r, k in zip(R, (1, 3, 1)):
        r = np.asarray(r, np.float64).reshape(k, -1)[:, w]
        ratio = np.abs((r * Ml).sum(axis=1)) / (np.abs(r) * Ml).sum(axis=1)
        assert np.all(ratio < 2e-6), ratio


def polynomial_gradient_error(m, grad_fn):
    """max relative error of d/dx_d x_d^P over working nodes away from the
    periodic seam, and the largest cross-derivative, over d = 0, 1, 2."""
    N, P = m.npoin, m.porder
    xyz = m.coord.reshape(3, -1).astype(np.float64)
    L = float(m.extra["L"])
    h = L / m.extra["nx"]
    work = np.zeros(N, bool)
    work[m.lpoin_w - 1] = True
    err = cross = 0.0
    for d in range(3):
        x = xyz[d]
        g = np.asarray(grad_fn((x ** P).astype(np.float32)), np.float64).reshape(3, N)
        exact = P * x ** (P - 1)
        inner = work & (x > h + 1e-4) & (x < L - h - 1e-4)
        scale = np.abs(exact[inner]).max()
        err = max(err, np.abs(g[d][inner] - exact[inner]).max() / scale)
        cross = max(cross, np.abs(np.delete(g, d, axis=0)[:, inner]).max() / scale)
    return err, cross


@pytest.mark.parametrize("porder", [3, 4])
def test_gradient_of_degree_p_polynomial_is_exact(porder):
    m = host.periodic_cube(porder, 4, jitter=0.0, seed=86, elem_shuffle=True, ordering=1)
    om = O.OracleMesh(m)
    err, cross = polynomial_gradient_error(m, lambda f: O.gradient(om, f))
    assert err < 2e-6 and cross < 2e-6, (err, cross)
