"""CPU checks of the numpy restatement of the learned preconditioner: the
analytic energy-norm gradient matches central finite differences, and the
network with a zero output layer is exactly Jacobi."""
import numpy as np

import oracle as O
import precond_ref as PR
from sod2d_b200 import host


def setup_case(seed=4):
    m = host.periodic_cube(3, 3, jitter=0.05, seed=seed, ordering=1)
    om = O.OracleMesh(m, np.float64)
    diag = O.laplacian_diag(O.OracleMesh(m))
    w = m.lpoin_w - 1
    Minv = np.zeros(m.npoin)
    Minv[w] = 1.0 / diag[w].astype(np.float64)
    net = PR.Net(m, Minv)
    lap = lambda v: O.laplacian(om, v)
    rng = np.random.default_rng(seed)
    n = (m.nnode + 6) * 32 + 32 + 32 * 32 + 32 + 32 * m.nnode + m.nnode
    params = rng.normal(0, 0.2, n)
    e = np.zeros(m.npoin)
    e[w] = rng.normal(size=w.size)
    r = lap(e)
    return m, net, lap, params, r, e


def test_gradient_matches_finite_differences():
    m, net, lap, params, r, e = setup_case()
    loss, grad = net.loss_grad(params, r, e, lap)
    rng = np.random.default_rng(1)
    idx = rng.choice(params.size, 12, replace=False)
    h = 1e-6
    for i in idx:
        p1, p2 = params.copy(), params.copy()
        p1[i] += h
        p2[i] -= h
        fd = (net.loss_grad(p1, r, e, lap)[0] - net.loss_grad(p2, r, e, lap)[0]) / (2 * h)
        assert abs(fd - grad[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, grad[i])


def test_zero_output_layer_is_jacobi():
    m, net, lap, params, r, e = setup_case()
    N = m.nnode
    p = params.copy()
    p[-(32 * N + N):] = 0.0
    z, _ = net.forward(p, r)
    w = m.lpoin_w - 1
    np.testing.assert_allclose(z[w], (r * net.Minv)[w], rtol=1e-12, atol=1e-14)
