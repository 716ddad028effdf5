"""CPU checks of the numpy restatement of the learned preconditioner: the
analytic energy-norm gradient matches central finite differences, the map is
symmetric, it is exactly Jacobi with zero patch modes and zero skip
exponent, and the patch table holds each element's face-neighbour layers."""
import numpy as np

import oracle as O
import precond_ref as PR
from sod2d_b200 import host


def setup_case(seed=4, n=3):
    m = host.periodic_cube(3, n, jitter=0.05, seed=seed, ordering=1, elem_shuffle=True)
    om = O.OracleMesh(m, np.float64)
    diag = O.laplacian_diag(O.OracleMesh(m))
    net = PR.Net(m, diag)
    lap = lambda v: O.laplacian(om, v)
    rng = np.random.default_rng(seed)
    params = rng.normal(0, 0.1, PR.num_params(3))
    w = m.lpoin_w - 1
    e = np.zeros(m.npoin)
    e[w] = rng.normal(size=w.size)
    r = lap(e)
    return m, net, lap, params, r, e, diag


def test_gradient_matches_finite_differences():
    m, net, lap, params, r, e, _ = setup_case()
    loss, grad = net.loss_grad(params, r, e, lap)
    rng = np.random.default_rng(1)
    off = PR.dims(3)[2]
    idx = list(rng.choice(params.size, 12, replace=False)) + [off["alpha"][0], off["b3"][0], off["W1T"][0]]
    h = 1e-6
    for i in idx:
        p1, p2 = params.copy(), params.copy()
        p1[i] += h
        p2[i] -= h
        fd = (net.loss_grad(p1, r, e, lap)[0] - net.loss_grad(p2, r, e, lap)[0]) / (2 * h)
        assert abs(fd - grad[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, grad[i])


def test_map_is_symmetric_positive():
    m, net, lap, params, r, e, _ = setup_case()
    w = m.lpoin_w - 1
    rng = np.random.default_rng(2)
    a, b = np.zeros(m.npoin), np.zeros(m.npoin)
    a[w], b[w] = rng.normal(size=w.size), rng.normal(size=w.size)
    ab = a[w] @ net.forward(params, b)[0][w]
    ba = b[w] @ net.forward(params, a)[0][w]
    assert abs(ab - ba) <= 1e-10 * abs(ab)
    assert a[w] @ net.forward(params, a)[0][w] > 0


def test_zero_modes_is_jacobi():
    m, net, lap, params, r, e, diag = setup_case()
    off = PR.dims(3)[2]
    p = params.copy()
    p[off["B"][0]:off["B"][0] + off["B"][1]] = 0.0
    p[off["alpha"][0]] = 0.0
    z, _ = net.forward(p, r)
    w = m.lpoin_w - 1
    np.testing.assert_allclose(z[w], r[w] / diag[w].astype(np.float64), rtol=1e-12, atol=1e-14)


def test_patch_layers_are_face_neighbour_nodes():
    m, net, *_ = setup_case(n=3)
    P, n1 = 3, 4
    N = n1 ** 3
    conn, pt = net.conn, net.pt
    # every layer node belongs to the neighbour across that face and not to the element itself
    for e in range(m.nelem):
        own = set(conn[e])
        for f in range(6):
            e2 = net.nbr[e, f]
            layer = pt[e, N + f * n1 * n1:N + (f + 1) * n1 * n1]
            assert (layer >= 0).all()
            assert set(layer).issubset(set(conn[e2]))
            assert not (set(layer) & own)
    # each node appears in a fixed number of patches on a periodic cube: its own elements plus the layers
    cnt = np.bincount(pt.ravel(), minlength=m.npoin)[m.lpoin_w - 1]
    assert cnt.min() >= 4 and cnt.max() <= 8
