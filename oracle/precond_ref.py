"""ORACLE -- test infrastructure only.

numpy (FP64) restatement of the learned element-patch preconditioner of the
GPU library: patch table, element geometry features, forward map, energy-norm
loss ||e - M r||_A^2 / ||e||_A^2 and its analytic gradient.  tests/ use it
to check the GPU inference, forward and backward kernels.

The preconditioner (no reference counterpart; it replaces nothing in SOD2D
and sits beside the reference's Jacobi preconditioner of
``conjGrad_pressure_incomp``, mod_solver_incomp.f90:253-506):

    u   = D^-1/2 r                        (D = eval_laplacian_diag)
    x_e = u on the patch of element e     (own nodes + the first node layer
                                           of the 6 face neighbours)
    h_e = B x_e                           (K modes; B is K x NP, shared)
    s_e = softplus(MLP(f_e))              (K positive gains from 8 geometry
                                           features, MLP 8 -> 32 -> 32 -> K)
    z   = D^-1/2 ( exp(alpha) u + sum_e P_e^T B^T diag(s_e) B P_e u )

M is linear in r and symmetric positive definite for any parameters, so it
is a valid conjugate-gradient preconditioner; with B = 0 and alpha = 0 it is
exactly Jacobi.

Element-local node order is the tensor order t = i + n1 j + n1^2 k (natural
GLL order).  Faces are ordered (i=0, i=P, j=0, j=P, k=0, k=P); the layer of
face f (normal direction d, tangential directions d1 < d2) is ordered
a + n1 b with a along d1 and b along d2 of the element's own frame.  Patch
slot j < N is own node t = j; slot N + f n1^2 + a + n1 b is layer node (f, a, b).
"""
from __future__ import annotations

import numpy as np

H = 32   # hidden width of the gain MLP
K = 32   # number of patch modes
F = 8    # geometry features per element


def dims(P):
    n1 = P + 1
    N = n1 ** 3
    NP = N + 6 * n1 * n1
    off = {}
    o = 0
    for name, size in (("B", K * NP), ("alpha", 1), ("W1T", F * H), ("b1", H), ("W2T", H * H), ("b2", H),
                       ("W3T", H * K), ("b3", K)):
        off[name] = (o, size)
        o += size
    return N, NP, off, o


def num_params(P):
    return dims(P)[3]


def unpack(params, P):
    N, NP, off, _ = dims(P)
    g = lambda k: params[off[k][0]:off[k][0] + off[k][1]]
    return (g("B").reshape(K, NP), g("alpha")[0], g("W1T").reshape(F, H), g("b1"), g("W2T").reshape(H, H), g("b2"),
            g("W3T").reshape(H, K), g("b3"))


def nat(porder, ii):
    return 0 if ii == 0 else (porder if ii == 1 else ii - 1)


def tensor_conn(mesh):
    """(E, N) 0-based node ids in tensor order from the reference layout."""
    P, E, N = mesh.porder, mesh.nelem, mesh.nnode
    n1 = P + 1
    cw = mesh.connecWork.reshape(N, E).T - 1  # [e, a]
    t_of_a = np.array([nat(P, mesh.gmshAtoI[a] - 1) + n1 * (nat(P, mesh.gmshAtoJ[a] - 1) +
                                                            n1 * nat(P, mesh.gmshAtoK[a] - 1)) for a in range(N)])
    conn = np.empty((E, N), np.int64)
    conn[:, t_of_a] = cw
    return conn


def _face_ijk(P, f, a, b):
    d, v = f // 2, (P if f % 2 else 0)
    ijk = [0, 0, 0]
    d1, d2 = [x for x in range(3) if x != d]
    ijk[d], ijk[d1], ijk[d2] = v, a, b
    return ijk


def face_neighbours(P, conn):
    """(E, 6) element across each face (the element itself on a boundary)."""
    E = conn.shape[0]
    n1 = P + 1
    tid = lambda ijk: ijk[0] + n1 * (ijk[1] + n1 * ijk[2])
    faces = {}
    for e in range(E):
        for f in range(6):
            key = tuple(sorted(conn[e, tid(_face_ijk(P, f, a, b))] for a in (0, P) for b in (0, P)))
            faces.setdefault(key, []).append((e, f))
    nbr = np.repeat(np.arange(E)[:, None], 6, axis=1)
    for v in faces.values():
        if len(v) == 2:
            (e0, f0), (e1, f1) = v
            nbr[e0, f0] = e1
            nbr[e1, f1] = e0
    return nbr


def patch_table(P, conn, nbr):
    """(E, NP) node ids of each element's patch, -1 where a face has no
    neighbour."""
    E, N = conn.shape
    n1 = P + 1
    NP = N + 6 * n1 * n1
    tid = lambda ijk: ijk[0] + n1 * (ijk[1] + n1 * ijk[2])
    pt = -np.ones((E, NP), np.int64)
    pt[:, :N] = conn
    for e in range(E):
        for f in range(6):
            e2 = nbr[e, f]
            if e2 == e:
                continue
            loc = {int(g): t for t, g in enumerate(conn[e2])}
            corners = [loc[int(conn[e, tid(_face_ijk(P, f, a, b))])] for a in (0, P) for b in (0, P)]
            cijk = np.array([[t % n1, (t // n1) % n1, t // (n1 * n1)] for t in corners])
            d2 = [d for d in range(3) if np.all(cijk[:, d] == cijk[0, d])]
            assert len(d2) == 1
            d2 = d2[0]
            step = 1 if cijk[0, d2] == 0 else -1
            for b in range(n1):
                for a in range(n1):
                    t2 = loc[int(conn[e, tid(_face_ijk(P, f, a, b))])]
                    ijk2 = [t2 % n1, (t2 // n1) % n1, t2 // (n1 * n1)]
                    ijk2[d2] += step
                    pt[e, N + f * n1 * n1 + a + n1 * b] = conn[e2, tid(ijk2)]
    return pt


def elem_features(mesh):
    """(E, 8) features: log of the normalised diagonal of the mean reference
    metric G = He^T He (3), its correlations (3), log element volume and
    log(tr G vol^(2/3)); the last two relative to their mesh mean."""
    E, N = mesh.nelem, mesh.nnode
    He = mesh.He.astype(np.float64).reshape(E, N, 3, 3)  # [e, a, j, i] = He(i, j) = dxi_j / dx_i
    G = np.einsum("eaji,eaki->ejk", He, He) / N          # G_jk = sum_i dxi_j/dx_i dxi_k/dx_i
    vol = mesh.gpvol.astype(np.float64).reshape(E, N).sum(1)
    tr = G[:, 0, 0] + G[:, 1, 1] + G[:, 2, 2]
    f = np.zeros((E, F))
    for b in range(3):
        f[:, b] = np.log(3.0 * G[:, b, b] / tr)
    f[:, 3] = G[:, 0, 1] / np.sqrt(G[:, 0, 0] * G[:, 1, 1])
    f[:, 4] = G[:, 0, 2] / np.sqrt(G[:, 0, 0] * G[:, 2, 2])
    f[:, 5] = G[:, 1, 2] / np.sqrt(G[:, 1, 1] * G[:, 2, 2])
    lv = np.log(vol)
    lm = np.log(tr) + (2.0 / 3.0) * lv
    f[:, 6] = lv - lv.mean()
    f[:, 7] = lm - lm.mean()
    return f


def softplus(o):
    return np.logaddexp(0.0, o)


def sigmoid(o):
    return 1.0 / (1.0 + np.exp(-o))


class Net:
    def __init__(self, mesh, diag):
        """diag: Jacobi diagonal at the nodes (eval_laplacian_diag)."""
        P = mesh.porder
        self.P = P
        self.mesh = mesh
        self.conn = tensor_conn(mesh)
        self.nbr = face_neighbours(P, self.conn)
        self.pt = patch_table(P, self.conn, self.nbr)
        self.ptx = np.where(self.pt >= 0, self.pt, mesh.npoin)
        self.feat = elem_features(mesh)
        self.w = mesh.lpoin_w - 1
        self.Dh = np.zeros(mesh.npoin)
        self.Dh[self.w] = 1.0 / np.sqrt(np.asarray(diag, np.float64)[self.w])

    def _ext(self, v):
        out = np.zeros(self.mesh.npoin + 1)
        out[self.w] = v[self.w]
        return out

    def gains(self, params):
        B, alpha, W1T, b1, W2T, b2, W3T, b3 = unpack(params, self.P)
        h1 = np.tanh(self.feat @ W1T + b1)
        h2 = np.tanh(h1 @ W2T + b2)
        o = h2 @ W3T + b3
        return softplus(o), (h1, h2, o)

    def forward(self, params, r):
        B, alpha = unpack(params, self.P)[:2]
        S, _ = self.gains(params)
        u = self._ext(self.Dh * r)
        X = u[self.ptx]
        Hm = X @ B.T
        O = (S * Hm) @ B
        acc = np.zeros(self.mesh.npoin + 1)
        np.add.at(acc, self.ptx.ravel(), O.ravel())
        z = np.zeros(self.mesh.npoin)
        z[self.w] = self.Dh[self.w] * (np.exp(alpha) * u[self.w] + acc[self.w])
        return z, (u, X, Hm, S)

    def loss_grad(self, params, r, e, lap):
        """lap(v) -> A v (FP64).  Returns loss, gradient (float64)."""
        w = self.w
        B, alpha, W1T, b1, W2T, b2, W3T, b3 = unpack(params, self.P)
        z, (u, X, Hm, S) = self.forward(params, r)
        _, (h1, h2, o) = self.gains(params)
        d = np.zeros_like(e)
        d[w] = e[w] - z[w]
        Ad = lap(d)
        Ae = lap(e)
        eAe = e[w] @ Ae[w]
        loss = d[w] @ Ad[w] / eAe
        g = np.zeros_like(e)
        g[w] = -2.0 * Ad[w] / eAe
        v = self._ext(self.Dh * g)
        dalpha = np.exp(alpha) * (v[w] @ u[w])
        Wv = v[self.ptx]
        Av = Wv @ B.T
        Y = S * Hm
        dB = Y.T @ Wv + (S * Av).T @ X
        dS = Hm * Av
        dO = dS * sigmoid(o)
        dW3T = h2.T @ dO
        db3 = dO.sum(0)
        dz2 = (dO @ W3T.T) * (1 - h2 * h2)
        dW2T = h1.T @ dz2
        db2 = dz2.sum(0)
        dz1 = (dz2 @ W2T.T) * (1 - h1 * h1)
        dW1T = self.feat.T @ dz1
        db1 = dz1.sum(0)
        grad = np.concatenate([dB.ravel(), [dalpha], dW1T.ravel(), db1, dW2T.ravel(), db2, dW3T.ravel(), db3])
        return loss, grad
