"""ORACLE -- test infrastructure only.

numpy restatement of the learned element-patch preconditioner of the GPU
library (forward pass, energy-norm loss ||e - M(r)||_A^2 / ||e||_A^2 and its
analytic gradient), used by tests/ to check the GPU forward and backward
kernels.  Element-local node order is the tensor order t = i + n1 j + n1^2 k
(natural GLL order), faces are ordered (i=0, i=P, j=0, j=P, k=0, k=P).
"""
from __future__ import annotations

import numpy as np

H = 32


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


def face_neighbours(mesh, conn):
    P, E = mesh.porder, mesh.nelem
    n1 = P + 1
    tid = lambda i, j, k: i + n1 * (j + n1 * k)
    faces = {}
    for e in range(E):
        for f in range(6):
            d, v = f // 2, (P if f % 2 else 0)
            key = []
            for a in (0, P):
                for b in (0, P):
                    ijk = [(v, a, b), (a, v, b), (a, b, v)][d]
                    key.append(conn[e, tid(*ijk)])
            faces.setdefault(tuple(sorted(key)), []).append((e, f))
    nbr = np.repeat(np.arange(E)[:, None], 6, axis=1)
    for v in faces.values():
        if len(v) == 2:
            (e0, f0), (e1, f1) = v
            nbr[e0, f0] = e1
            nbr[e1, f1] = e0
    return nbr


def unpack(params, N):
    NIN = N + 6
    o = 0
    W1T = params[o:o + NIN * H].reshape(NIN, H); o += NIN * H
    b1 = params[o:o + H]; o += H
    W2T = params[o:o + H * H].reshape(H, H); o += H * H
    b2 = params[o:o + H]; o += H
    W3T = params[o:o + H * N].reshape(H, N); o += H * N
    b3 = params[o:o + N]; o += N
    return W1T, b1, W2T, b2, W3T, b3


class Net:
    def __init__(self, mesh, Minv):
        self.mesh = mesh
        self.conn = tensor_conn(mesh)
        self.nbr = face_neighbours(mesh, self.conn)
        E, N = self.conn.shape
        lel = np.bincount(self.conn.ravel(), minlength=mesh.npoin)
        self.w = 1.0 / lel[self.conn]
        self.Minv = Minv
        self.N = N

    def forward(self, params, r):
        conn, N = self.conn, self.N
        x_own = r[conn] * self.Minv[conn]                 # (E, N)
        emean = x_own.mean(1)
        x = np.concatenate([x_own, emean[self.nbr]], 1)   # (E, NIN)
        s = np.sqrt((x * x).mean(1))
        inv = np.where(s > 0, 1.0 / np.where(s > 0, s, 1.0), 0.0)
        xh = x * inv[:, None]
        W1T, b1, W2T, b2, W3T, b3 = unpack(params, N)
        h1 = np.tanh(xh @ W1T + b1)
        h2 = np.tanh(h1 @ W2T + b2)
        y = h2 @ W3T + b3
        out = s[:, None] * self.w * (xh[:, :N] + y)
        z = np.zeros(self.mesh.npoin)
        np.add.at(z, conn.ravel(), out.ravel())
        return z, (s, xh, h1, h2)

    def loss_grad(self, params, r, e, lap):
        """lap(v) -> A v (FP64).  Returns loss, gradient (float64)."""
        w_idx = self.mesh.lpoin_w - 1
        z, (s, xh, h1, h2) = self.forward(params, r)
        d = np.zeros_like(e)
        d[w_idx] = e[w_idx] - z[w_idx]
        Ad = lap(d)
        Ae = lap(e)
        eAe = e[w_idx] @ Ae[w_idx]
        loss = d[w_idx] @ Ad[w_idx] / eAe
        g = np.zeros_like(e)
        g[w_idx] = -2.0 * Ad[w_idx] / eAe
        N = self.N
        W1T, b1, W2T, b2, W3T, b3 = unpack(params, N)
        dy = g[self.conn] * s[:, None] * self.w           # (E, N)
        dW3T = h2.T @ dy
        db3 = dy.sum(0)
        dz2 = (dy @ W3T.T) * (1 - h2 * h2)
        dW2T = h1.T @ dz2
        db2 = dz2.sum(0)
        dz1 = (dz2 @ W2T.T) * (1 - h1 * h1)
        dW1T = xh.T @ dz1
        db1 = dz1.sum(0)
        grad = np.concatenate([dW1T.ravel(), db1, dW2T.ravel(), db2, dW3T.ravel(), db3])
        return loss, grad
