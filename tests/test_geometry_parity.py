"""Geometry set-up (row a14) against two independent computations, on the CPU.

The library's host set-up (`sod_host_elem_jacobian`, `sod_host_lumped_mass`,
csrc/host_setup.cpp) produces He = J^-1 and gpvol = w det J per Gauss point
and the lumped mass Ml, which both the GPU kernels and the oracle then read.
Here they are checked, on curved elements (element-interior GLL nodes
jittered by +-5 % of the local spacing, elements shuffled, non-vertex local
numbering shuffled, a non-cubic mesh), against

* the oracle's restatement of elem_jacobian
  (src/lib_sod2d/sources/jacobian_oper.f90:7-139): bit-identical in the
  reference's FP32 arithmetic, and within FP32 rounding (5e-6 relative,
  max norm) of its FP64 instantiation on the same inputs;
* a central finite-difference Jacobian of the isoparametric map
  x(xi) = sum_a N_a(xi) x_a evaluated with Lagrange polynomials through the
  GLL nodes in FP64, independent of the shape-function tables: the FP64
  restatement agrees to 2e-6 (the O(h^2) difference error), which pins the
  oracle's geometry on curved elements;
* the lumped mass as an FP64 sum of gpvol over the working connectivity
  (mass_matrix.f90:11-42) and the domain volume L^3.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

from sod2d_b200 import host

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
import oracle as O  # noqa: E402


def _nat(porder, ii):
    """Natural (ascending) GLL index of the reference's 1-D index ii (0-based):
    the reference orders -1, +1, then the interior nodes."""
    return 0 if ii == 0 else (porder if ii == 1 else ii - 1)


def _lagrange(xs, x):
    """Values of the Lagrange polynomials through nodes xs at points x."""
    L = np.ones((len(x), len(xs)))
    for a, xa in enumerate(xs):
        for b, xb in enumerate(xs):
            if a != b:
                L[:, a] *= (x - xb) / (xa - xb)
    return L


def _fd_geometry(m, h=1e-4):
    """He and gpvol from central differences of the isoparametric map."""
    P, n, E = m.porder, m.nnode, m.nelem
    xs, ws = host.gll(P)
    xs = np.asarray(xs, np.float64)
    ws = np.asarray(ws, np.float64)
    nat = np.array([[_nat(P, int(c) - 1) for c in g] for g in (m.gmshAtoI, m.gmshAtoJ, m.gmshAtoK)])  # (3, n)
    coord = m.coord.reshape(3, m.npoin).astype(np.float64)
    conn = m.connecOrig.reshape(n, E) - 1
    # nodal coordinates in a natural tensor grid X[e, i, j, k, c]
    X = np.zeros((E, P + 1, P + 1, P + 1, 3))
    X[:, nat[0], nat[1], nat[2], :] = coord[:, conn].transpose(2, 1, 0)

    def x_at(pts):  # pts (n, 3) reference coordinates -> (E, n, 3)
        Li, Lj, Lk = (_lagrange(xs, pts[:, d]) for d in range(3))
        return np.einsum("gi,gj,gk,eijkc->egc", Li, Lj, Lk, X)

    gp = np.stack([xs[nat[0]], xs[nat[1]], xs[nat[2]]], axis=1)  # Gauss point a -> (xi, eta, zeta)
    J = np.zeros((E, n, 3, 3))  # J[e, a, c, d] = d x_c / d xi_d
    for d in range(3):
        dp = np.zeros(3)
        dp[d] = h
        J[:, :, :, d] = (x_at(gp + dp) - x_at(gp - dp)) / (2 * h)
    Jinv = np.linalg.inv(J)  # Jinv[e, a, d, c] = d xi_d / d x_c
    He = np.transpose(Jinv, (0, 1, 3, 2))  # He(c, d) = d xi_d / d x_c
    w = ws[nat[0]] * ws[nat[1]] * ws[nat[2]]
    gpvol = w[None, :] * np.linalg.det(J)
    # reference layout: He(3,3,n,E) with the first index fastest, gpvol(1,n,E)
    return He.transpose(0, 1, 3, 2).reshape(-1), gpvol.reshape(-1)


def _rel(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / np.abs(b).max())


MESHES = [(3, (3, 3, 3)), (3, (4, 3, 2)), (4, (2, 3, 2)), (4, (3, 3, 3))]


@pytest.mark.parametrize("porder,dims", MESHES)
def test_host_geometry_matches_oracle_and_finite_differences(porder, dims):
    m = host.periodic_cube(porder, *dims, jitter=0.05, seed=7 + porder, elem_shuffle=True, ordering=1)
    n = m.nnode
    # curved elements: det J varies inside an element
    gv = m.gpvol.reshape(m.nelem, n)
    w = np.tile(m.wgp, 1)
    detJ = gv / w[None, :]
    assert np.ptp(detJ, axis=1).max() > 1e-3 * np.abs(detJ).max()

    # the oracle's restatement in the reference's FP32 arithmetic: identical
    gpvol32, He32 = O.elem_jacobian(porder, m.nelem, m.npoin, m.connecOrig, m.coord, m.dNgp, m.wgp, np.float32)
    assert np.array_equal(m.He, He32) and np.array_equal(m.gpvol, gpvol32)
    # ... and in FP64 on the same FP32 inputs: FP32 rounding apart
    gpvol64, He64 = O.elem_jacobian(porder, m.nelem, m.npoin, m.connecOrig, m.coord.astype(np.float64),
                                    m.dNgp.astype(np.float64), m.wgp.astype(np.float64), np.float64)
    assert _rel(m.He, He64) < 5e-6
    assert _rel(m.gpvol, gpvol64) < 2e-6

    # finite differences of the isoparametric map (independent of the tables)
    # pin the FP64 restatement itself
    He_fd, gpvol_fd = _fd_geometry(m)
    assert _rel(He64, He_fd) < 2e-6
    assert _rel(gpvol64, gpvol_fd) < 2e-6
    assert _rel(m.He, He_fd) < 5e-6

    # lumped mass: FP64 sum of gpvol over the working connectivity
    # (connecWork is (E,n) element-fastest, gpvol (1,n,E) node-fastest)
    cw = m.connecWork.reshape(n, m.nelem).T.reshape(-1) - 1
    Ml64 = np.bincount(cw, weights=m.gpvol.astype(np.float64), minlength=m.npoin)
    w_ = m.lpoin_w - 1
    assert _rel(m.Ml[w_], Ml64[w_]) < 2e-6
    assert np.allclose(m.invMl[w_], 1.0 / m.Ml[w_], rtol=1e-6)
    L = m.extra["L"]
    assert abs(m.vol_total - L ** 3) < 1e-5 * L ** 3
    assert abs(gpvol_fd.sum() - L ** 3) < 1e-5 * L ** 3
