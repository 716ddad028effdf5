"""Python view of the host-side set-up library (``libsod2d_host.so``).

``periodic_cube`` builds a synthetic periodic hexahedral mesh and every
geometric table the SOD2D solver computes before its time loop, in the
reference's Fortran layout (column-major arrays, 1-based connectivity).  The
arrays are exactly what a SOD2D Fortran caller hands to the GPU library.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import build as _build

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = _build.LIBDIR / "libsod2d_host.so"
        if not path.exists():
            _build.build_host()
        _lib = C.CDLL(str(path))
        _declare(_lib)
    return _lib


P_I = C.POINTER(C.c_int)
P_F = C.POINTER(C.c_float)
P_D = C.POINTER(C.c_double)


def _declare(L):
    L.sod_host_gll.argtypes = [C.c_int, P_D, P_D]
    L.sod_host_atoijk.argtypes = [C.c_int, C.c_int, C.c_uint64, P_I]
    L.sod_host_atoijk_inverse.argtypes = [C.c_int, P_I, P_I, P_I, P_I, P_I]
    L.sod_host_shape_tables.argtypes = [C.c_int, P_I, P_F, P_F, P_F, P_F, P_F]
    L.sod_host_cube_sizes.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, P_I, P_I, P_I]
    L.sod_host_cube_mesh.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                     C.c_uint64, C.c_int, P_I, P_F, P_I, P_I, P_I]
    L.sod_host_elem_jacobian.argtypes = [C.c_int, C.c_int, C.c_int, P_I, P_F, P_F, P_F, P_F, P_F]
    L.sod_host_lumped_mass.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, P_I, P_I, P_F, P_F, P_F, P_D]
    L.sod_host_char_length.argtypes = [C.c_int, C.c_int, C.c_int, P_I, P_F, P_F, P_F]
    L.sod_host_elem_per_node.argtypes = [C.c_int, C.c_int, C.c_int, P_I, P_I]
    L.sod_host_tgv_comp_init.argtypes = [C.c_int, P_F] + [C.c_float] * 7 + [P_F] * 11
    for name in ("sod_host_gll", "sod_host_atoijk", "sod_host_atoijk_inverse", "sod_host_shape_tables",
                 "sod_host_cube_sizes", "sod_host_cube_mesh", "sod_host_elem_jacobian",
                 "sod_host_lumped_mass", "sod_host_char_length", "sod_host_elem_per_node",
                 "sod_host_tgv_comp_init"):
        getattr(L, name).restype = C.c_int


def ptr(a: np.ndarray):
    """ctypes pointer to a contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"]
    t = {np.float32: P_F, np.float64: P_D, np.int32: P_I}[a.dtype.type]
    return a.ctypes.data_as(t)


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} failed with code {rc}")


def gll(porder: int):
    x = np.zeros(porder + 1)
    w = np.zeros(porder + 1)
    _check(lib().sod_host_gll(porder, ptr(x), ptr(w)), "sod_host_gll")
    return x, w


@dataclass
class Mesh:
    """Mesh + geometry in the reference layout.  Fortran array ``A(n1,n2,..)``
    is stored as a flat numpy array with the first index fastest."""
    porder: int
    nelem: int
    npoin: int
    npoin_w: int
    coord: np.ndarray        # (N,3) f32
    connecOrig: np.ndarray   # (E,n) i32, 1-based
    connecWork: np.ndarray   # (E,n) i32, 1-based
    lpoin_w: np.ndarray      # (N_w) i32, 1-based
    atoIJK: np.ndarray
    invAtoIJK: np.ndarray
    gmshAtoI: np.ndarray
    gmshAtoJ: np.ndarray
    gmshAtoK: np.ndarray
    xgp: np.ndarray
    wgp: np.ndarray
    Ngp: np.ndarray
    dNgp: np.ndarray
    dlxigp_ip: np.ndarray
    He: np.ndarray           # (3,3,n,E) f32
    gpvol: np.ndarray        # (1,n,E) f32
    Ml: np.ndarray
    invMl: np.ndarray
    helem: np.ndarray
    helem_l: np.ndarray      # (E,n)
    lelpn: np.ndarray
    vol_total: float
    extra: dict = field(default_factory=dict)

    @property
    def nnode(self) -> int:
        return (self.porder + 1) ** 3


def periodic_cube(porder: int, nx: int, ny: int | None = None, nz: int | None = None,
                  L: float = 2.0 * 3.14159265, jitter: float = 0.0, seed: int = 1234,
                  elem_shuffle: bool = False, ordering: int = 0) -> Mesh:
    """Periodic cube [0,L]^3 of nx*ny*nz order-``porder`` hexahedra.

    ``L`` defaults to 2*3.14159265, the box of the reference's TGV test meshes
    (``Tests/*/cube.geo``).  ``ordering`` 0 numbers element-local nodes vertex
    first; 1 also shuffles the non-vertex numbers (seeded)."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    Lb = lib()
    ne, nn, nw = C.c_int(), C.c_int(), C.c_int()
    _check(Lb.sod_host_cube_sizes(porder, nx, ny, nz, C.byref(ne), C.byref(nn), C.byref(nw)), "cube_sizes")
    ne, nn, nw = ne.value, nn.value, nw.value
    n = (porder + 1) ** 3
    np1 = porder + 1
    ato = np.zeros(n, np.int32)
    _check(Lb.sod_host_atoijk(porder, ordering, seed, ptr(ato)), "atoijk")
    inv = np.zeros(np1 ** 3, np.int32)
    gI, gJ, gK = (np.zeros(n, np.int32) for _ in range(3))
    _check(Lb.sod_host_atoijk_inverse(porder, ptr(ato), ptr(inv), ptr(gI), ptr(gJ), ptr(gK)), "atoijk_inverse")
    xgp = np.zeros(n * 3, np.float32)
    wgp = np.zeros(n, np.float32)
    Ngp = np.zeros(n * n, np.float32)
    dNgp = np.zeros(3 * n * n, np.float32)
    dl = np.zeros(n * 3 * np1, np.float32)
    _check(Lb.sod_host_shape_tables(porder, ptr(ato), ptr(xgp), ptr(wgp), ptr(Ngp), ptr(dNgp), ptr(dl)),
           "shape_tables")
    coord = np.zeros(nn * 3, np.float32)
    cO = np.zeros(ne * n, np.int32)
    cW = np.zeros(ne * n, np.int32)
    lw = np.zeros(nw, np.int32)
    _check(Lb.sod_host_cube_mesh(porder, nx, ny, nz, L, jitter, seed, int(elem_shuffle), ptr(ato),
                                 ptr(coord), ptr(cO), ptr(cW), ptr(lw)), "cube_mesh")
    He = np.zeros(9 * n * ne, np.float32)
    gpvol = np.zeros(n * ne, np.float32)
    _check(Lb.sod_host_elem_jacobian(porder, ne, nn, ptr(cO), ptr(coord), ptr(dNgp), ptr(wgp),
                                     ptr(gpvol), ptr(He)), "elem_jacobian")
    Ml = np.zeros(nn, np.float32)
    invMl = np.zeros(nn, np.float32)
    vol = C.c_double()
    _check(Lb.sod_host_lumped_mass(porder, ne, nn, nw, ptr(cW), ptr(lw), ptr(gpvol), ptr(Ml), ptr(invMl),
                                   C.byref(vol)), "lumped_mass")
    helem = np.zeros(ne, np.float32)
    helem_l = np.zeros(ne * n, np.float32)
    _check(Lb.sod_host_char_length(porder, ne, nn, ptr(cO), ptr(coord), ptr(helem), ptr(helem_l)), "char_length")
    lelpn = np.zeros(nn, np.int32)
    _check(Lb.sod_host_elem_per_node(porder, ne, nn, ptr(cW), ptr(lelpn)), "elem_per_node")
    return Mesh(porder, ne, nn, nw, coord, cO, cW, lw, ato, inv, gI, gJ, gK, xgp, wgp, Ngp, dNgp, dl,
                He, gpvol, Ml, invMl, helem, helem_l, lelpn, vol.value,
                extra=dict(nx=nx, ny=ny, nz=nz, L=L, jitter=jitter, seed=seed))


@dataclass
class CompIC:
    rho: np.ndarray
    u: np.ndarray
    q: np.ndarray
    pr: np.ndarray
    E: np.ndarray
    Tem: np.ndarray
    e_int: np.ndarray
    csound: np.ndarray
    machno: np.ndarray
    eta: np.ndarray
    Rgas: float
    Cp: float
    rho0: float
    P0: float
    mu_factor: float
    gamma: float
    Prt: float
    Ma: float


def tgv_comp_init(mesh: Mesh, Ma: float = 0.1, V0: float = 1.0, L: float = 1.0, T0: float = 1.0,
                  Re: float = 1600.0, gamma: float = 1.4, Prt: float = 0.71) -> CompIC:
    """Compressible Taylor-Green initial state (TGVCompSolver.f90:154-214)."""
    N = mesh.npoin
    f = {k: np.zeros(N * (3 if k in ("u", "q") else 1), np.float32)
         for k in ("rho", "u", "q", "pr", "E", "Tem", "e_int", "csound", "machno", "eta")}
    consts = np.zeros(8, np.float32)
    _check(lib().sod_host_tgv_comp_init(N, ptr(mesh.coord), Ma, V0, L, T0, Re, gamma, Prt,
                                        *(ptr(f[k]) for k in ("rho", "u", "q", "pr", "E", "Tem", "e_int",
                                                              "csound", "machno", "eta")), ptr(consts)),
           "tgv_comp_init")
    return CompIC(**f, Rgas=float(consts[0]), Cp=float(consts[1]), rho0=float(consts[2]),
                  P0=float(consts[3]), mu_factor=float(consts[4]), gamma=float(consts[5]),
                  Prt=float(consts[6]), Ma=float(consts[7]))


def random_comp_state(mesh: Mesh, seed: int = 7, p0: float | None = None, gamma: float = 1.4,
                      Ma: float = 0.1):
    """Random conserved state of the RHS micro-benchmark: rho ~ U[0.9,1.1],
    momentum rho*U[-1,1]^3, energy from p ~ U[0.9,1.1]*p0 (p0 = 1/(gamma Ma^2)).
    Returns FP32 arrays (rho, q(N,3), E) on all nodes (slaves copy masters)."""
    if p0 is None:
        p0 = 1.0 / (gamma * Ma * Ma)
    rng = np.random.default_rng(seed)
    N = mesh.npoin
    rho = rng.uniform(0.9, 1.1, N).astype(np.float32)
    vel = rng.uniform(-1.0, 1.0, (3, N)).astype(np.float32)
    q = (rho[None, :] * vel).astype(np.float32).reshape(-1)
    p = (rng.uniform(0.9, 1.1, N) * p0).astype(np.float32)
    kin = 0.5 * (vel.astype(np.float64) ** 2).sum(0)
    E = (p / (gamma - 1.0) + rho * kin).astype(np.float32)
    return rho, q, E
