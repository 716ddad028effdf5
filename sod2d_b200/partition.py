"""Element partitions of a mesh, the per-rank sub-meshes and the halo plans
between them, in the reference's comms layout.

A rank holds the elements of its part and every node they touch (renumbered
in ascending global order), with the geometry of those elements and the
lumped mass of the WHOLE mesh on its nodes, as the reference's partitioned
mesh files give each rank (connecParWork, workingNodesPar and Ml after the
halo sum of the set-up, src/lib_sod2d/sources/mod_hdf5.f90:2731-2806,
CFDSolverBase.f90:1761-1795).  The halo plan between ranks has the arrays
of src/lib_sod2d/sources/mod_comms.f90:
  ranksToComm(numRanksWithComms)   neighbour ranks, ascending
  commsMemPosInLoc / commsMemSize  1-based start and length of each
                                   neighbour's range in nodesToComm
  nodesToComm(numNodesToComm)      local node ids (1-based), each range in
                                   ascending global id, so both sides of a
                                   pair list the shared nodes in one order.
"""
from __future__ import annotations

from dataclasses import dataclass, replace

import numpy as np

from .host import Mesh


@dataclass
class HaloPlan:
    rank: int
    ranksToComm: np.ndarray       # int32, ascending
    commsMemPosInLoc: np.ndarray  # int32, 1-based
    commsMemSize: np.ndarray      # int32
    nodesToComm: np.ndarray       # int32, 1-based local node ids

    @property
    def numRanksWithComms(self) -> int:
        return int(self.ranksToComm.size)

    @property
    def numNodesToComm(self) -> int:
        return int(self.nodesToComm.size)

    def range_of(self, neighbour: int) -> tuple[int, int]:
        """0-based [start, end) of `neighbour`'s range in nodesToComm."""
        i = int(np.flatnonzero(self.ranksToComm == neighbour)[0])
        a = int(self.commsMemPosInLoc[i]) - 1
        return a, a + int(self.commsMemSize[i])


@dataclass
class Part:
    rank: int
    mesh: Mesh                 # the rank's sub-mesh, local numbering
    elems: np.ndarray          # global element ids (0-based), in local order
    nodes: np.ndarray          # global node ids (0-based) of the local nodes, ascending
    plan: HaloPlan


def partition_elements(mesh: Mesh, grid=(1, 1, 2)) -> np.ndarray:
    """Part id of every element: a gx x gy x gz grid of boxes over the
    element centroids (from the unwrapped coordinates of connecOrig), part
    = ix + gx*(iy + gy*iz)."""
    gx, gy, gz = grid
    n, E = mesh.nnode, mesh.nelem
    N = mesh.coord.size // 3
    xyz = mesh.coord.reshape(3, N).astype(np.float64)
    co = mesh.connecOrig.reshape(n, E) - 1
    cen = np.stack([xyz[d][co].mean(axis=0) for d in range(3)])
    lo = xyz.min(axis=1)[:, None]
    hi = xyz.max(axis=1)[:, None]
    rel = (cen - lo) / np.maximum(hi - lo, 1e-30)
    idx = [np.clip((rel[d] * g).astype(np.int64), 0, g - 1) for d, g in enumerate((gx, gy, gz))]
    return (idx[0] + gx * (idx[1] + gy * idx[2])).astype(np.int32)


def _submesh(mesh: Mesh, elems: np.ndarray, nodes: np.ndarray) -> Mesh:
    n, E = mesh.nnode, mesh.nelem
    Ne = elems.size
    cw = mesh.connecWork.reshape(n, E)[:, elems] - 1
    local = (np.searchsorted(nodes, cw) + 1).astype(np.int32).reshape(-1)
    N = mesh.coord.size // 3
    coord = mesh.coord.reshape(3, N)[:, nodes].reshape(-1).copy()
    return replace(
        mesh,
        nelem=int(Ne), npoin=int(nodes.size), npoin_w=int(nodes.size), coord=coord,
        connecOrig=local.copy(), connecWork=local,
        lpoin_w=np.arange(1, nodes.size + 1, dtype=np.int32),
        He=mesh.He.reshape(E, -1)[elems].reshape(-1).copy(),
        gpvol=mesh.gpvol.reshape(E, n)[elems].reshape(-1).copy(),
        Ml=mesh.Ml[nodes].copy(), invMl=mesh.invMl[nodes].copy(),
        helem=mesh.helem[elems].copy(),
        helem_l=mesh.helem_l.reshape(n, E)[:, elems].reshape(-1).copy(),
        lelpn=mesh.lelpn[nodes].copy(),
        extra=dict(mesh.extra, global_nodes=nodes, global_elems=elems))


def split(mesh: Mesh, part_of_elem: np.ndarray, nparts: int | None = None) -> list[Part]:
    """Sub-meshes and halo plans of every part.  Only working nodes (the
    periodic masters that connecWork references) exist on the ranks."""
    part_of_elem = np.asarray(part_of_elem, np.int32)
    if part_of_elem.shape != (mesh.nelem,):
        raise ValueError("one part id per element")
    nparts = int(part_of_elem.max()) + 1 if nparts is None else nparts
    if part_of_elem.min() < 0 or part_of_elem.max() >= nparts:
        raise ValueError("part ids must lie in [0, nparts)")
    n, E = mesh.nnode, mesh.nelem
    cw = mesh.connecWork.reshape(n, E) - 1
    elems = [np.flatnonzero(part_of_elem == r).astype(np.int64) for r in range(nparts)]
    if any(e.size == 0 for e in elems):
        raise ValueError("every part needs at least one element")
    nodes = [np.unique(cw[:, e]) for e in elems]
    parts = []
    for r in range(nparts):
        nbs, pos, size, lst = [], [], [], []
        at = 1
        for s in range(nparts):
            if s == r:
                continue
            shared = np.intersect1d(nodes[r], nodes[s], assume_unique=True)
            if shared.size == 0:
                continue
            nbs.append(s)
            pos.append(at)
            size.append(shared.size)
            lst.append(np.searchsorted(nodes[r], shared) + 1)
            at += shared.size
        plan = HaloPlan(r, np.array(nbs, np.int32), np.array(pos, np.int32), np.array(size, np.int32),
                        (np.concatenate(lst) if lst else np.zeros(0, np.int64)).astype(np.int32))
        parts.append(Part(r, _submesh(mesh, elems[r], nodes[r]), elems[r], nodes[r], plan))
    return parts
