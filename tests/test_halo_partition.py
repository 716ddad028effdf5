"""Partitioned meshes on the CPU: the sub-meshes and halo plans of
sod2d_b200.partition, and the exchange of sod2d_b200.halo over gloo.

- Plan invariants: every element in one part, every shared node listed in
  the same order on both sides of each pair, Ml of the whole mesh on every
  rank's nodes, the parts' volumes adding up to the mesh's.
- World size 4 (a 2 x 1 x 2 grid of parts, so corner nodes sit on four
  ranks), gloo: each rank runs the oracle's updateF on its sub-mesh with the
  reference's halo sums (mod_comms.f90:467-627) at the reference's places,
  the buffers moving through DistHaloTransport.  Every rank's residuals and
  projections match the whole-mesh oracle on its nodes.
- World size 4, gloo: the oracle's whole TGV loop on each rank's sub-mesh,
  with the reference's halo sums and MPI_Allreduce calls (min rho, dt, the
  analysis integrals) through DistHaloTransport, reproduces the whole-mesh
  history.
"""
import os
import socket

import numpy as np
import pytest

import oracle as O
from sod2d_b200 import host, partition

torch = pytest.importorskip("torch")


def _mesh(porder=3, n=4):
    return host.periodic_cube(porder, n, jitter=0.05, seed=61, elem_shuffle=True, ordering=1)


@pytest.mark.parametrize("grid", [(1, 1, 2), (2, 1, 2), (2, 2, 2)])
def test_plan_invariants(grid):
    m = _mesh()
    pe = partition.partition_elements(m, grid)
    parts = partition.split(m, pe)
    assert len(parts) == int(np.prod(grid))
    allel = np.concatenate([p.elems for p in parts])
    assert np.array_equal(np.sort(allel), np.arange(m.nelem))
    owners = {}
    for p in parts:
        for g in p.nodes:
            owners.setdefault(int(g), []).append(p.rank)
        assert np.array_equal(p.mesh.Ml, m.Ml[p.nodes])
        assert p.plan.commsMemPosInLoc.tolist() == (1 + np.concatenate([[0], np.cumsum(p.plan.commsMemSize)[:-1]])).tolist()
    assert abs(sum(float(p.mesh.gpvol.astype(np.float64).sum()) for p in parts) -
               float(m.gpvol.astype(np.float64).sum())) < 1e-6 * m.vol_total
    for p in parts:
        for nb in p.plan.ranksToComm.tolist():
            a, b = p.plan.range_of(nb)
            q = parts[nb]
            qa, qb = q.plan.range_of(p.rank)
            mine = p.nodes[p.plan.nodesToComm[a:b] - 1]
            theirs = q.nodes[q.plan.nodesToComm[qa:qb] - 1]
            assert np.array_equal(mine, theirs)
            assert np.all(np.diff(mine) > 0)
        # a node appears once per other rank that holds it
        cnt = np.bincount(p.plan.nodesToComm - 1, minlength=p.mesh.npoin)
        for loc, g in enumerate(p.nodes):
            assert cnt[loc] == len(owners[int(g)]) - 1
    if grid == (2, 2, 2):
        assert max(len(v) for v in owners.values()) == 8


def test_ragged_random_partition_plan():
    """A random element-to-part assignment on a non-cubic mesh (ragged parts,
    nodes on all three ranks): every node's ranks list it, both sides of a
    pair agree on the order, and each part's nodes are exactly the nodes
    its elements touch."""
    m = host.periodic_cube(3, 3, 4, 5, jitter=0.05, seed=91, elem_shuffle=True, ordering=1)
    pe = np.random.default_rng(92).integers(0, 3, m.nelem).astype(np.int32)
    parts = partition.split(m, pe)
    n = m.nnode
    cw = m.connecWork.reshape(n, m.nelem) - 1
    owners = {}
    for p in parts:
        assert np.array_equal(p.nodes, np.unique(cw[:, p.elems]))
        # local connectivity maps back to the global one
        lc = p.mesh.connecWork.reshape(n, -1) - 1
        assert np.array_equal(p.nodes[lc], cw[:, p.elems])
        for g in p.nodes:
            owners.setdefault(int(g), []).append(p.rank)
    assert max(len(v) for v in owners.values()) == 3
    for p in parts:
        for nb in p.plan.ranksToComm.tolist():
            a, b = p.plan.range_of(nb)
            qa, qb = parts[nb].plan.range_of(p.rank)
            assert np.array_equal(p.nodes[p.plan.nodesToComm[a:b] - 1],
                                  parts[nb].nodes[parts[nb].plan.nodesToComm[qa:qb] - 1])
    with pytest.raises(ValueError):
        partition.split(m, np.zeros(m.nelem - 1, np.int32))
    with pytest.raises(ValueError):
        partition.split(m, np.full(m.nelem, 1, np.int32), nparts=2)  # part 0 empty


def _rank_main(rank, world, port, grid, out_dir):
    import torch.distributed as dist
    from sod2d_b200.halo import DistHaloTransport
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m = _mesh()
        ic = host.tgv_comp_init(m, Ma=0.5)
        rho, q, E = host.random_comp_state(m, seed=62)
        N, n = m.npoin, m.nnode
        u = (q.reshape(3, N) / rho).astype(np.float32)
        csound = np.full(N, 2.0, np.float32)
        mu_e = np.random.default_rng(63).uniform(0, 2e-3, m.nelem * n).astype(np.float32)
        prm = O.comp_params(ic)
        om = O.OracleMesh(m)
        tau = O.comp_tau(om, csound, u.reshape(-1))
        whole = O.rhs(om, prm, rho, q, E, mu_e, ic.mu_factor, tau, want_proj=True)

        p = partition.split(m, partition.partition_elements(m, grid))[rank]
        nd, el = p.nodes, p.elems
        loc = lambda a, k: np.ascontiguousarray(a.reshape(k, N)[:, nd].reshape(-1))
        tr = DistHaloTransport()
        O.set_halo(lambda comps: O.halo_exchange_add(p.plan, comps, tr))
        try:
            pom = O.OracleMesh(p.mesh)
            got = O.rhs(pom, prm, loc(rho, 1), loc(q, 3), loc(E, 1),
                        np.ascontiguousarray(mu_e.reshape(n, -1)[:, el].reshape(-1)), ic.mu_factor, tau[el],
                        want_proj=True)
        finally:
            O.set_halo(None)
        errs = []
        for g, w, k in zip(got, whole, (1, 3, 1, 15)):
            ref = loc(np.asarray(w), k).astype(np.float64)
            errs.append(float(np.linalg.norm(g - ref) / np.linalg.norm(ref)))
        np.save(os.path.join(out_dir, f"err{rank}.npy"), np.array(errs))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_gloo_partitioned_rhs_matches_whole_mesh(tmp_path):
    import torch.multiprocessing as mp
    grid = (2, 1, 2)
    world = int(np.prod(grid))
    mp.spawn(_rank_main, args=(world, _free_port(), grid, str(tmp_path)), nprocs=world, join=True)
    for r in range(world):
        errs = np.load(tmp_path / f"err{r}.npy")
        print(f"rank {r}: rel L2 mass {errs[0]:.1e} momentum {errs[1]:.1e} energy {errs[2]:.1e} proj {errs[3]:.1e}")
        assert np.all(errs < 1e-5), (r, errs)


def _loop_rank_main(rank, world, port, grid, nsteps, out_dir):
    """The oracle's whole TGV loop (rk_4_ls_main with entropy viscosity,
    LPS, CFL dt and the analysis) on this rank's sub-mesh, with the
    reference's halo sums and MPI_Allreduce calls going through
    DistHaloTransport over gloo."""
    import dataclasses

    import torch.distributed as dist
    from sod2d_b200.halo import DistHaloTransport
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m = _mesh(4, 4)
        ic = host.tgv_comp_init(m, Ma=1.25)
        prm = O.comp_params(ic, stages=5, rk_n=1, log_step=1)
        p = partition.split(m, partition.partition_elements(m, grid))[rank]
        N = m.npoin
        loc = lambda a: np.ascontiguousarray(np.asarray(a).reshape(-1, N)[:, p.nodes].reshape(-1))
        ic_p = dataclasses.replace(ic, **{f.name: loc(getattr(ic, f.name)) for f in dataclasses.fields(ic)
                                          if isinstance(getattr(ic, f.name), np.ndarray)
                                          and getattr(ic, f.name).size % N == 0 and getattr(ic, f.name).size >= N})
        tr = DistHaloTransport()

        def reduce(vals, kind):
            t = torch.from_numpy(vals.copy())
            tr.allreduce(rank, t, kind)
            vals[:] = t.numpy()

        O.set_halo(lambda comps: O.halo_exchange_add(p.plan, comps, tr))
        O.set_reduce(reduce)
        try:
            hist, _ = O.tgv_comp_run(O.OracleMesh(p.mesh), ic_p, prm, nsteps)
        finally:
            O.set_halo(None)
            O.set_reduce(None)
        np.save(os.path.join(out_dir, f"hist{rank}.npy"), hist)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_gloo_partitioned_time_loop_matches_whole_mesh(tmp_path):
    """World size 4: the oracle's partitioned TGV history (P=4, Ma 1.25,
    SSP53_2N_1, 20 steps logged every step) equals the whole-mesh oracle's
    to 1e-5 relative per column, and the ranks agree exactly."""
    import torch.multiprocessing as mp
    grid, nsteps = (2, 1, 2), 20
    world = int(np.prod(grid))
    m = _mesh(4, 4)
    ic = host.tgv_comp_init(m, Ma=1.25)
    whole, _ = O.tgv_comp_run(O.OracleMesh(m), ic, O.comp_params(ic, stages=5, rk_n=1, log_step=1), nsteps)
    mp.spawn(_loop_rank_main, args=(world, _free_port(), grid, nsteps, str(tmp_path)), nprocs=world, join=True)
    hists = [np.load(tmp_path / f"hist{r}.npy") for r in range(world)]
    for h in hists[1:]:
        assert np.array_equal(h, hists[0])
    h = hists[0]
    assert h.shape == whole.shape
    rel = np.abs(h - whole) / np.maximum(np.abs(whole), 1e-30)
    print("max relative difference per column (time, EK, eps_S, eps_D, eps_T, Mach):", rel.max(axis=0))
    assert rel.max() < 1e-5
