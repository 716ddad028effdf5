"""The partitioned path on one GPU: every part of the mesh gets its own
context and halo plan; the parts run as host threads of one process and
exchange through LocalHaloGroup (device-to-device copies, barriers bounded
by a timeout; no kernel waits on another).

- sod_gpu_halo_update: each shared node ends up with the sum over its parts
  in ascending rank order, bit-identical to the same sum done in numpy, and
  identical on every part.
- sod_gpu_updateF and sod_gpu_full_proj_ijk with the halo plan: every
  part's residuals and projections match the whole-mesh oracle to 1e-5
  relative L2 on its nodes, and the parts agree bit for bit on the nodes
  they share.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from sod2d_b200 import host, partition
from sod2d_b200.halo import LocalHaloGroup

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_b200 import gpu as g
    return g


def _setup(gpu, porder, grid, Ma=0.5):
    if grid == "random":  # ragged parts on a non-cubic mesh
        m = host.periodic_cube(porder, 3, 4, 5, jitter=0.05, seed=91, elem_shuffle=True, ordering=1)
        pe = np.random.default_rng(92).integers(0, 3, m.nelem).astype(np.int32)
    else:
        m = host.periodic_cube(porder, 4, jitter=0.05, seed=71, elem_shuffle=True, ordering=1)
        pe = partition.partition_elements(m, grid)
    ic = host.tgv_comp_init(m, Ma=Ma)
    parts = partition.split(m, pe)
    group = LocalHaloGroup([p.plan for p in parts], timeout=120.0)
    ctxs = []
    for p in parts:
        ctx = gpu.Context(p.mesh, gpu.phys_from_ic(ic))
        ctx.set_halo(p.plan, group)
        ctxs.append(ctx)
    return m, ic, parts, group, ctxs


@pytest.mark.parametrize("grid", [(1, 1, 2), (2, 1, 2), (2, 2, 2), "random"])
def test_halo_update_rank_ordered_sum(gpu, grid):
    m, ic, parts, group, ctxs = _setup(gpu, 3, grid)
    rng = np.random.default_rng(72)
    ncomp = 14  # more than one 12-wide exchange
    vals = [rng.normal(size=ncomp * p.mesh.npoin).astype(np.float32) for p in parts]
    dev = [torch.from_numpy(v).cuda() for v in vals]
    group.run([lambda c=c, d=d: c.call("sod_gpu_halo_update", gpu.dptr(d), ncomp) for c, d in zip(ctxs, dev)])
    # expected: per global node, sequential float32 sum over the parts that hold it, ascending rank
    N = m.npoin
    exp = np.zeros((ncomp, N), np.float32)
    seen = np.zeros(N, bool)
    for p, v in zip(parts, vals):
        v = v.reshape(ncomp, -1)
        first = ~seen[p.nodes]
        exp[:, p.nodes[first]] = v[:, first]
        exp[:, p.nodes[~first]] = exp[:, p.nodes[~first]] + v[:, ~first]
        seen[p.nodes] = True
    for p, d in zip(parts, dev):
        got = d.cpu().numpy().reshape(ncomp, -1)
        assert np.array_equal(got.view(np.uint32), exp[:, p.nodes].view(np.uint32))
    for c in ctxs:
        c.close()


@pytest.mark.parametrize("porder,grid", [(3, (1, 1, 2)), (3, (2, 1, 2)), (4, (2, 1, 2)), (3, (2, 2, 2)),
                                         (3, "random")])
def test_partitioned_updateF_matches_whole_mesh(gpu, porder, grid):
    m, ic, parts, group, ctxs = _setup(gpu, porder, grid)
    rho, q, E = host.random_comp_state(m, seed=73)
    N, n = m.npoin, m.nnode
    u = (q.reshape(3, N) / rho).astype(np.float32)
    csound = np.full(N, 2.0, np.float32)
    mu_e = np.random.default_rng(74).uniform(0, 2e-3, m.nelem * n).astype(np.float32)
    om = O.OracleMesh(m)
    tau = O.comp_tau(om, csound, u.reshape(-1))
    Rm, Rq, Re, proj = O.rhs(om, O.comp_params(ic), rho, q, E, mu_e, ic.mu_factor, tau, want_proj=True)
    whole = (Rm, Rq, Re)

    def loc(a, k, nd):
        return np.ascontiguousarray(np.asarray(a).reshape(k, N)[:, nd].reshape(-1))

    dv = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    outs, projs, jobs = [], [], []
    for p, ctx in zip(parts, ctxs):
        nd, el = p.nodes, p.elems
        Np = p.mesh.npoin
        ins = [dv(loc(rho, 1, nd)), dv(loc(q, 3, nd)), dv(loc(E, 1, nd)),
               dv(mu_e.reshape(n, -1)[:, el].reshape(-1)), dv(tau[el])]
        up = [dv(loc(u, 3, nd))]
        T = ins[2] * 0  # filled by updateF
        out = [torch.zeros(k * Np, device="cuda") for k in (1, 3, 1)]
        extra = [torch.zeros(3 * Np, device="cuda"), torch.zeros(Np, device="cuda"), T,
                 torch.zeros(Np, device="cuda")]
        pj = [torch.zeros(3 * Np, device="cuda") for _ in range(5)]
        outs.append(out)
        projs.append(pj)

        def job(ctx=ctx, ins=ins, out=out, extra=extra, pj=pj, up=up):
            ctx.call("sod_gpu_updateF", *(gpu.dptr(x) for x in ins[:4]), C.c_float(ic.mu_factor), gpu.dptr(ins[4]),
                     *(gpu.dptr(x) for x in out), *(gpu.dptr(x) for x in extra))
            # projections alone: rho, u, Tem from the EOS outputs of updateF
            ctx.call("sod_gpu_full_proj_ijk", gpu.dptr(ins[0]), gpu.dptr(extra[0]), gpu.dptr(extra[2]),
                     *(gpu.dptr(x) for x in pj))
        jobs.append(job)
    group.run(jobs)

    # projections of the oracle: ProjMass, ProjEner, ProjMX, ProjMY, ProjMZ, each (N,3)
    oproj = np.asarray(proj).reshape(5, 3, N)
    gathered = {}
    for p, out, pj in zip(parts, outs, projs):
        nd = p.nodes
        for name, g, w, k in zip(("mass", "momentum", "energy"), out, whole, (1, 3, 1)):
            g = g.cpu().numpy()
            ref = loc(w, k, nd).astype(np.float64)
            err = np.linalg.norm(g - ref) / np.linalg.norm(ref)
            assert err < 1e-5, (p.rank, name, err)
            gathered.setdefault(name, []).append((nd, g.reshape(k, -1)))
        # the entry's outputs are ProjMass, ProjEner, ProjMX, ProjMY, ProjMZ in that order
        got = np.stack([x.cpu().numpy().reshape(3, -1) for x in pj])
        ref = oproj[:, :, nd]
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert err < 1e-5, (p.rank, "proj", err)
    # shared nodes: identical bits on every part that holds them
    for name, lst in gathered.items():
        val = {}
        for nd, g in lst:
            for j, node in enumerate(nd.tolist()):
                bits = g[:, j].view(np.uint32).tobytes()
                assert val.setdefault(node, bits) == bits, (name, node)
    for c in ctxs:
        c.close()


def test_bad_plans_and_failing_exchange(gpu):
    """sod_gpu_set_halo rejects plans the reference's comms arrays cannot
    describe (SOD_GPU_EINVAL, checked on the host before any device work),
    and a transport that fails makes the calling entry point fail with the
    transport's error, leaving the context usable."""
    m = host.periodic_cube(3, 4, seed=75)
    parts = partition.split(m, partition.partition_elements(m, (1, 1, 2)))
    p = parts[0]
    ctx = gpu.Context(p.mesh, gpu.default_phys())
    lib = gpu.lib()
    buf = torch.zeros(12 * max(p.plan.numNodesToComm, 1), device="cuda")
    noop = gpu.HALO_FN(lambda *a: 0)
    ip = lambda a: np.ascontiguousarray(a, np.int32)

    def set_plan(rank, nbs, pos, size, nodes):
        arrs = [ip(nbs), ip(pos), ip(size), ip(nodes if len(nodes) else [1])]
        return lib.sod_gpu_set_halo(ctx.h, rank, len(nbs), *(a.ctypes.data_as(gpu.P_I) for a in arrs),
                                    gpu.dptr(buf), gpu.dptr(buf), noop, None)

    nodes = p.plan.nodesToComm
    n = nodes.size
    assert set_plan(0, [1], [1], [n], nodes) == 0
    assert set_plan(0, [0], [1], [n], nodes) == -1                       # own rank as neighbour
    assert set_plan(0, [1], [2], [n], nodes) == -1                       # range not starting at 1
    assert set_plan(0, [1, 1], [1, 2], [1, n - 1], nodes) == -1          # neighbour twice
    bad = nodes.copy(); bad[0] = p.mesh.npoin + 1
    assert set_plan(0, [1], [1], [n], bad) == -1                         # node id out of range
    dup = nodes.copy(); dup[1] = dup[0]
    assert set_plan(0, [1], [1], [n], dup) == -1                         # node twice for one neighbour
    assert set_plan(0, [], [], [], []) == 0                              # removes the plan

    class Failing:
        def exchange(self, plan, send, recv, width):
            raise ConnectionError("peer went away")

    ctx.set_halo(p.plan, Failing())
    f = torch.ones(p.mesh.npoin, device="cuda")
    with pytest.raises(RuntimeError) as ei:
        ctx.call("sod_gpu_halo_update", gpu.dptr(f), 1)
    assert isinstance(ei.value.__cause__, ConnectionError)
    assert "halo exchange" in gpu.last_error()
    # still usable without the plan
    assert set_plan(0, [], [], [], []) == 0
    ctx.call("sod_gpu_halo_update", gpu.dptr(f), 1)
    assert float(f.sum()) == p.mesh.npoin
    ctx.close()


@pytest.mark.parametrize("porder,grid,stages", [(3, (2, 1, 2), 4), (4, (2, 2, 2), 5)])
def test_partitioned_rk_time_loop_matches_whole_mesh(gpu, porder, grid, stages):
    """rk_4_ls_main on a partitioned mesh: every part runs sod_gpu_comp_rk_ls_step
    with the halo sums of the RHS, the entropy residual, the divergence and
    the vorticity, and the global min rho / dt / analysis reductions.  The
    parts agree on every dt and analysis row bit for bit; those rows and
    the final state match the whole-mesh GPU run to 1e-5 (the reference's
    TGV at Ma 1.25, entropy viscosity and LPS on)."""
    m = host.periodic_cube(porder, 4, jitter=0.05, seed=76, elem_shuffle=True, ordering=1)
    ic = host.tgv_comp_init(m, Ma=1.25)
    nsteps = 8
    whole = gpu.CompSolver(m, ic, stages=stages)
    hw = whole.run(nsteps, log_first=1, log_step=1)
    sw = whole.state()
    whole.close()

    parts = partition.split(m, partition.partition_elements(m, grid))
    group = LocalHaloGroup([p.plan for p in parts], timeout=120.0)
    solvers = group.run([lambda p=p: gpu.CompSolver(m, ic, stages=stages, partition=(p, group)) for p in parts])
    hists = group.run([lambda s=s: s.run(nsteps, log_first=1, log_step=1) for s in solvers])
    states = [s.state() for s in solvers]
    for h in hists[1:]:
        assert np.array_equal(h, hists[0])
    hp = hists[0]
    assert hp.shape == hw.shape
    # time, EK, eps_S, eps_D, eps_T, max Mach: dt is a minimum over the state,
    # so it follows the state's rounding-level differences (different
    # summation orders of the halo sums)
    rel = np.abs(hp - hw) / np.maximum(np.abs(hw), 1e-30)
    print(f"P={porder} {len(parts)} parts: max relative difference per column {rel.max(axis=0)}")
    assert rel.max() < 1e-5
    N, n = m.npoin, m.nnode
    for p, st in zip(parts, states):
        for key, k in (("rho", 1), ("q", 3), ("E", 1)):
            ref = sw[key].reshape(k, N)[:, p.nodes].astype(np.float64)
            err = np.linalg.norm(st[key].reshape(k, -1) - ref) / np.linalg.norm(ref)
            assert err < 1e-5, (p.rank, key, err)
        mref = sw["mu_e"].reshape(n, -1)[:, p.elems].astype(np.float64)
        err = np.linalg.norm(st["mu_e"].reshape(n, -1) - mref) / max(np.linalg.norm(mref), 1e-30)
        assert err < 1e-4, (p.rank, "mu_e", err)
    for s in solvers:
        s.close()


@pytest.mark.parametrize("porder,grid,stages", [(4, (2, 1, 2), 4), (3, (2, 2, 2), 3)])
def test_partitioned_imex_loop_matches_whole_mesh(gpu, porder, grid, stages):
    """imex_main on a partitioned mesh: halo sums of the stage residuals,
    the LPS terms and the implicit solve's operator, CG dot products over
    the owned nodes summed over the ranks (lpoin_o and MPI_Allreduce,
    mod_solver_imex.f90:171-181), the entropy chain's halo sums and
    reductions.  Every part takes the same CG iterations as the whole-mesh
    run; the analysis rows agree between parts bit for bit and match the
    whole-mesh GPU run (the reference's IMEX settings: Ma 1.25, CFL 0.95)."""
    m = host.periodic_cube(porder, 4, jitter=0.05, seed=78, elem_shuffle=True, ordering=1)
    ic = host.tgv_comp_init(m, Ma=1.25)
    nsteps = 6
    kw = dict(stages=stages, fp64_state=False, cfl_conv=0.95, cfl_diff=1000.5, imex=True)

    def run(s):
        rows, its = [s.analysis()], []
        for _ in range(nsteps):
            s.step()
            it = gpu.C.c_int()
            s.ctx.call("sod_gpu_comp_imex_stats", gpu.C.byref(it), None)
            its.append(it.value)
            rows.append(s.analysis())
            s.dt = s.adapt_dt()
        return np.array(rows), its

    whole = gpu.CompSolver(m, ic, **kw)
    hw, itw = run(whole)
    whole.close()
    parts = partition.split(m, partition.partition_elements(m, grid))
    group = LocalHaloGroup([p.plan for p in parts], timeout=120.0)
    solvers = group.run([lambda p=p: gpu.CompSolver(m, ic, partition=(p, group), **kw) for p in parts])
    out = group.run([lambda s=s: run(s) for s in solvers])
    for s in solvers:
        s.close()
    for h, its in out[1:]:
        assert np.array_equal(h, out[0][0]) and its == out[0][1]
    hp, itp = out[0]
    print(f"P={porder} {len(parts)} parts, CG iterations whole {itw} parts {itp}")
    assert itp == itw
    rel = np.abs(hp - hw) / np.maximum(np.abs(hw), 1e-30)
    print("max relative difference per column", rel.max(axis=0))
    assert rel.max() < 1e-4


@pytest.mark.parametrize("porder,grid", [(3, (2, 1, 2)), (4, (2, 2, 2))])
def test_partitioned_incomp_loop_matches_whole_mesh(gpu, porder, grid):
    """bdfext3_main_incomp on a partitioned mesh with the reference's FP32
    solves (conjGrad_pressure_incomp and conjGrad_veloc_incomp at maxIter 20,
    tol 1e-2): halo sums inside the Laplacian, its diagonal, the gradient,
    the divergence and the velocity projection, on the convection and on the
    velocity operator; CG dots over owned nodes summed over the ranks; the
    dt and analysis reductions.  The parts agree bit for bit; the pressure
    and velocity CG iterations equal the whole-mesh run's and the analysis
    rows match it."""
    m = host.periodic_cube(porder, 4, jitter=0.05, seed=79, elem_shuffle=True, ordering=1)
    opts = gpu.SolveOpts(20, 1e-2, 2, 50, 0)
    nsteps = 8

    def run(s):
        rows, its = [s.analysis()], []
        for _ in range(nsteps):
            s.step(opts)
            vi, vr = C.c_int(), C.c_double()
            s.ctx.call("sod_gpu_incomp_veloc_stats", C.byref(vi), C.byref(vr))
            its.append((s.stats.iterations, vi.value))
            rows.append(s.analysis())
            s.dt = s.adapt_dt()
        return np.array(rows), its

    whole = gpu.IncompSolver(m, Re=1600.0, cfl_conv=0.5, veloc=(20, 1e-2))
    hw, itw = run(whole)
    whole.close()
    parts = partition.split(m, partition.partition_elements(m, grid))
    group = LocalHaloGroup([p.plan for p in parts], timeout=120.0)
    solvers = group.run([lambda p=p: gpu.IncompSolver(m, Re=1600.0, cfl_conv=0.5, veloc=(20, 1e-2),
                                                      partition=(p, group)) for p in parts])
    out = group.run([lambda s=s: run(s) for s in solvers])
    for s in solvers:
        s.close()
    for h, its in out[1:]:
        assert np.array_equal(h, out[0][0]) and its == out[0][1]
    hp, itp = out[0]
    print(f"P={porder} {len(parts)} parts: (pressure, velocity) CG iterations whole {itw} parts {itp}")
    assert itp == itw
    rel = np.abs(hp[:, :5] - hw[:, :5]) / np.maximum(np.abs(hw[:, :5]), 1e-30)
    print("max relative difference per column (time, EK, eps_S, eps_D, eps_T)", rel.max(axis=0))
    assert rel.max() < 1e-4


@pytest.mark.parametrize("porder,grid", [(3, (2, 1, 2)), (3, (2, 2, 2))])
def test_partitioned_fp64_pressure_solve_matches_whole_mesh(gpu, porder, grid):
    """The FP64-certified Jacobi pressure solve on a partitioned mesh (a
    host-driven PCG with the Laplacian and its diagonal summed over the
    ranks and the dots over the owned nodes): in the incompressible loop,
    every solve is certified below 1e-8 on every part, the parts agree bit
    for bit, and the analysis rows match the whole-mesh run with the
    device-resident solve."""
    m = host.periodic_cube(porder, 4, jitter=0.05, seed=80, elem_shuffle=True, ordering=1)
    opts = gpu.SolveOpts(4000, 1e-8, 0, 50, 0)
    nsteps = 5

    def run(s):
        rows, its = [s.analysis()], []
        for _ in range(nsteps):
            s.step(opts)
            assert s.stats.res_rel < 1e-8
            its.append(s.stats.iterations)
            rows.append(s.analysis())
            s.dt = s.adapt_dt()
        return np.array(rows), its

    whole = gpu.IncompSolver(m, Re=1600.0, cfl_conv=0.5, veloc=(20, 1e-4))
    hw, itw = run(whole)
    whole.close()
    parts = partition.split(m, partition.partition_elements(m, grid))
    group = LocalHaloGroup([p.plan for p in parts], timeout=120.0)
    solvers = group.run([lambda p=p: gpu.IncompSolver(m, Re=1600.0, cfl_conv=0.5, veloc=(20, 1e-4),
                                                      partition=(p, group)) for p in parts])
    out = group.run([lambda s=s: run(s) for s in solvers])
    for s in solvers:
        s.close()
    for h, its in out[1:]:
        assert np.array_equal(h, out[0][0]) and its == out[0][1]
    hp, itp = out[0]
    print(f"P={porder} {len(parts)} parts: FP64 Jacobi iterations whole {itw} parts {itp}")
    rel = np.abs(hp[:, :5] - hw[:, :5]) / np.maximum(np.abs(hw[:, :5]), 1e-30)
    print("max relative difference per column (time, EK, eps_S, eps_D, eps_T)", rel.max(axis=0))
    assert rel.max() < 1e-5
    assert all(abs(a - b) <= max(3, 0.05 * b) for a, b in zip(itp, itw))


def test_partition_refuses_global_solves(gpu):
    """The learned preconditioner, whose patches cross the part boundaries,
    is refused on a context with a halo plan (the pressure solve and the
    incompressible step with precond 1) instead of giving a rank-local
    answer."""
    m = host.periodic_cube(3, 4, seed=77)
    parts = partition.split(m, partition.partition_elements(m, (1, 1, 2)))
    p = parts[0]
    ctx = gpu.Context(p.mesh, gpu.default_phys())
    group = LocalHaloGroup([p.plan], timeout=10.0)  # never exchanges here
    ctx.set_halo(p.plan, group)
    N = p.mesh.npoin
    b, x = torch.zeros(N, dtype=torch.float64, device="cuda"), torch.zeros(N, dtype=torch.float64, device="cuda")
    st = gpu.SolveStats()
    with pytest.raises(RuntimeError, match="halo plan"):
        ctx.call("sod_gpu_pressure_solve", gpu.dptr(b), gpu.dptr(x), C.byref(gpu.SolveOpts(10, 1e-8, 1, 50, 0)),
                 C.byref(st))
    u = torch.zeros(3 * N, device="cuda")
    ctx.call("sod_gpu_incomp_init", gpu.dptr(u), 1e-3)
    with pytest.raises(RuntimeError, match="halo plan"):
        ctx.call("sod_gpu_incomp_step", C.c_float(1e-3), C.byref(gpu.SolveOpts(10, 1e-8, 1, 50, 0)), C.byref(st))
    ctx.close()
