"""Edge cases of the GPU library: a non-cubic periodic mesh (3 x 4 x 5
elements, shuffled element and node numbering) for the RHS, the Laplacian and
the learned preconditioner's patch table; invalid arguments returning
SOD_GPU_EINVAL with a message; a zero right-hand side."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import precond_ref as PR
from sod2d_b200 import host

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
TOL = 1e-5
EINVAL = -1


@pytest.fixture(scope="module")
def gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_b200 import gpu as g
    return g


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def box(porder=3):
    m = host.periodic_cube(porder, 3, 4, 5, jitter=0.05, seed=21, elem_shuffle=True, ordering=1)
    return m


def test_updateF_on_a_non_cubic_mesh(gpu):
    m = box()
    rho, q, E = host.random_comp_state(m, seed=22)
    ic = host.tgv_comp_init(m, Ma=0.1)
    N = m.npoin
    u = (q.reshape(3, N) / rho).astype(np.float32)
    eint = E / rho - 0.5 * (u.astype(np.float64) ** 2).sum(0)
    pr = (rho * (ic.gamma - 1.0) * eint).astype(np.float32)
    csound = np.sqrt(ic.gamma * pr / rho).astype(np.float32)
    om = O.OracleMesh(m)
    mu_e = np.random.default_rng(3).uniform(0, 2e-3, m.nelem * m.nnode).astype(np.float32)
    tau = O.comp_tau(om, csound, u.reshape(-1))
    Rm, Rq, Re = O.rhs(om, O.comp_params(ic), rho, q, E, mu_e, ic.mu_factor, tau)
    ctx = gpu.Context(m, gpu.phys_from_ic(ic))
    dv = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    d = {k: dv(v) for k, v in dict(rho=rho, q=q, E=E, mu_e=mu_e, tau=tau).items()}
    out = [torch.zeros(n, device="cuda") for n in (N, 3 * N, N)]
    ctx.call("sod_gpu_updateF", gpu.dptr(d["rho"]), gpu.dptr(d["q"]), gpu.dptr(d["E"]), gpu.dptr(d["mu_e"]),
             float(ic.mu_factor), gpu.dptr(d["tau"]), *(gpu.dptr(x) for x in out), None, None, None, None)
    for name, a, b in (("mass", out[0], Rm), ("mom", out[1], Rq), ("ener", out[2], Re)):
        err = rel_l2(a.cpu().numpy(), b)
        print(name, err)
        assert err < TOL, name
    # Laplacian (FP64) against the oracle
    om64 = O.OracleMesh(m, np.float64)
    w = m.lpoin_w - 1
    p = np.zeros(N)
    p[w] = np.random.default_rng(4).normal(size=w.size)
    ref = O.laplacian(om64, p)
    dp, Ap = dv(p), torch.zeros(N, dtype=torch.float64, device="cuda")
    ctx.call("sod_gpu_eval_laplacian_mult64", gpu.dptr(dp), gpu.dptr(Ap))
    assert rel_l2(Ap.cpu().numpy()[w], ref[w]) < 1e-6
    ctx.close()


def test_patch_preconditioner_on_a_non_cubic_mesh(gpu):
    m = box()
    ctx = gpu.Context(m, gpu.default_phys())
    ctx.call("sod_gpu_precond_init", 3, 0)
    n = gpu.lib().sod_gpu_precond_num_params(ctx.h)
    rng = np.random.default_rng(5)
    params = rng.normal(0, 0.2, n)
    o, k = PR.dims(3)[2]["B"]
    params[o:o + k] = rng.normal(0, 0.05, k)
    params = params.astype(np.float32)
    ctx.call("sod_gpu_precond_set_params", params.ctypes.data_as(C.c_void_p), n)
    diag = torch.zeros(m.npoin, device="cuda")
    ctx.call("sod_gpu_eval_laplacian_diag", gpu.dptr(diag))
    net = PR.Net(m, diag.cpu().numpy())
    w = m.lpoin_w - 1
    r = np.zeros(m.npoin)
    r[w] = rng.normal(size=w.size)
    z = torch.zeros(m.npoin, dtype=torch.float64, device="cuda")
    ctx.call("sod_gpu_precond_apply", gpu.dptr(torch.from_numpy(r).cuda()), gpu.dptr(z))
    zr, _ = net.forward(params.astype(np.float64), r)
    err = rel_l2(z.cpu().numpy()[w], zr[w])
    print("apply", err)
    assert err < 3e-3
    ctx.close()


def test_invalid_arguments_return_einval(gpu):
    lib = gpu.lib()
    m = host.periodic_cube(3, 2)
    ctx = gpu.Context(m, gpu.default_phys())
    # unsupported element order at init
    sm = gpu.SodMesh.from_buffer_copy(ctx.sm)
    sm.porder = 5
    h = gpu.VP()
    assert lib.sod_gpu_init(C.byref(sm), C.byref(ctx.phys), C.byref(h)) == EINVAL
    assert b"porder" in lib.sod_gpu_last_error()
    N = m.npoin
    b = torch.zeros(N, dtype=torch.float64, device="cuda")
    x = torch.zeros(N, dtype=torch.float64, device="cuda")
    st = gpu.SolveStats()
    for opts in (gpu.SolveOpts(0, 1e-8, 0, 50, 0), gpu.SolveOpts(10, 0.0, 0, 50, 0),
                 gpu.SolveOpts(10, 1e-8, 2, 50, 0)):
        assert lib.sod_gpu_pressure_solve(ctx.h, gpu.dptr(b), gpu.dptr(x), C.byref(opts), C.byref(st)) == EINVAL
    # learned preconditioner requested before sod_gpu_precond_init
    o = gpu.SolveOpts(10, 1e-8, 1, 50, 0)
    b[m.lpoin_w[0] - 1] = 1.0
    b[m.lpoin_w[1] - 1] = -1.0
    assert lib.sod_gpu_pressure_solve(ctx.h, gpu.dptr(b), gpu.dptr(x), C.byref(o), C.byref(st)) == EINVAL
    assert b"sod_gpu_precond_init" in lib.sod_gpu_last_error()
    # training with nothing harvested
    ctx.call("sod_gpu_precond_init", 1, 4)
    loss = C.c_float()
    assert lib.sod_gpu_precond_train(ctx.h, 1, 1, 1e-3, 1, C.byref(loss)) == EINVAL
    # null pointers
    assert lib.sod_gpu_updateF(ctx.h, None, None, None, None, 1.0, None, None, None, None, None, None, None,
                               None) == EINVAL
    ctx.close()


def test_zero_rhs_gives_zero_solution(gpu):
    m = host.periodic_cube(3, 3)
    ctx = gpu.Context(m, gpu.default_phys())
    N = m.npoin
    b = torch.zeros(N, dtype=torch.float64, device="cuda")
    x = torch.ones(N, dtype=torch.float64, device="cuda")
    st = gpu.SolveStats()
    ctx.call("sod_gpu_pressure_solve", gpu.dptr(b), gpu.dptr(x), C.byref(gpu.SolveOpts(100, 1e-8, 0, 50, 0)),
             C.byref(st))
    assert st.iterations == 0
    assert float(x.abs().max()) == 0.0
    ctx.close()


def test_new_step_entries_reject_missing_state(gpu):
    """The incompressible and IMEX entries refuse to run before their state
    exists, and refuse bad arguments, with an error status (no kernel runs
    on an unset state)."""
    m = host.periodic_cube(3, 2, seed=5)
    ctx = gpu.Context(m, gpu.default_phys())
    dt, out4 = C.c_float(), (C.c_double * 4)()
    its, res = C.c_int(), C.c_double()
    for name, args in (("sod_gpu_incomp_adapt_dt", (0.5, C.byref(dt))), ("sod_gpu_incomp_analysis", (out4,)),
                       ("sod_gpu_incomp_set_pressure", (None,)), ("sod_gpu_incomp_get", (None, None)),
                       ("sod_gpu_comp_imex_step", (1e-3, 200, 1e-3)),
                       ("sod_gpu_comp_imex_stats", (C.byref(its), C.byref(res)))):
        with pytest.raises(RuntimeError):
            ctx.call(name, *args)
    N = m.npoin
    u = torch.zeros(3 * N, device="cuda")
    ctx.call("sod_gpu_incomp_init", gpu.dptr(u), 0.01)
    with pytest.raises(RuntimeError):  # non-positive CFL
        ctx.call("sod_gpu_incomp_adapt_dt", 0.0, C.byref(dt))
    with pytest.raises(RuntimeError):  # unknown preconditioner kind
        ctx.call("sod_gpu_incomp_step", 0.01, C.byref(gpu.SolveOpts(20, 1e-8, 3, 50, 0)), C.byref(gpu.SolveStats()))
    # a zero velocity field: analysis is zero, dt is the initial 1e14
    ctx.call("sod_gpu_incomp_analysis", out4)
    assert list(out4) == [0.0, 0.0, 0.0, 0.0]
    ctx.call("sod_gpu_incomp_adapt_dt", 0.5, C.byref(dt))
    assert dt.value > 1e13
    ctx.close()
