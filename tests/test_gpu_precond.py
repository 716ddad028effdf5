"""Learned preconditioner on the GPU: inference, forward and backward kernels
against the numpy restatement (P=3 and P=4, shuffled element and node
numbering), and the gain of the trained network over Jacobi inside the
FP64-certified CG on pressure systems of an incompressible Taylor-Green
run."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import precond_ref as PR
from sod2d_b200 import host

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_b200 import gpu as g
    return g


def _random_params(P, seed):
    rng = np.random.default_rng(seed)
    off = PR.dims(P)[2]
    p = rng.normal(0, 0.2, PR.num_params(P))
    o, n = off["B"]
    p[o:o + n] = rng.normal(0, 0.05, n)
    return p.astype(np.float32)


@pytest.mark.parametrize("porder", [3, 4])
def test_loss_and_gradient_match_oracle(gpu, porder):
    m = host.periodic_cube(porder, 4, jitter=0.05, seed=6, ordering=1, elem_shuffle=True)
    ctx = gpu.Context(m, gpu.default_phys())
    ctx.call("sod_gpu_precond_init", 7, 0)
    n = gpu.lib().sod_gpu_precond_num_params(ctx.h)
    assert n == PR.num_params(porder)
    params = _random_params(porder, 3)
    ctx.call("sod_gpu_precond_set_params", params.ctypes.data_as(C.c_void_p), n)
    om = O.OracleMesh(m, np.float64)
    diag = torch.zeros(m.npoin, device="cuda")
    ctx.call("sod_gpu_eval_laplacian_diag", gpu.dptr(diag))
    w = m.lpoin_w - 1
    net = PR.Net(m, diag.cpu().numpy())
    rng = np.random.default_rng(3)
    e = np.zeros(m.npoin)
    e[w] = rng.normal(size=w.size)
    r = O.laplacian(om, e)
    dr, de = torch.from_numpy(r).cuda(), torch.from_numpy(e).cuda()
    # inference (tensor cores, TF32 operands with FP32 accumulation: ~1e-3)
    z = torch.zeros(m.npoin, dtype=torch.float64, device="cuda")
    ctx.call("sod_gpu_precond_apply", gpu.dptr(dr), gpu.dptr(z))
    zr, _ = net.forward(params.astype(np.float64), r)
    zerr = np.linalg.norm(z.cpu().numpy()[w] - zr[w]) / np.linalg.norm(zr[w])
    print("apply rel L2", zerr)
    assert zerr < 3e-3
    # loss and gradient (FP32 forward and backward kernels)
    ref_loss, ref_grad = net.loss_grad(params.astype(np.float64), r, e, lambda v: O.laplacian(om, v))
    loss = C.c_double()
    grad = np.zeros(n, np.float32)
    ctx.call("sod_gpu_precond_loss_grad", gpu.dptr(dr), gpu.dptr(de), C.byref(loss), grad.ctypes.data_as(C.c_void_p))
    print("loss", loss.value, ref_loss)
    assert abs(loss.value - ref_loss) / ref_loss < 1e-4
    off = PR.dims(porder)[2]
    for name, (o, k) in off.items():
        err = np.linalg.norm(grad[o:o + k] - ref_grad[o:o + k]) / max(np.linalg.norm(ref_grad[o:o + k]), 1e-30)
        print("grad", name, "rel L2", err)
        assert err < 1e-3, name
    ctx.close()


def test_trained_network_beats_jacobi(gpu):
    m = host.periodic_cube(3, 8)
    N = m.npoin
    x, y, z = (m.coord[i * N:(i + 1) * N].astype(np.float64) for i in range(3))
    u = np.concatenate([np.sin(x) * np.cos(y) * np.cos(z), -np.cos(x) * np.sin(y) * np.cos(z),
                        np.zeros(N)]).astype(np.float32)
    ctx = gpu.Context(m, gpu.default_phys())
    ctx.call("sod_gpu_precond_init", 11, 48)
    du = torch.from_numpy(u).cuda()
    ctx.call("sod_gpu_incomp_init", gpu.dptr(du), 1.0 / 1600.0)
    dt = 0.02
    jac = gpu.SolveOpts(20000, 1e-8, 0, 100, 1)
    st = gpu.SolveStats()
    its_j = []
    for k in range(12):  # Jacobi steps, harvesting
        ctx.call("sod_gpu_incomp_step", dt, C.byref(jac), C.byref(st))
        its_j.append(st.iterations)
        assert st.res_rel < 1e-8
    assert gpu.lib().sod_gpu_precond_harvest_count(ctx.h) > 10
    loss = C.c_float()
    ctx.call("sod_gpu_precond_train", 300, 8, 3e-3, 5, C.byref(loss))
    print("Jacobi iterations", its_j, "final training loss", loss.value)
    # a pressure system of the current flow state (first-order explicit
    # predictor), solved from the same zero initial guess by both
    uu = torch.zeros(3 * N, device="cuda")
    ctx.call("sod_gpu_incomp_get", gpu.dptr(uu), None)
    R = torch.zeros(3 * N, device="cuda")
    ctx.call("sod_gpu_full_convec_ijk_incomp", gpu.dptr(uu), gpu.dptr(uu), gpu.dptr(R))
    L = torch.zeros(3 * N, device="cuda")
    for d in range(3):
        ctx.call("sod_gpu_eval_laplacian_mult", gpu.dptr(uu[d * N:]), gpu.dptr(L[d * N:]))
    invMl = torch.from_numpy(m.invMl).cuda().repeat(3)
    us = uu - dt * (R + (1.0 / 1600.0) * L) * invMl
    div = torch.zeros(N, device="cuda")
    ctx.call("sod_gpu_eval_divergence", gpu.dptr(us), gpu.dptr(div))
    b = (-div.double() / dt).contiguous()
    out = {}
    for name, kind in (("jacobi", 0), ("learned", 1)):
        x0 = torch.zeros(N, dtype=torch.float64, device="cuda")
        o = gpu.SolveOpts(20000, 1e-8, kind, 200, 0)
        st = gpu.SolveStats()
        ctx.call("sod_gpu_pressure_solve", gpu.dptr(b), gpu.dptr(x0), C.byref(o), C.byref(st))
        out[name] = (st.iterations, st.res_rel, st.fallback, st.seconds)
    print("jacobi:", out["jacobi"], " learned:", out["learned"])
    assert out["learned"][1] < 1e-8 and out["learned"][2] == 0
    assert out["learned"][0] < 0.6 * out["jacobi"][0]
    ctx.close()


def test_self_harvest_finetune(gpu):
    """Pairs harvested from the learned solver's own iterations (after
    sod_gpu_precond_restart_harvest) fine-tune the map; the fine-tuned map
    still certifies every solve and needs no more iterations than before."""
    m = host.periodic_cube(3, 8)
    N = m.npoin
    x, y, z = (m.coord[i * N:(i + 1) * N].astype(np.float64) for i in range(3))
    u = np.concatenate([np.sin(x) * np.cos(y) * np.cos(z), -np.cos(x) * np.sin(y) * np.cos(z),
                        np.zeros(N)]).astype(np.float32)
    ctx = gpu.Context(m, gpu.default_phys())
    ctx.call("sod_gpu_precond_init", 11, 96)
    du = torch.from_numpy(u).cuda()
    ctx.call("sod_gpu_incomp_init", gpu.dptr(du), 1.0 / 1600.0)
    dt = 0.02
    st = gpu.SolveStats()
    for k in range(10):
        ctx.call("sod_gpu_incomp_step", dt, C.byref(gpu.SolveOpts(20000, 1e-8, 0, 100, 1)), C.byref(st))
    loss = C.c_float()
    ctx.call("sod_gpu_precond_train", 300, 8, 3e-3, 5, C.byref(loss))
    with pytest.raises(RuntimeError):  # no context
        gpu.check(gpu.lib().sod_gpu_precond_restart_harvest(None), "sod_gpu_precond_restart_harvest")
    ctx.call("sod_gpu_precond_restart_harvest")
    assert gpu.lib().sod_gpu_precond_harvest_count(ctx.h) == 0
    its_before = []
    for k in range(4):
        ctx.call("sod_gpu_incomp_step", dt, C.byref(gpu.SolveOpts(20000, 1e-8, 1, 200, 1)), C.byref(st))
        assert st.res_rel < 1e-8 and st.fallback == 0
        its_before.append(st.iterations)
    n_pairs = gpu.lib().sod_gpu_precond_harvest_count(ctx.h)
    assert n_pairs >= 4 * 9  # iterations 0-8 of every learned solve at least
    ctx.call("sod_gpu_precond_train", 200, 8, 5e-4, 11, C.byref(loss))
    its_after = []
    for k in range(4):
        ctx.call("sod_gpu_incomp_step", dt, C.byref(gpu.SolveOpts(20000, 1e-8, 1, 200, 0)), C.byref(st))
        assert st.res_rel < 1e-8 and st.fallback == 0
        its_after.append(st.iterations)
    print("learned iterations before fine-tuning", its_before, "after", its_after, "pairs", n_pairs)
    assert np.mean(its_after) <= 1.1 * np.mean(its_before)
    ctx.close()
