"""The fused compressible RHS at the benchmark's full size: the 64^3 HEX64
jittered cube with the random state of `bench.py` (7,077,888 working
nodes).  The oracle's FP32 RHS (OpenMP) finishes it in seconds, so the
full-size check is parity itself: every residual within 1e-5 relative L2
of the oracle, and two evaluations bit-identical (deterministic assembly,
no floating-point atomics)."""
import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_b200 import gpu as g
    return g


def test_full_size_rhs_parity_and_determinism(gpu):
    import bench  # the benchmark's own workload builder
    m, ic, rho, q, E, mu_e, u, csound = bench.build_workload(64)
    N = m.npoin
    ctx = gpu.Context(m, gpu.phys_from_ic(ic))
    dv = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    d = [dv(a) for a in (rho, q, E, mu_e, u, csound)]
    tau = torch.zeros(m.nelem, device="cuda")
    ctx.call("sod_gpu_comp_tau", gpu.dptr(d[5]), gpu.dptr(d[4]), gpu.dptr(tau))
    runs = []
    for _ in range(2):
        out = [torch.zeros(n, device="cuda") for n in (N, 3 * N, N)]
        ctx.call("sod_gpu_updateF", gpu.dptr(d[0]), gpu.dptr(d[1]), gpu.dptr(d[2]), gpu.dptr(d[3]),
                 float(ic.mu_factor), gpu.dptr(tau), *(gpu.dptr(x) for x in out), None, None, None, None)
        runs.append([x.cpu().numpy() for x in out])
    tau_h = tau.cpu().numpy()
    ctx.close()
    for a, b in zip(*runs):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    om = O.OracleMesh(m)
    tau_ref = O.comp_tau(om, csound, u)
    assert np.abs(tau_h - tau_ref).max() <= 1e-6 * np.abs(tau_ref).max()
    ref = O.rhs(om, O.comp_params(ic), rho, q, E, mu_e, ic.mu_factor, tau_ref)
    w = m.lpoin_w - 1
    for name, g, r, k in zip(("mass", "momentum", "energy"), runs[0], ref, (1, 3, 1)):
        g = g.reshape(k, N)[:, w].astype(np.float64)
        r = np.asarray(r).reshape(k, N)[:, w]
        err = np.linalg.norm(g - r) / np.linalg.norm(r)
        print(f"64^3 {name}: rel L2 {err:.2e}")
        assert err < 1e-5, name
