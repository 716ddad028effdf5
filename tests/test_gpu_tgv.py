"""Full compressible Taylor-Green time loop on the GPU against the oracle.

The GPU loop (FP32 state, the reference's USE_RP=4 arithmetic) and the
oracle run the same steps from the same initial state; their analysis
histories (EK, eps_S, eps_D, eps_T, max Mach) must agree to 1e-4 relative
(the reference's own regression tolerance, testcheck.py:5) and the final
conserved fields to 1e-4 relative L2.  The t=0 row is checked against the
reference's history file.
"""
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from sod2d_b200 import host

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_b200 import gpu as g
    return g


def rel(a, b):
    return np.abs(a - b) / (np.abs(b) + 1e-4)


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


@pytest.mark.parametrize("porder,n,Ma,stages,nsteps", [(4, 8, 1.25, 5, 21), (3, 8, 0.1, 4, 21)])
def test_tgv_history_matches_oracle(gpu, porder, n, Ma, stages, nsteps):
    m = host.periodic_cube(porder, n)
    ic = host.tgv_comp_init(m, Ma=Ma)
    om = O.OracleMesh(m)
    ref_hist, ref_fin = O.tgv_comp_run(om, ic, O.comp_params(ic, stages=stages, first_mue=True), nsteps)
    s = gpu.CompSolver(m, ic, stages=stages, fp64_state=False)
    hist = s.run(nsteps)
    fin = s.state()
    s.close()
    assert hist.shape == ref_hist.shape
    r = rel(hist, ref_hist)
    print("max rel per column:", r.max(0))
    assert r.max() < 1e-4
    w = m.lpoin_w - 1
    for k in ("rho", "E"):
        assert rel_l2(fin[k][w], ref_fin[k][w]) < 1e-5, k
    if porder == 4 and n == 8 and Ma == 1.25:
        gold = O.load_history(GOLD / "tgv_comp_cpu_lsrk5_8x8x8_p4.dat")
        assert rel(hist[0], gold[0]).max() < 2e-6
        assert abs(hist[1, 0] - gold[1, 0]) / gold[1, 0] < 1e-6


def test_fp64_state_close_to_fp32(gpu):
    """FP64 RK accumulation stays within FP32 round-off growth of the FP32 run."""
    m = host.periodic_cube(3, 6)
    ic = host.tgv_comp_init(m, Ma=0.1)
    a = gpu.CompSolver(m, ic, stages=4, fp64_state=False)
    ha = a.run(10)
    a.close()
    b = gpu.CompSolver(m, ic, stages=4, fp64_state=True)
    hb = b.run(10)
    b.close()
    assert rel(hb, ha).max() < 1e-4


@pytest.mark.parametrize("porder,Ma,stages", [(4, 1.25, 4), (4, 1.25, 3), (3, 0.1, 4)])
def test_imex_history_matches_oracle(gpu, porder, Ma, stages):
    """IMEX integrator (imex_main with conjGrad_imex) on the reference's
    IMEX test case (8^3 order-4 cube, Ma = 1.25, CFL 0.95) and on an
    order-3 cube at Ma = 0.1: the GPU
    analysis rows agree with the oracle's to 1e-4 relative, the final
    conserved fields to 1e-5 relative L2; with stages = 4 the first step's
    time is the reference history's."""
    m = host.periodic_cube(porder, 8)
    ic = host.tgv_comp_init(m, Ma=Ma)
    om = O.OracleMesh(m)
    nsteps = 21
    prm = O.comp_params(ic, cfl_conv=0.95, cfl_diff=1000.5, stages=stages, imex=True, first_mue=True)
    ref_hist, ref_fin = O.tgv_comp_run(om, ic, prm, nsteps)
    s = gpu.CompSolver(m, ic, stages=stages, fp64_state=False, cfl_conv=0.95, cfl_diff=1000.5, imex=True)
    hist = s.run(nsteps)
    fin = s.state()
    its, res = gpu.C.c_int(), gpu.C.c_double()
    s.ctx.call("sod_gpu_comp_imex_stats", gpu.C.byref(its), gpu.C.byref(res))
    s.close()
    assert hist.shape == ref_hist.shape
    r = rel(hist, ref_hist)
    print("IMEX stages", stages, "max rel per column:", r.max(0), "CG iterations of the last step", its.value,
          "residual", res.value)
    assert r.max() < 1e-4
    w = m.lpoin_w - 1
    for k in ("rho", "E"):
        assert rel_l2(fin[k][w], ref_fin[k][w]) < 1e-5, k
    assert its.value >= stages - 1 and res.value < 1e-3
    if stages == 4 and porder == 4:
        gold = O.load_history(GOLD / "tgv_comp_cpu_imex4_8x8x8_p4.dat")
        assert abs(hist[1, 0] - gold[1, 0]) / gold[1, 0] < 1e-6


def test_imex_arguments(gpu):
    m = host.periodic_cube(3, 2)
    ic = host.tgv_comp_init(m, Ma=0.1)
    s = gpu.CompSolver(m, ic, stages=5, fp64_state=False)
    with pytest.raises(RuntimeError):  # five stages: no IMEX table
        s.ctx.call("sod_gpu_comp_imex_step", 1e-3, 200, 1e-3)
    s.close()
    s = gpu.CompSolver(m, ic, stages=4, fp64_state=True)
    with pytest.raises(RuntimeError):  # FP64 state
        s.ctx.call("sod_gpu_comp_imex_step", 1e-3, 200, 1e-3)
    s.close()
    s = gpu.CompSolver(m, ic, stages=4, fp64_state=False)
    for args in ((0.0, 200, 1e-3), (1e-3, 0, 1e-3), (1e-3, 200, 0.0)):
        with pytest.raises(RuntimeError):
            s.ctx.call("sod_gpu_comp_imex_step", *args)
    s.close()
