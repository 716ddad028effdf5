"""The plain compressible Taylor-Green case as configured, on the GPU.

Periodic cube [0, 2*3.14159265]^3 of 16^3 HEX64 elements (p = 3, 48^3
unique nodes), Ma = 0.1, gamma = 1.4, Pr = 0.71, Re = 1600, LPS and entropy
viscosity on, SSPRK(4,3) ("RK4", time_integ_ls.f90:99-111) at CFL 0.5,
200 steps, analysis rows every 10 steps (CFDSolverBase.f90:1929-2164).

* GPU all-FP32 (the reference's USE_RP=4 arithmetic) against the oracle in
  FP32: every analysis row within 1e-4 relative (the reference's regression
  tolerance, testcheck.py:5; relative to |value| + 1e-4), rho and E within
  1e-5 relative L2, rho*u within MOM_TOL.
* GPU with FP32 element kernels and FP64 RK state (the production mode)
  against the oracle in FP64: the errors are printed, and bounded by the
  FP32 rounding growth of the Taylor-Green dynamics over 200 steps.

The oracle runs in the test (about half a minute per precision on 16 host
cores).
"""
import numpy as np
import pytest

import oracle as O
from sod2d_b200 import host

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

NSTEPS = 200
# rho*u is the field that FP32 rounding moves most over the 200 steps: two
# FP32 runs with different summation orders (the oracle's and the GPU's)
# drift apart by the same mechanism that separates FP32 from FP64.
MOM_TOL = 1e-4


@pytest.fixture(scope="module")
def gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_b200 import gpu as g
    return g


@pytest.fixture(scope="module")
def case():
    m = host.periodic_cube(3, 16)
    ic = host.tgv_comp_init(m, Ma=0.1)
    return m, ic


def rel(a, b):
    return np.abs(a - b) / (np.abs(b) + 1e-4)


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def fields(m, st):
    w = m.lpoin_w - 1
    N = m.npoin
    return {"rho": st["rho"][w], "rhou": st["q"].reshape(3, N)[:, w], "E": st["E"][w]}


def run_gpu(gpu, m, ic, fp64):
    s = gpu.CompSolver(m, ic, stages=4, fp64_state=fp64)
    hist = s.run(NSTEPS)
    st = s.state()
    s.close()
    return hist, fields(m, st)


def run_oracle(m, ic, dtype):
    hist, fin = O.tgv_comp_run(O.OracleMesh(m, dtype), ic, O.comp_params(ic, stages=4, first_mue=True), NSTEPS)
    return hist, fields(m, fin)


def test_cfg0_fp32_against_fp32_oracle(gpu, case):
    m, ic = case
    ref_hist, ref = run_oracle(m, ic, np.float32)
    hist, got = run_gpu(gpu, m, ic, fp64=False)
    assert hist.shape == ref_hist.shape == (NSTEPS // 10 + 1, 6)  # t = 0, steps 1, 11, ..., 191
    r = rel(hist, ref_hist)
    errs = {k: rel_l2(got[k], ref[k]) for k in got}
    print("FP32 GPU vs FP32 oracle: max rel per analysis column", r.max(0), "field rel L2", errs)
    assert r.max() < 1e-4
    assert errs["rho"] < 1e-5 and errs["E"] < 1e-5
    assert errs["rhou"] < MOM_TOL


def test_cfg0_fp64_state_against_fp64_oracle(gpu, case):
    m, ic = case
    ref_hist, ref = run_oracle(m, ic, np.float64)
    hist, got = run_gpu(gpu, m, ic, fp64=True)
    assert hist.shape == ref_hist.shape
    # errors relative to each column's peak (eps_D starts at zero and stays
    # near FP32 noise at Ma = 0.1)
    peak_err = np.abs(hist - ref_hist).max(0) / np.abs(ref_hist).max(0)
    errs = {k: rel_l2(got[k], ref[k]) for k in got}
    print("FP32 kernels + FP64 state vs FP64 oracle: max error / column peak", peak_err, "field rel L2", errs)
    assert peak_err[1] < 1e-3 and peak_err[2] < 1e-4 and peak_err[4] < 1e-4  # EK, eps_S, eps_T
    assert errs["rho"] < 1e-4 and errs["E"] < 1e-4 and errs["rhou"] < 1e-3
