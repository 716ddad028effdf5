"""The allocation-free analysis entry point (sod_gpu_analysis_noalloc).

Callers that cannot allocate device memory -- a solver whose device memory
belongs to its own pool, or callers that must not let cudaMalloc synchronise
the device inside the time loop -- get the analysis integrals through this
entry point, which keeps its scratch in a fixed device array.  This test
calls it through the C-ABI on the state of a short Taylor-Green run, for
element orders 3 and 4, and compares it, on two calls in a row (the second
reuses the scratch the first left behind), with the context-based
sod_gpu_comp_analysis.  Tolerance: 1e-5 relative, as the other FP32 parity
tests.  The free device memory after the second call equals that after the
first: the call allocates nothing.  The file is collected last.
"""
import ctypes as C

import numpy as np
import pytest

from sod2d_b200 import host

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.fixture(scope="module")
def gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_b200 import gpu as g
    return g


@pytest.mark.parametrize("porder,nelem1d", [(3, 6), (4, 4)])
def test_noalloc_analysis_matches_context_entry_point(gpu, porder, nelem1d):
    m = host.periodic_cube(porder, nelem1d, jitter=0.05, seed=21, ordering=1)
    ic = host.tgv_comp_init(m, Ma=0.1)
    s = gpu.CompSolver(m, ic, stages=4, fp64_state=False)
    for _ in range(3):  # non-zero entropy viscosity
        s.step()
        s.dt = s.adapt_dt()
    ref = np.array(s.analysis()[1:])
    st = s.state()
    s.close()

    # primitive fields at the same state, as the library's end-of-step EOS
    N = m.npoin
    f32 = np.float32
    rho, q, E = st["rho"], st["q"].reshape(3, N), st["E"]
    u = (q / rho).astype(f32)
    umag = (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]).astype(f32)
    eint = (E / rho - f32(0.5) * umag).astype(f32)
    pr = (rho * f32(ic.gamma - 1.0) * eint).astype(f32)
    c = np.sqrt(f32(ic.gamma) * pr / rho).astype(f32)
    machno = (np.sqrt(umag) / c).astype(f32)
    T = (pr / (rho * f32(ic.Rgas))).astype(f32)
    mu = (f32(ic.mu_factor) * f32(1.458e-6) * np.power(T, f32(1.5)) / (T + f32(110.4))).astype(f32)

    dv = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    d = {k: dv(getattr(m, k)) for k in ("connecWork", "lpoin_w", "invAtoIJK", "gmshAtoI", "gmshAtoJ", "gmshAtoK",
                                         "dlxigp_ip", "He", "gpvol", "Ngp")}
    fields = {k: dv(v) for k, v in dict(rho=rho, u=u.reshape(-1), mu=mu, mu_e=st["mu_e"], machno=machno).items()}
    volT = float(np.float32(m.vol_total))
    torch.cuda.synchronize()

    def call(nelem=m.nelem):
        out = (C.c_double * 5)()
        rc = gpu.lib().sod_gpu_analysis_noalloc(
            m.porder, nelem, N, m.npoin_w, *(gpu.dptr(d[k]) for k in (
                "connecWork", "lpoin_w", "invAtoIJK", "gmshAtoI", "gmshAtoJ", "gmshAtoK", "dlxigp_ip", "He",
                "gpvol", "Ngp")),
            *(gpu.dptr(fields[k]) for k in ("rho", "u", "mu", "mu_e", "machno")),
            float(ic.rho0), volT, None, out)
        return rc, np.array(out[:])

    free_after = []
    for attempt in range(2):  # two calls in a row share the scratch
        rc, got = call()
        assert rc == 0, gpu.lib().sod_gpu_last_error()
        free_after.append(torch.cuda.mem_get_info()[0])
        rel = np.abs(got - ref) / np.abs(ref)
        print(f"p={porder} call {attempt}: rel diff {rel}")
        assert rel.max() < TOL, (got, ref)
    # the first call may load the library's device code into this context;
    # the second finds nothing more to set up and must allocate nothing
    assert free_after[1] == free_after[0], free_after

    # sizes beyond the fixed scratch are rejected with a clear error
    rc, _ = call(nelem=(1 << 20) + 1)
    assert rc == -1
    assert b"SOD_NOALLOC_MAX_ELEM" in gpu.lib().sod_gpu_last_error()
