"""The C-ABI from a compiled, non-Python caller (tests/abi_harness.cpp): the
mesh and state go in as flat host arrays of the reference's Fortran layout,
as a Fortran solver would hold them; the residuals the harness writes back
match the oracle to 1e-5 relative L2.  Compiled with g++ against
libsod2d_gpu.so and the CUDA runtime."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from sod2d_b200 import host

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
CUDA = Path("/usr/local/cuda")


@pytest.fixture(scope="module")
def gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_b200 import gpu as g
    return g


def test_cpp_caller_matches_oracle(gpu):
    out = ROOT / "tests" / "_build" / "abi"
    out.mkdir(parents=True, exist_ok=True)
    lib = gpu.lib_path().parent
    exe = out / "abi_harness"
    subprocess.run(["g++", "-O2", "-std=c++17", str(ROOT / "tests" / "abi_harness.cpp"), f"-I{ROOT / 'include'}",
                    f"-I{CUDA / 'include'}", f"-L{lib}", "-lsod2d_gpu", f"-L{CUDA / 'lib64'}", "-lcudart",
                    f"-Wl,-rpath,{lib}", f"-Wl,-rpath,{CUDA / 'lib64'}", "-o", str(exe)], check=True)

    m = host.periodic_cube(3, 4, jitter=0.05, seed=51, ordering=1, elem_shuffle=True)
    ic = host.tgv_comp_init(m, Ma=0.1)
    rho, q, E = host.random_comp_state(m, seed=52)
    N = m.npoin
    u = (q.reshape(3, N) / rho).astype(np.float32).reshape(-1)
    csound = np.full(N, 10.0, np.float32)
    mu_e = np.random.default_rng(53).uniform(0, 2e-3, m.nelem * m.nnode).astype(np.float32)
    ph = gpu.phys_from_ic(ic)
    phys = np.array([getattr(ph, f) for f, _ in ph._fields_], np.float32)
    (out / "sizes.txt").write_text(f"{m.porder} {m.nelem} {m.npoin} {m.npoin_w}\n")
    arrays = dict(connec=(m.connecWork, np.int32), lpoin_w=(m.lpoin_w, np.int32),
                  invAtoIJK=(m.invAtoIJK, np.int32), gmshAtoI=(m.gmshAtoI, np.int32),
                  gmshAtoJ=(m.gmshAtoJ, np.int32), gmshAtoK=(m.gmshAtoK, np.int32),
                  dlxigp_ip=(m.dlxigp_ip, np.float32), He=(m.He, np.float32), gpvol=(m.gpvol, np.float32),
                  Ml=(m.Ml, np.float32), invMl=(m.invMl, np.float32), helem=(m.helem, np.float32),
                  helem_l=(m.helem_l, np.float32), lelpn=(m.lelpn, np.int32), Ngp=(m.Ngp, np.float32),
                  phys=(phys, np.float32), rho=(rho, np.float32), q=(q, np.float32), E=(E, np.float32),
                  u=(u, np.float32), csound=(csound, np.float32), mu_e=(mu_e, np.float32),
                  mu_factor=(np.array([ic.mu_factor]), np.float32))
    for name, (a, dt) in arrays.items():
        np.ascontiguousarray(a, dt).tofile(out / f"{name}.bin")
    p = subprocess.run([str(exe), str(out)], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    got = [np.fromfile(out / f"{n}.bin", np.float32) for n in ("Rmass", "Rmom", "Rener")]

    om = O.OracleMesh(m)
    tau = O.comp_tau(om, csound, u)
    ref = O.rhs(om, O.comp_params(ic), rho, q, E, mu_e, ic.mu_factor, tau)
    w = m.lpoin_w - 1
    for name, g, r, k in zip(("mass", "momentum", "energy"), got, ref, (1, 3, 1)):
        g = g.reshape(k, N)[:, w].astype(np.float64)
        r = np.asarray(r).reshape(k, N)[:, w]
        err = np.linalg.norm(g - r) / np.linalg.norm(r)
        print(f"C++ caller {name}: rel L2 {err:.2e}")
        assert err < 1e-5, name
