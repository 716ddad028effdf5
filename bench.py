"""Benchmark of the SOD2D spectral-element RHS hot path on B200.

Workload (RHS micro-benchmark): periodic cube of 64^3 hexahedra of order 3
(HEX64, GLL nodes, 192^3 = 7,077,888 unique nodes) with element-interior GLL
nodes jittered by a seeded uniform +-5% of the local spacing; random FP32
conserved state rho ~ U[0.9,1.1], momentum rho*U[-1,1]^3, energy from
p ~ U[0.9,1.1]*p0 (p0 = 1/(gamma Ma^2), Ma = 0.1); element viscosity
mu_e ~ U[0, 2e-3] (seeded).  One step = one fused RHS evaluation
(sod_gpu_updateF: equation of state, Sutherland viscosity, convection, LPS
projection, stabilised diffusion, deterministic assembly and lumped-mass
inversion) over device-resident inputs.

Metric: node-stages/s = working nodes x RHS evaluations / s (reported in
Mnode-stages/s), with the HBM roofline fraction computed from the
algorithmic traffic of 402 B per node-stage (p=3: per unique node the two
element passes read the state twice (40 B), write and re-read the 15
projections (120 B), read invMl and write 5 residuals (24 B); per element
they read He+gpvol twice, the connectivity twice and mu_e once, 5888 B per
element = 218 B per node).

--impl reference times the CPU restatement of the reference's FP32 path
(the oracle, OpenMP over all host cores; the Fortran reference cannot be
built here) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

B_PER_NODE_STAGE = 402.0
# DRAM bytes (read + write) of one RHS evaluation per working node, from one
# ncu capture of the four RHS kernels on the 64^3 workload itself
# (5,535,995,392 B for 7,077,888 working nodes).
DRAM_B_PER_NODE_STAGE = 5535995392 / 7077888
NELEM_1D = 64
PORDER = 3


def max_over_ranks(ms: float, world: int, device: str) -> float:
    """Time of the slowest rank (every rank calls this collectively)."""
    if world == 1:
        return float(ms)
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world: int, units_per_rank: int, steps: int, ms: float) -> float:
    """Whole-job rate in millions of units per second: every rank processes
    units_per_rank units per step (replicas, weak scaling); ms is the time of
    the slowest rank."""
    return world * units_per_rank * steps / (ms / 1e3) / 1e6


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """Samples SM clocks and clock-event (throttle) reasons during the timed
    region: NVML every 10 ms (read-only queries), else nvidia-smi every
    200 ms."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index: int):
        self.index = index
        self.sm, self.mx, self.reasons = [], [], set()
        self._stop = threading.Event()
        self._t = None
        self.source = "nvidia-smi"
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self._bits = [pynvml.nvmlClocksEventReasonHwSlowdown, pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                          pynvml.nvmlClocksEventReasonSwThermalSlowdown, pynvml.nvmlClocksEventReasonSwPowerCap]
            self.source = "nvml"
        except Exception:
            self._nv = None

    def _sample_nvml(self):
        nv, h = self._nv, self._h
        self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
        self.mx.append(float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)))
        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        for name, bit in zip(self.NAMES, self._bits):
            if r & bit:
                self.reasons.add(name)

    def _sample_smi(self):
        out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                              "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
        parts = [x.strip() for x in out.stdout.strip().split(",")]
        if len(parts) >= 7:
            if parts[0].replace(".", "").isdigit():
                self.sm.append(float(parts[0]))
            if parts[1].replace(".", "").isdigit():
                self.mx.append(float(parts[1]))
            for i in range(4):
                if parts[3 + i].lower() == "active":
                    self.reasons.add(self.NAMES[i])

    def _run(self):
        while not self._stop.is_set():
            try:
                self._sample_nvml() if self._nv else self._sample_smi()
            except Exception:
                pass
            self._stop.wait(0.01 if self._nv else 0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "source": self.source}
        return {"sm_mhz": statistics.median(self.sm), "sm_max_mhz": max(self.mx) if self.mx else None,
                "reasons": sorted(self.reasons), "samples": len(self.sm), "source": self.source}


def build_workload(nelem_1d: int, seed: int = 2024):
    from sod2d_b200 import host
    m = host.periodic_cube(PORDER, nelem_1d, jitter=0.05, seed=seed)
    rho, q, E = host.random_comp_state(m, seed=seed + 1)
    ic = host.tgv_comp_init(m, Ma=0.1)
    rng = np.random.default_rng(seed + 2)
    mu_e = rng.uniform(0.0, 2e-3, m.nelem * m.nnode).astype(np.float32)
    N = m.npoin
    u = (q.reshape(3, N) / rho).astype(np.float32)
    eint = E / rho - 0.5 * (u.astype(np.float64) ** 2).sum(0)
    pr = rho * (ic.gamma - 1.0) * eint
    csound = np.sqrt(ic.gamma * pr / rho).astype(np.float32)
    return m, ic, rho, q, E, mu_e, u.reshape(-1), csound


class CpuBaseline:
    """The oracle's FP32 RHS (OpenMP over all host cores) on the benchmarked
    workload itself (the same nelem1d^3 jittered cube and state); a bounded
    number of whole-mesh evaluations is timed."""

    def __init__(self, nelem1d=NELEM_1D):
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O
        self.O = O
        self.NELEM_1D = nelem1d
        m, ic, rho, q, E, mu_e, u, csound = build_workload(nelem1d)
        self.m, self.ic, self.args = m, ic, (rho, q, E, mu_e)
        self.om = O.OracleMesh(m)
        self.tau = O.comp_tau(self.om, csound, u)
        self.prm = O.comp_params(ic)
        self.cores = os.cpu_count() or 1

    def step(self):
        rho, q, E, mu_e = self.args
        t0 = time.perf_counter()
        self.O.rhs(self.om, self.prm, rho, q, E, mu_e, self.ic.mu_factor, self.tau)
        return time.perf_counter() - t0

    def sample(self, min_seconds=10.0, max_evals=50):
        self.step()  # warm-up
        times = []
        while sum(times) < min_seconds and len(times) < max_evals:
            times.append(self.step())
        dt = sum(times)
        val = self.m.npoin_w * len(times) / dt / 1e6
        return {"value": round(val, 3), "unit": "Mnode-stages/s", "cores": self.cores, "kind": "port",
                "sample": f"oracle FP32 RHS (OpenMP, {self.cores} threads) on a {self.NELEM_1D}^3 HEX64 jittered "
                          f"cube, {self.m.npoin_w} working nodes x {len(times)} evaluations in {dt:.1f} s"}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    cb = CpuBaseline(args.nelem1d)
    for _ in range(args.warmup):
        cb.step()
    times = [cb.step() for _ in range(args.steps)]
    v = cb.m.npoin_w * len(times) / sum(times) / 1e6
    info = {"value": round(v, 3), "unit": "Mnode-stages/s", "cores": cb.cores, "kind": "port",
            "sample": f"oracle FP32 RHS (OpenMP, {cb.cores} threads) on a {cb.NELEM_1D}^3 HEX64 jittered cube, "
                      f"{cb.m.npoin_w} working nodes per step, {len(times)} steps in {sum(times):.1f} s"}
    line = {"impl": "reference", "metric": "Mnode-stages/s (fused compressible RHS, FP32)", "value": round(v, 3),
            "unit": "Mnode-stages/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * sum(times) / len(times), 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": workload_config(args.nelem1d),
            "cpu_baseline": info, "e2e": {"value": round(v, 3), "unit": "Mnode-stages/s", "h2d_bytes_per_step": 0,
                                          "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def pressure_leg(nelem1d=32, harvest_steps=200, compare_steps=800, dt=None, train_steps=300, lr=1e-3, capacity=256,
                 self_steps=16, ft_steps=200, ft_lr=5e-4, ft_batch=8, extrap_arm=True):
    """Pressure-Poisson solve to a 1e-8 FP64-certified relative residual on
    the incompressible Taylor-Green vortex (periodic cube nelem1d^3 HEX64,
    Re=1600): Jacobi-preconditioned flexible CG from the previous pressure
    (the reference's initial guess), Jacobi-preconditioned CG from the
    learned path's guess 2 p^n - p^(n-1), and the learned element-patch
    preconditioner from that guess, each on its own trajectory of the
    BDF3/EXT3 incompressible step (with its implicit velocity solve) from the
    same initial velocity.  The first `harvest_steps` steps (200) run Jacobi
    and harvest (residual, error) pairs; the network is then trained on the
    GPU.  The next `compare_steps` solves (800) are timed on both
    trajectories (device time of each solve), with the velocity divergence
    after each step; on the learned trajectory the first `self_steps` (16)
    of them also harvest pairs from the learned solver's own iterations, and
    the network is fine-tuned on those (`ft_steps` Adam steps) before the
    rest.  Training and fine-tuning time is reported apart from the solves,
    and `speedup_wall_amortized` charges it, with the extra solve time of
    the harvesting steps, to the learned path.  `extrap_arm` False leaves out
    the Jacobi trajectory from the extrapolated guess (large meshes, where
    every arm costs minutes)."""
    import ctypes as C
    import torch
    from sod2d_b200 import gpu, host
    if dt is None:  # 0.01 on the 32^3 mesh, the same convective CFL on finer meshes
        dt = 0.01 * 32 / nelem1d
    m = host.periodic_cube(PORDER, nelem1d)
    N = m.npoin
    x, y, z = (m.coord[i * N:(i + 1) * N].astype(np.float64) for i in range(3))
    u0 = torch.from_numpy(np.concatenate([np.sin(x) * np.cos(y) * np.cos(z), -np.cos(x) * np.sin(y) * np.cos(z),
                                          np.zeros(N)]).astype(np.float32)).cuda()
    nu = 1.0 / 1600.0
    # ctxs[0]: learned trajectory (harvests during the Jacobi steps);
    # ctxs[1]: Jacobi from the previous pressure (the reference's guess);
    # ctxs[2]: Jacobi from the learned path's guess 2 p^n - p^(n-1)
    ctxs = [gpu.Context(m, gpu.default_phys()) for _ in range(3 if extrap_arm else 2)]
    for c in ctxs:
        c.call("sod_gpu_incomp_init", gpu.dptr(u0), nu)
    ctxs[0].call("sod_gpu_precond_init", 2024, capacity)
    st = gpu.SolveStats()
    harvest_ms = [0.0, 0.0]  # device time of the harvesting and of the plain Jacobi solves
    for k in range(harvest_steps):
        for i, c in enumerate(ctxs):
            o = gpu.SolveOpts(50000, 1e-8, 3 if i == 2 else 0, 100, 1 if i == 0 else 0)
            c.call("sod_gpu_incomp_step", dt, C.byref(o), C.byref(st))
            if i < 2:
                harvest_ms[i] += st.seconds * 1e3
    loss = C.c_float()
    t0 = time.perf_counter()
    ctxs[0].call("sod_gpu_precond_train", train_steps, 16, lr, 7, C.byref(loss))
    train_s = time.perf_counter() - t0
    res = {}
    uu = torch.zeros(3 * N, device="cuda")
    div = torch.zeros(N, device="cuda")
    w = torch.from_numpy((m.lpoin_w - 1).astype(np.int64)).cuda()
    ft_s, ft_loss, ft_pairs = 0.0, C.c_float(), 0
    peak_used = [0]  # device memory in use (all contexts and torch), sampled every 50 steps
    arms = (("jacobi", 0), ("jacobi_extrapolated_guess", 3), ("learned", 1))
    for i, (name, kind) in enumerate(a for a in arms if extrap_arm or a[1] != 3):
        c = {0: ctxs[1], 3: ctxs[-1], 1: ctxs[0]}[kind]
        it, ms, rmax, fb, dv, vits, step_ms = [], [], 0.0, 0, [], [], []
        vit = C.c_int()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        if kind == 1 and self_steps > 0:
            c.call("sod_gpu_precond_restart_harvest")
        for k in range(compare_steps):
            if kind == 1 and self_steps > 0 and k == self_steps:
                ft_pairs = gpu.lib().sod_gpu_precond_harvest_count(c.h)
                t0 = time.perf_counter()
                c.call("sod_gpu_precond_train", ft_steps, ft_batch, ft_lr, 11, C.byref(ft_loss))
                ft_s = time.perf_counter() - t0
            o = gpu.SolveOpts(50000, 1e-8, kind, 200, 1 if (kind == 1 and k < self_steps) else 0)
            ev[0].record()
            c.call("sod_gpu_incomp_step", dt, C.byref(o), C.byref(st))
            ev[1].record()
            ev[1].synchronize()
            step_ms.append(ev[0].elapsed_time(ev[1]))
            it.append(st.iterations)
            ms.append(st.seconds * 1e3)
            rmax = max(rmax, st.res_rel)
            fb += st.fallback
            # velocity divergence after the step: L2 norm of the assembled int N div u
            c.call("sod_gpu_incomp_get", gpu.dptr(uu), None)
            c.call("sod_gpu_eval_divergence", gpu.dptr(uu), gpu.dptr(div))
            dv.append(float(div[w].double().norm()))
            c.call("sod_gpu_incomp_veloc_stats", C.byref(vit), None)
            vits.append(vit.value)
            if k % 50 == 0:
                free, total = torch.cuda.mem_get_info()
                peak_used[0] = max(peak_used[0], int(total - free))
        res[name] = {"mean_iterations": round(float(np.mean(it)), 1), "mean_solve_ms": round(float(np.mean(ms)), 3),
                     "mean_velocity_cg_iterations": round(float(np.mean(vits)), 2),
                     "mean_step_ms": round(float(np.mean(step_ms)), 3),
                     "max_true_residual": rmax, "fallbacks": fb, "mean_div_u_l2": float(np.mean(dv)),
                     "mean_solve_ms_first_100": round(float(np.mean(ms[:100])), 3),
                     "total_solve_s": round(float(np.sum(ms)) / 1e3, 3),
                     "iterations_every_50_steps": it[::50],
                     # the rest of the step (convection, diffusion, velocity solve, BDF/EXT, div/grad)
                     "step_without_pressure_Mnodes_per_s": round(m.npoin_w / max(1e-9, float(np.mean(step_ms)) -
                                                                                 float(np.mean(ms))) / 1e3, 1)}
    dev_bytes = [c.device_bytes for c in ctxs]
    for c in ctxs:
        c.close()
    return {"workload": f"incompressible TGV, periodic cube {nelem1d}^3 HEX64 ({N} nodes), Re=1600, dt={dt:.6g}, "
                        f"BDF3/EXT3-step pressure systems, FP64-certified tol 1e-8",
            "harvest_steps": harvest_steps, "compare_steps": compare_steps, "harvest_capacity": capacity,
            "train_steps": train_steps, "train_batch": 16, "train_lr": lr, "train_seconds": round(train_s, 2),
            "final_training_loss": round(float(loss.value), 4),
            "self_harvest_steps": self_steps, "self_harvest_pairs": ft_pairs, "finetune_steps": ft_steps,
            "finetune_batch": ft_batch, "finetune_lr": ft_lr, "finetune_seconds": round(ft_s, 2),
            "finetune_loss": round(float(ft_loss.value), 4), "jacobi": res["jacobi"],
            "jacobi_extrapolated_guess": res.get("jacobi_extrapolated_guess"), "learned": res["learned"],
            "speedup_wall": round(res["jacobi"]["mean_solve_ms"] / res["learned"]["mean_solve_ms"], 3),
            "speedup_wall_vs_jacobi_same_guess": (round(res["jacobi_extrapolated_guess"]["mean_solve_ms"] /
                                                        res["learned"]["mean_solve_ms"], 3) if extrap_arm else None),
            "harvest_overhead_s": round((harvest_ms[0] - harvest_ms[1]) / 1e3, 3),
            "speedup_wall_amortized": round(res["jacobi"]["total_solve_s"] /
                                            (res["learned"]["total_solve_s"] + train_s + ft_s +
                                             max(0.0, (harvest_ms[0] - harvest_ms[1]) / 1e3)), 3),
            "amortized_over": f"the {compare_steps} compared steps: Jacobi solve time against learned solve time "
                              f"+ training + fine-tuning + the extra solve time of the {harvest_steps} harvesting "
                              f"Jacobi steps",
            "speedup_wall_first_100_steps": round(res["jacobi"]["mean_solve_ms_first_100"] /
                                                  res["learned"]["mean_solve_ms_first_100"], 3),
            "device_bytes_jacobi_ctx": dev_bytes[1], "device_bytes_learned_ctx": dev_bytes[0],
            "harvest_seconds": round(harvest_ms[0] / 1e3, 3),
            "torch_peak_bytes": int(torch.cuda.max_memory_allocated()),
            "device_used_bytes_peak": peak_used[0]}


def time_step_leg(nelem1d=NELEM_1D, stages=4, steps=10, warmup=3):
    """Full compressible time steps (sod_gpu_comp_rk_ls_step: `stages` RHS
    evaluations, the FP64 low-storage stage updates and, once per step, the
    entropy-viscosity chain) on the Taylor-Green initial state of a periodic
    cube nelem1d^3 HEX64, Ma=0.1, at the CFL 0.5 dt of the first step."""
    import torch
    from sod2d_b200 import gpu, host
    m = host.periodic_cube(PORDER, nelem1d)
    ic = host.tgv_comp_init(m, Ma=0.1)
    sv = gpu.CompSolver(m, ic, stages=stages, fp64_state=True)
    for _ in range(warmup):
        sv.step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        sv.step()
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    sv.close()
    return {"workload": f"compressible TGV time step, periodic cube {nelem1d}^3 HEX64 (p=3), Ma=0.1, "
                        f"{stages}-stage SSP RK, FP64 state, entropy viscosity + LPS",
            "ms_per_step": round(ms, 4), "stages": stages,
            "Mnode_stages_per_s": round(m.npoin_w * stages / (ms / 1e3) / 1e6, 2), "steps_timed": steps}


def imex_step_leg(nelem1d=NELEM_1D, stages=4, steps=10, warmup=3, Ma=1.25, cfl=0.95):
    """IMEX time steps (sod_gpu_comp_imex_step: explicit convection, implicit
    diffusion through conjGrad_imex per stage, LPS of the step's initial
    state, entropy viscosity) on the Taylor-Green state of a periodic cube
    nelem1d^3 HEX64 with the reference's IMEX test settings (Ma 1.25, CFL
    0.95 convective, 4 stages, maxIter 200, tol 1e-3), FP32 state."""
    import ctypes as C
    import torch
    from sod2d_b200 import gpu, host
    m = host.periodic_cube(PORDER, nelem1d)
    ic = host.tgv_comp_init(m, Ma=Ma)
    sv = gpu.CompSolver(m, ic, stages=stages, fp64_state=False, cfl_conv=cfl, cfl_diff=1000.5, imex=True)
    for _ in range(warmup):
        sv.step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    its, res, cg = C.c_int(), C.c_double(), []
    e0.record()
    for _ in range(steps):
        sv.step()
        sv.ctx.call("sod_gpu_comp_imex_stats", C.byref(its), C.byref(res))
        cg.append(its.value)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    sv.close()
    return {"workload": f"compressible TGV IMEX step, periodic cube {nelem1d}^3 HEX64 (p=3), Ma={Ma}, CFL {cfl}, "
                        f"{stages}-stage ARK, FP32 state, implicit diffusion CG tol 1e-3, entropy viscosity + LPS",
            "ms_per_step": round(ms, 4), "stages": stages, "dt": round(float(sv.dt), 6),
            "cg_iterations_per_step": round(float(np.mean(cg)), 2),
            "Mnode_stages_per_s": round(m.npoin_w * stages / (ms / 1e3) / 1e6, 2), "steps_timed": steps}


def precision_study(nelem1d=16, nsteps=200, porder=3, Ma=0.1, stages=4):
    """Compressible TGV (periodic cube nelem1d^3, order porder, Ma, SSP RK
    with `stages` stages, CFL 0.5, LPS and entropy viscosity on) run three
    ways from the same initial state: the FP64 oracle (reference arithmetic
    in double precision), the GPU with FP32 element kernels and FP64 RK
    state, and the GPU all-FP32.  Reports the relative L2 error of the final
    rho, rho*u and E and the largest relative error of the kinetic-energy and
    dissipation histories against the FP64 run."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    from sod2d_b200 import gpu, host
    m = host.periodic_cube(porder, nelem1d)
    ic = host.tgv_comp_init(m, Ma=Ma)
    t0 = time.perf_counter()
    ref_hist, ref_fin = O.tgv_comp_run(O.OracleMesh(m, np.float64), ic, O.comp_params(ic, stages=stages), nsteps)
    t_ref = time.perf_counter() - t0
    w = m.lpoin_w - 1
    N = m.npoin
    rl2 = lambda a, b: float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))
    out = {"workload": f"compressible TGV, periodic cube {nelem1d}^3 HEX{(porder + 1) ** 3}, Ma={Ma}, Re=1600, "
                       f"{stages}-stage SSP RK, CFL 0.5, {nsteps} steps, LPS + entropy viscosity",
           "reference": f"oracle in FP64 ({t_ref:.1f} s on the host)"}
    for name, fp64 in (("fp32_kernels_fp64_state", True), ("all_fp32", False)):
        sv = gpu.CompSolver(m, ic, stages=stages, fp64_state=fp64)
        hist = sv.run(nsteps)
        fin = sv.state()
        sv.close()
        q = fin["q"].reshape(3, N)[:, w]
        qr = ref_fin["q"].reshape(3, N)[:, w]
        rows = min(len(hist), len(ref_hist))
        # history errors relative to each column's peak (eps_D starts at zero)
        relh = np.abs(hist[:rows] - ref_hist[:rows]).max(0) / np.abs(ref_hist[:rows]).max(0)
        out[name] = {"rel_l2_rho": rl2(fin["rho"][w], ref_fin["rho"][w]), "rel_l2_rhou": rl2(q, qr),
                     "rel_l2_E": rl2(fin["E"][w], ref_fin["E"][w]),
                     "EK_err_over_peak": float(relh[1]), "eps_S_err_over_peak": float(relh[2]),
                     "eps_D_err_over_peak": float(relh[3]), "eps_T_err_over_peak": float(relh[4]),
                     "history_rows": rows,
                     "eps_D_peak_over_eps_T_peak": float(np.abs(ref_hist[:rows, 3]).max() /
                                                         np.abs(ref_hist[:rows, 4]).max())}
    return out


def workload_config(nelem1d=NELEM_1D):
    ne = nelem1d ** 3
    nw = (PORDER * nelem1d) ** 3
    state_mb = nw * 5 * 4 / 1e6                   # rho, q(3), E in FP32
    geo_mb = ne * (PORDER + 1) ** 3 * 10 * 4 / 1e6  # J^-1 (9) + gpvol per Gauss point
    slots_gb = 1.6 * ne / 64 ** 3                   # element slots of both passes, 1.6 GB at 64^3
    l2 = "inputs larger than L2" if state_mb + geo_mb > 126 else "inputs partly L2-resident"
    return {"workload": f"RHS micro-benchmark: periodic cube {nelem1d}^3 HEX64 (p=3), interior GLL nodes jittered "
                        f"+-5%, random FP32 state, fused convective+diffusive(LPS)+entropy-viscosity residual with "
                        f"assembly and lumped-mass inversion",
            "nelem": ne, "porder": PORDER, "working_nodes": nw,
            "l2": f"{l2} (state {state_mb:.0f} MB, geometry {geo_mb:.0f} MB, assembly slots {slots_gb:.2f} GB)",
            "parallelism": "replicas"}


def halo_leg(nelem1d=NELEM_1D, nparts=8, steps=5, warmup=3):
    """The fused RHS on a partitioned mesh: the nelem1d^3 workload split into
    nparts z-slabs, every part a context with its halo plan (the halo sums
    of the projections and of the residuals inside sod_gpu_updateF).  The
    parts run as host threads of one process on ONE device and exchange
    through LocalHaloGroup, so the wall time here serialises the parts and
    includes host barriers: it is not a multi-GPU number.  The leg is for
    the kernel launch list (the halo pack and sum kernels beside the element
    kernels at a realistic part size) and reports the exchange volume."""
    import torch
    from sod2d_b200 import gpu, partition
    from sod2d_b200.halo import LocalHaloGroup
    m, ic, rho, q, E, mu_e, u, csound = build_workload(nelem1d)
    N, n = m.npoin, m.nnode
    parts = partition.split(m, partition.partition_elements(m, (1, 1, nparts)))
    group = LocalHaloGroup([p.plan for p in parts], timeout=300.0)
    dv = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    loc = lambda a, k, nd: np.asarray(a).reshape(k, N)[:, nd].reshape(-1)
    jobs, ctxs = [], []
    for p in parts:
        ctx = gpu.Context(p.mesh, gpu.phys_from_ic(ic))
        ctx.set_halo(p.plan, group)
        ctxs.append(ctx)
        nd, el = p.nodes, p.elems
        d = [dv(loc(rho, 1, nd)), dv(loc(q, 3, nd)), dv(loc(E, 1, nd)), dv(mu_e.reshape(n, -1)[:, el].reshape(-1))]
        uu, cs = dv(loc(u, 3, nd)), dv(loc(csound, 1, nd))
        tau = torch.zeros(p.mesh.nelem, device="cuda")
        ctx.call("sod_gpu_comp_tau", gpu.dptr(cs), gpu.dptr(uu), gpu.dptr(tau))
        out = [torch.zeros(k * p.mesh.npoin, device="cuda") for k in (1, 3, 1)]

        def job(ctx=ctx, d=d, tau=tau, out=out, k=0):
            for _ in range(k):
                ctx.call("sod_gpu_updateF", *(gpu.dptr(x) for x in d), float(ic.mu_factor), gpu.dptr(tau),
                         *(gpu.dptr(x) for x in out), None, None, None, None)
        jobs.append(job)
    group.run([lambda j=j: j(k=warmup) for j in jobs])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    group.run([lambda j=j: j(k=steps) for j in jobs])
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) / steps * 1e3
    for c in ctxs:
        c.close()
    entries = [p.plan.numNodesToComm for p in parts]
    return {"workload": f"fused RHS, {nelem1d}^3 HEX64 (p=3) split into {nparts} z-slabs, parts as host threads "
                        f"on one device (LocalHaloGroup)",
            "shared_entries_per_part": [min(entries), max(entries)],
            "exchange_bytes_per_rhs_per_part": int(max(entries) * (12 + 5) * 4),
            "wall_ms_per_rhs_all_parts_serialised": round(wall, 3), "steps": steps,
            "note": "one device: the parts' kernels run one after another and the exchanges are host-side "
                    "copies behind barriers; the launch list, not this time, is what this leg is for"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nelem1d", type=int, default=NELEM_1D)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-pressure", action="store_true")
    ap.add_argument("--pressure-only", action="store_true",
                    help="run only the pressure-solve comparison (prints its JSON object)")
    ap.add_argument("--p-nelem1d", type=int, default=32)
    ap.add_argument("--p-harvest", type=int, default=200)
    ap.add_argument("--p-compare", type=int, default=800)
    ap.add_argument("--p-train", type=int, default=300)
    ap.add_argument("--p-capacity", type=int, default=256, help="harvested (r, e) pairs kept for training")
    ap.add_argument("--p-self", type=int, default=16,
                    help="learned steps that harvest from their own solves before fine-tuning (0: none)")
    ap.add_argument("--p-finetune", type=int, default=200, help="Adam steps of the fine-tuning")
    ap.add_argument("--p-no-extrap", action="store_true",
                    help="leave out the Jacobi arm from the extrapolated guess (large meshes)")
    ap.add_argument("--precision-study", action="store_true",
                    help="run only the FP32/FP64 precision study against the FP64 oracle (prints its JSON object)")
    ap.add_argument("--ps-nelem1d", type=int, default=16)
    ap.add_argument("--ps-steps", type=int, default=200)
    ap.add_argument("--halo-split", type=int, default=0,
                    help="run only the partitioned-RHS leg with this many z-slabs on one device (prints its JSON object)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    pkw = dict(nelem1d=args.p_nelem1d, harvest_steps=args.p_harvest, compare_steps=args.p_compare,
               train_steps=args.p_train, capacity=args.p_capacity, self_steps=args.p_self, ft_steps=args.p_finetune,
               extrap_arm=not args.p_no_extrap)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.precision_study:
        if rank == 0:
            import torch
            torch.cuda.set_device(local)
            print(json.dumps({"precision_study": precision_study(args.ps_nelem1d, args.ps_steps)}))
        return 0
    if args.halo_split > 0:
        if rank == 0:
            import torch
            torch.cuda.set_device(local)
            print(json.dumps({"halo_split": halo_leg(args.nelem1d, args.halo_split, steps=min(args.steps, 5),
                                                     warmup=args.warmup)}))
        return 0
    if args.pressure_only:
        if rank == 0:
            import torch
            torch.cuda.set_device(local)
            print(json.dumps({"pressure_solve": pressure_leg(**pkw)}))
        return 0

    import torch
    import torch.distributed as dist
    from sod2d_b200 import gpu

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))

    m, ic, rho, q, E, mu_e, u, csound = build_workload(args.nelem1d)
    ctx = gpu.Context(m, gpu.phys_from_ic(ic))
    stream = torch.cuda.Stream()
    ctx.call("sod_gpu_set_stream", gpu.VP(stream.cuda_stream))
    ctx.call("sod_gpu_set_async", 1)
    N = m.npoin
    dv = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    d = {k: dv(v) for k, v in dict(rho=rho, q=q, E=E, mu_e=mu_e, u=u, csound=csound).items()}
    tau = torch.zeros(m.nelem, device="cuda")
    out = [torch.zeros(n, device="cuda") for n in (N, 3 * N, N)]
    with torch.cuda.stream(stream):
        ctx.call("sod_gpu_comp_tau", gpu.dptr(d["csound"]), gpu.dptr(d["u"]), gpu.dptr(tau))
        ctx.call("sod_gpu_set_mu_e", gpu.dptr(d["mu_e"]))
    stream.synchronize()

    def step():
        ctx.call("sod_gpu_updateF", gpu.dptr(d["rho"]), gpu.dptr(d["q"]), gpu.dptr(d["E"]), None,
                 float(ic.mu_factor), gpu.dptr(tau), *(gpu.dptr(x) for x in out), None, None, None, None)

    launches_per_step = 4  # k_proj, gather(A), k_rhs, gather(B)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    stream.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            ev0.record(stream)
            for _ in range(args.steps):
                step()
            ev1.record(stream)
        ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = max_over_ranks(ms, world, "cuda")
    ms_step = ms / args.steps
    value = job_throughput(world, m.npoin_w, args.steps, ms)  # Mnode-stages/s, all ranks

    # end-to-end through the C-ABI with pinned host buffers: every step
    # uploads its state (H2D), evaluates one RHS and downloads the residuals
    # (D2H).  Steps are independent, so they are pipelined on three streams
    # with double buffers: the upload of step k+1 and the download of step
    # k-1 overlap the RHS of step k (PCIe is full duplex).  All copies of
    # every step are inside the timed region.
    h_in = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in (rho, q, E)]
    h_out = [[torch.empty(n, dtype=torch.float32).pin_memory() for n in (N, 3 * N)] + [torch.empty(N).pin_memory()]
             for _ in range(2)]
    d_in = [[torch.empty_like(x, device="cuda") for x in (d["rho"], d["q"], d["E"])] for _ in range(2)]
    d_out = [[torch.empty_like(x) for x in out] for _ in range(2)]
    s_up, s_dn = torch.cuda.Stream(), torch.cuda.Stream()
    e2e_steps = max(4, min(args.steps, 20))
    up_done = [torch.cuda.Event() for _ in range(2)]
    rhs_done = [torch.cuda.Event() for _ in range(2)]
    dn_done = [torch.cuda.Event() for _ in range(2)]

    def e2e_run(nsteps):
        for k in range(nsteps):
            b = k % 2
            with torch.cuda.stream(s_up):
                if k >= 2:
                    s_up.wait_event(rhs_done[b])  # the RHS of step k-2 has read this input buffer
                for hd, dd in zip(h_in, d_in[b]):
                    dd.copy_(hd, non_blocking=True)
                up_done[b].record(s_up)
            with torch.cuda.stream(stream):
                stream.wait_event(up_done[b])
                if k >= 2:
                    stream.wait_event(dn_done[b])  # step k-2's residuals are downloaded
                ctx.call("sod_gpu_updateF", gpu.dptr(d_in[b][0]), gpu.dptr(d_in[b][1]), gpu.dptr(d_in[b][2]), None,
                         float(ic.mu_factor), gpu.dptr(tau), *(gpu.dptr(x) for x in d_out[b]), None, None, None,
                         None)
                rhs_done[b].record(stream)
            with torch.cuda.stream(s_dn):
                s_dn.wait_event(rhs_done[b])
                for ho, dd in zip(h_out[b], d_out[b]):
                    ho.copy_(dd, non_blocking=True)
                dn_done[b].record(s_dn)

    e2e_run(2)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s_up)
    stream.wait_event(e0)
    s_dn.wait_event(e0)
    e2e_run(e2e_steps)
    s_dn.wait_event(rhs_done[(e2e_steps - 1) % 2])
    s_dn.wait_stream(s_up)
    s_dn.wait_stream(stream)
    e1.record(s_dn)
    e1.synchronize()
    e2e_val = job_throughput(world, m.npoin_w, e2e_steps, max_over_ranks(e0.elapsed_time(e1), world, "cuda"))
    h2d = sum(t.numel() * 4 for t in h_in)
    d2h = sum(t.numel() * 4 for t in h_out[0])

    # the copies alone, same buffers and streams, both directions at once:
    # the bound the end-to-end number can reach over the host link
    def copies_only(nsteps):
        for k in range(nsteps):
            b = k % 2
            with torch.cuda.stream(s_up):
                for hd, dd in zip(h_in, d_in[b]):
                    dd.copy_(hd, non_blocking=True)
            with torch.cuda.stream(s_dn):
                for ho, dd in zip(h_out[b], d_out[b]):
                    ho.copy_(dd, non_blocking=True)

    copies_only(2)
    torch.cuda.synchronize()
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0.record(s_up)
    s_dn.wait_event(c0)
    copies_only(e2e_steps)
    s_dn.wait_stream(s_up)
    c1.record(s_dn)
    c1.synchronize()
    copy_ms = max_over_ranks(c0.elapsed_time(c1), world, "cuda")
    copy_bound = job_throughput(world, m.npoin_w, e2e_steps, copy_ms)
    # the pipelined result must equal the device-resident one
    torch.cuda.synchronize()
    e2e_check = max(float((h_out[(e2e_steps - 1) % 2][i].cuda() - out[i]).abs().max()) for i in range(3))

    peak, peak_kind = measured_peaks()
    achieved = B_PER_NODE_STAGE * m.npoin_w / (ms_step / 1e3) / 1e9
    line = {
        "metric": "Mnode-stages/s (fused compressible RHS, FP32)", "value": round(value, 2),
        "unit": "Mnode-stages/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "config": workload_config(args.nelem1d),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4),
                     "traffic": int(round(DRAM_B_PER_NODE_STAGE * m.npoin_w)),
                     "traffic_source": "ncu dram__bytes_read+write of the 4 RHS kernels at 64^3 (per working node, times "
                                       "this mesh's working nodes)",
                     "peak_source": f"{peak_kind} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)",
                     "unit_of_work": "one fused RHS evaluation (4 launches): 402 B x working nodes"},
        "e2e": {"value": round(e2e_val, 2), "unit": "Mnode-stages/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "steps": e2e_steps,
                "pipelining": "H2D(k+1) and D2H(k-1) overlap RHS(k) on 3 streams, double buffers",
                "max_abs_diff_vs_device_resident": e2e_check,
                "copy_bound": {"value": round(copy_bound, 2), "frac": round(e2e_val / copy_bound, 4),
                               "link_gbs_per_direction": round(max(h2d, d2h) * e2e_steps / (copy_ms / 1e3) / 1e9, 1),
                               "what": "the same H2D and D2H copies alone, both directions at once"}},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk.summary(),
        "device_bytes": ctx.device_bytes,
    }
    ctx.close()
    if rank == 0 and world == 1 and not args.no_pressure:
        line["time_step"] = time_step_leg(args.nelem1d)
        line["imex_step"] = imex_step_leg(args.nelem1d)
        line["pressure_solve"] = pressure_leg(**pkw)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = CpuBaseline(args.nelem1d).sample()
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
