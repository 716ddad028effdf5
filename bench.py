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
# ncu capture of the four RHS kernels on the 32^3 workload (548,663,296 B for
# 884,736 working nodes; profiles/rhs_kernels_64cube_p3.md), scaled by the
# working nodes of the benchmarked mesh.
DRAM_B_PER_NODE_STAGE = 548663296 / 884736
NELEM_1D = 64
PORDER = 3


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                parts = [x.strip() for x in out.stdout.strip().split(",")]
                if len(parts) >= 7:
                    self.samples.append(parts)
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


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
    """The oracle's FP32 RHS (OpenMP over all host cores) on a bounded sample
    of the workload: a 32^3-element jittered cube of the same order (884,736
    working nodes)."""

    NELEM_1D = 32

    def __init__(self):
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O
        self.O = O
        m, ic, rho, q, E, mu_e, u, csound = build_workload(self.NELEM_1D)
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
    cb = CpuBaseline()
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
            "data": "synthetic", "config": workload_config(),
            "cpu_baseline": info, "e2e": {"value": round(v, 3), "unit": "Mnode-stages/s", "h2d_bytes_per_step": 0,
                                          "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def pressure_leg(nelem1d=32, harvest_steps=40, compare_steps=20, dt=0.01, train_steps=300, lr=1e-3):
    """Pressure-Poisson solve to a 1e-8 FP64-certified relative residual on
    the incompressible Taylor-Green vortex (periodic cube nelem1d^3 HEX64,
    Re=1600): Jacobi-preconditioned flexible CG against the learned
    element-patch preconditioner, each on its own trajectory of the
    projection-step driver from the same initial velocity.  The first
    `harvest_steps` steps run Jacobi and harvest (residual, error) pairs;
    the network is then trained on the GPU; the next `compare_steps` solves
    are timed on both trajectories (device time of each solve)."""
    import ctypes as C
    import torch
    from sod2d_b200 import gpu, host
    m = host.periodic_cube(PORDER, nelem1d)
    N = m.npoin
    x, y, z = (m.coord[i * N:(i + 1) * N].astype(np.float64) for i in range(3))
    u0 = torch.from_numpy(np.concatenate([np.sin(x) * np.cos(y) * np.cos(z), -np.cos(x) * np.sin(y) * np.cos(z),
                                          np.zeros(N)]).astype(np.float32)).cuda()
    nu = 1.0 / 1600.0
    ctxs = [gpu.Context(m, gpu.default_phys()) for _ in range(2)]
    for c in ctxs:
        c.call("sod_gpu_incomp_init", gpu.dptr(u0), nu)
    ctxs[0].call("sod_gpu_precond_init", 2024, 256)
    st = gpu.SolveStats()
    for k in range(harvest_steps):
        for i, c in enumerate(ctxs):
            o = gpu.SolveOpts(50000, 1e-8, 0, 100, 1 if i == 0 else 0)
            c.call("sod_gpu_incomp_step", dt, C.byref(o), C.byref(st))
    loss = C.c_float()
    t0 = time.perf_counter()
    ctxs[0].call("sod_gpu_precond_train", train_steps, 16, lr, 7, C.byref(loss))
    train_s = time.perf_counter() - t0
    res = {}
    for i, (name, kind) in enumerate((("jacobi", 0), ("learned", 1))):
        c = ctxs[0] if kind == 1 else ctxs[1]
        it, ms, rmax, fb = [], [], 0.0, 0
        for k in range(compare_steps):
            o = gpu.SolveOpts(50000, 1e-8, kind, 200, 0)
            c.call("sod_gpu_incomp_step", dt, C.byref(o), C.byref(st))
            it.append(st.iterations)
            ms.append(st.seconds * 1e3)
            rmax = max(rmax, st.res_rel)
            fb += st.fallback
        res[name] = {"mean_iterations": round(float(np.mean(it)), 1), "mean_solve_ms": round(float(np.mean(ms)), 3),
                     "max_true_residual": rmax, "fallbacks": fb}
    for c in ctxs:
        c.close()
    return {"workload": f"incompressible TGV, periodic cube {nelem1d}^3 HEX64 ({N} nodes), Re=1600, dt={dt}, "
                        f"projection-step pressure systems, FP64-certified tol 1e-8",
            "harvest_steps": harvest_steps, "train_steps": train_steps, "train_batch": 16, "train_lr": lr, "train_seconds": round(train_s, 2),
            "final_training_loss": round(float(loss.value), 4), "jacobi": res["jacobi"], "learned": res["learned"],
            "speedup_wall": round(res["jacobi"]["mean_solve_ms"] / res["learned"]["mean_solve_ms"], 3)}


def workload_config():
    return {"workload": f"RHS micro-benchmark: periodic cube {NELEM_1D}^3 HEX64 (p=3), interior GLL nodes jittered "
                        f"+-5%, random FP32 state, fused convective+diffusive(LPS)+entropy-viscosity residual with "
                        f"assembly and lumped-mass inversion",
            "nelem": NELEM_1D ** 3, "porder": PORDER, "working_nodes": (PORDER * NELEM_1D) ** 3,
            "l2": "inputs larger than L2 (state 142 MB, geometry 671 MB, assembly slots 1.6 GB)",
            "parallelism": "replicas"}


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
    ap.add_argument("--p-harvest", type=int, default=40)
    ap.add_argument("--p-compare", type=int, default=20)
    ap.add_argument("--p-train", type=int, default=300)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    pkw = dict(nelem1d=args.p_nelem1d, harvest_steps=args.p_harvest, compare_steps=args.p_compare,
               train_steps=args.p_train)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
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
    t_ms = torch.tensor([ms], device="cuda", dtype=torch.float64)
    if world > 1:
        dist.barrier()
        dist.all_reduce(t_ms, op=dist.ReduceOp.MAX)
    ms = float(t_ms.item())
    ms_step = ms / args.steps
    value = world * m.npoin_w * args.steps / (ms / 1e3) / 1e6  # Mnode-stages/s, all ranks

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
    e2e_ms = torch.tensor([e0.elapsed_time(e1)], device="cuda", dtype=torch.float64)
    if world > 1:
        dist.all_reduce(e2e_ms, op=dist.ReduceOp.MAX)
    e2e_val = world * m.npoin_w * e2e_steps / (float(e2e_ms.item()) / 1e3) / 1e6
    h2d = sum(t.numel() * 4 for t in h_in)
    d2h = sum(t.numel() * 4 for t in h_out[0])
    # the pipelined result must equal the device-resident one
    torch.cuda.synchronize()
    e2e_check = max(float((h_out[(e2e_steps - 1) % 2][i].cuda() - out[i]).abs().max()) for i in range(3))

    peak, peak_kind = measured_peaks()
    achieved = B_PER_NODE_STAGE * m.npoin_w / (ms_step / 1e3) / 1e9
    line = {
        "metric": "Mnode-stages/s (fused compressible RHS, FP32)", "value": round(value, 2),
        "unit": "Mnode-stages/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "config": workload_config(),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4),
                     "traffic": int(round(DRAM_B_PER_NODE_STAGE * m.npoin_w)),
                     "traffic_source": "ncu dram__bytes_read+write of the 4 RHS kernels at 32^3, scaled by working nodes",
                     "peak_source": f"{peak_kind} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)",
                     "unit_of_work": "one fused RHS evaluation (4 launches): 402 B x working nodes"},
        "e2e": {"value": round(e2e_val, 2), "unit": "Mnode-stages/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "steps": e2e_steps,
                "pipelining": "H2D(k+1) and D2H(k-1) overlap RHS(k) on 3 streams, double buffers",
                "max_abs_diff_vs_device_resident": e2e_check},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk.summary(),
        "device_bytes": ctx.device_bytes,
    }
    ctx.close()
    if rank == 0 and world == 1 and not args.no_pressure:
        line["pressure_solve"] = pressure_leg(**pkw)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = CpuBaseline().sample()
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
