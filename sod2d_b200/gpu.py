"""Python view of the C-ABI in ``include/sod2d_gpu.h`` (``libsod2d_gpu.so``).

Device buffers come from torch (plumbing only); every call goes through the
C entry points with raw device pointers, exactly as a Fortran caller would
bind them.  Importing this module on a machine without CUDA works; creating
a ``Context`` needs a GPU and fails loudly if the library is missing.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import build as _build

_lib = None

P_I = C.POINTER(C.c_int)
P_F = C.POINTER(C.c_float)
VP = C.c_void_p
# sod_halo_exchange_fn(user, send_buf, recv_buf, width, stream)
HALO_FN = C.CFUNCTYPE(C.c_int, VP, VP, VP, C.c_int, VP)
# sod_allreduce_fn(user, buf, count, kind, stream)
REDUCE_FN = C.CFUNCTYPE(C.c_int, VP, VP, C.c_int, C.c_int, VP)
REDUCE_MIN_F32, REDUCE_MAX_F32, REDUCE_SUM_F64 = 0, 1, 2


class SodMesh(C.Structure):
    _fields_ = [("porder", C.c_int), ("nelem", C.c_int), ("npoin", C.c_int), ("npoin_w", C.c_int),
                ("connec", VP), ("lpoin_w", VP), ("invAtoIJK", VP), ("gmshAtoI", VP), ("gmshAtoJ", VP),
                ("gmshAtoK", VP), ("dlxigp_ip", VP), ("He", VP), ("gpvol", VP), ("Ml", VP), ("invMl", VP),
                ("helem", VP), ("helem_l", VP), ("lelpn", VP), ("Ngp", VP)]


class SolveOpts(C.Structure):
    _fields_ = [("max_iter", C.c_int), ("tol", C.c_double), ("precond", C.c_int), ("stagnation_window", C.c_int),
                ("harvest", C.c_int)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("fallback", C.c_int), ("res_rel", C.c_double), ("seconds", C.c_double)]


class RkCfg(C.Structure):
    _fields_ = [("stages", C.c_int), ("rk_n", C.c_int), ("fp64_state", C.c_int), ("mu_factor", C.c_float)]


class SodPhys(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("gamma_gas", "Rgas", "Cp", "Prt", "c_lps", "c_rho", "c_ener", "ce",
                                         "cmax", "cglob", "ducros_min_val", "c_species_stab", "p_inf",
                                         "rho_inf")]


# name -> (restype, argtypes); every entry point declared in sod2d_gpu.h
SIGNATURES = {
    "sod_gpu_init": (C.c_int, [C.POINTER(SodMesh), C.POINTER(SodPhys), C.POINTER(VP)]),
    "sod_gpu_finalize": (C.c_int, [VP]),
    "sod_gpu_set_stream": (C.c_int, [VP, VP]),
    "sod_gpu_set_async": (C.c_int, [VP, C.c_int]),
    "sod_gpu_synchronize": (C.c_int, [VP]),
    "sod_gpu_last_error": (C.c_char_p, []),
    "sod_gpu_device_bytes": (C.c_size_t, [VP]),
    "sod_gpu_full_convec_ijk": (C.c_int, [VP] + [VP] * 8 + [C.c_int, C.c_float]),
    "sod_gpu_full_proj_ijk": (C.c_int, [VP] + [VP] * 8),
    "sod_gpu_full_diff_stab_ijk": (C.c_int, [VP, C.c_float, C.c_float] + [VP] * 16 + [C.c_int, C.c_float]),
    "sod_gpu_full_diffusion_ijk": (C.c_int, [VP, C.c_float, C.c_float] + [VP] * 10 + [C.c_int, C.c_float]),
    "sod_gpu_lumped_solver": (C.c_int, [VP, VP, C.c_int]),
    "sod_gpu_updateF": (C.c_int, [VP, VP, VP, VP, VP, C.c_float] + [VP] * 8),
    "sod_gpu_comp_tau": (C.c_int, [VP, VP, VP, VP]),
    "sod_gpu_generic_scalar_convec_ijk": (C.c_int, [VP] * 5 + [C.c_int, C.c_float]),
    "sod_gpu_smart_visc_spectral_imex": (C.c_int, [VP] * 6),
    "sod_gpu_ducros_visc_limit": (C.c_int, [VP] * 7),
    "sod_gpu_rk_ls_stage": (C.c_int, [VP, C.c_int] + [C.c_float] * 4 + [VP] * 9),
    "sod_gpu_set_mu_e": (C.c_int, [VP, VP]),
    "sod_gpu_comp_init_state": (C.c_int, [VP, C.POINTER(RkCfg)] + [VP] * 9),
    "sod_gpu_comp_rk_ls_step": (C.c_int, [VP, C.c_float]),
    "sod_gpu_comp_imex_step": (C.c_int, [VP, C.c_float, C.c_int, C.c_double]),
    "sod_gpu_comp_imex_stats": (C.c_int, [VP, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "sod_gpu_comp_adapt_dt": (C.c_int, [VP, C.c_float, C.c_float, C.POINTER(C.c_float)]),
    "sod_gpu_comp_analysis": (C.c_int, [VP, C.c_float, C.POINTER(C.c_double)]),
    "sod_gpu_comp_get_state": (C.c_int, [VP] + [VP] * 4),
    "sod_gpu_eval_laplacian_mult": (C.c_int, [VP, VP, VP]),
    "sod_gpu_eval_laplacian_mult64": (C.c_int, [VP, VP, VP]),
    "sod_gpu_eval_laplacian_diag": (C.c_int, [VP, VP]),
    "sod_gpu_eval_gradient": (C.c_int, [VP, VP, VP]),
    "sod_gpu_eval_divergence": (C.c_int, [VP, VP, VP]),
    "sod_gpu_full_convec_ijk_incomp": (C.c_int, [VP, VP, VP, VP]),
    "sod_gpu_conjgrad_pressure": (C.c_int, [VP, VP, VP, C.c_int, C.c_double, C.POINTER(C.c_int),
                                            C.POINTER(C.c_double)]),
    "sod_gpu_pressure_solve": (C.c_int, [VP, VP, VP, VP, VP]),
    "sod_gpu_precond_num_params": (C.c_int, [VP]),
    "sod_gpu_precond_init": (C.c_int, [VP, C.c_uint64, C.c_int]),
    "sod_gpu_precond_set_params": (C.c_int, [VP, VP, C.c_int]),
    "sod_gpu_precond_get_params": (C.c_int, [VP, VP, C.c_int]),
    "sod_gpu_precond_apply": (C.c_int, [VP, VP, VP]),
    "sod_gpu_precond_loss_grad": (C.c_int, [VP, VP, VP, C.POINTER(C.c_double), VP]),
    "sod_gpu_precond_harvest_count": (C.c_int, [VP]),
    "sod_gpu_precond_restart_harvest": (C.c_int, [VP]),
    "sod_gpu_precond_train": (C.c_int, [VP, C.c_int, C.c_int, C.c_float, C.c_uint64, C.POINTER(C.c_float)]),
    "sod_gpu_incomp_init": (C.c_int, [VP, VP, C.c_double]),
    "sod_gpu_incomp_step": (C.c_int, [VP, C.c_float, VP, VP]),
    "sod_gpu_incomp_get": (C.c_int, [VP, VP, VP]),
    "sod_gpu_incomp_set_veloc_solver": (C.c_int, [VP, C.c_int, C.c_double]),
    "sod_gpu_incomp_set_pressure": (C.c_int, [VP, VP]),
    "sod_gpu_incomp_adapt_dt": (C.c_int, [VP, C.c_float, C.POINTER(C.c_float)]),
    "sod_gpu_incomp_analysis": (C.c_int, [VP, C.POINTER(C.c_double)]),
    "sod_gpu_incomp_veloc_stats": (C.c_int, [VP, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "sod_gpu_species_tau": (C.c_int, [VP, VP, VP]),
    "sod_gpu_eval_tau_veloc": (C.c_int, [VP] * 5),
    "sod_gpu_full_diff_stab_incomp": (C.c_int, [VP] * 9),
    "sod_gpu_conjgrad_veloc": (C.c_int, [VP, C.c_float, C.c_float, VP, VP, VP, VP, C.c_int, C.c_double,
                                         C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "sod_gpu_analysis_noalloc": (C.c_int, [C.c_int] * 4 + [VP] * 15 + [C.c_float, C.c_float, VP,
                                                                       C.POINTER(C.c_double)]),
    "sod_gpu_set_halo": (C.c_int, [VP, C.c_int, C.c_int, P_I, P_I, P_I, P_I, VP, VP, HALO_FN, VP]),
    "sod_gpu_halo_update": (C.c_int, [VP, VP, C.c_int]),
    "sod_gpu_set_allreduce": (C.c_int, [VP, REDUCE_FN, VP]),
}


def lib_path():
    return _build.LIBDIR / "libsod2d_gpu.so"


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = lib_path()
        if not path.exists():
            raise RuntimeError(f"{path} is missing: run `python -m sod2d_b200.build` (no CPU fallback exists)")
        _lib = C.CDLL(str(path))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(_lib, name)
            f.restype = res
            f.argtypes = args
    return _lib


def check(rc, what=""):
    if rc != 0:
        raise RuntimeError(f"{what} failed ({rc}): {lib().sod_gpu_last_error().decode()}")


def last_error() -> str:
    """sod_gpu_last_error() of the calling thread."""
    return lib().sod_gpu_last_error().decode()


def _hp(a):
    return None if a is None else a.ctypes.data_as(VP)


class _CudaBuffer:
    def __init__(self, ptr, count, typestr):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


def device_view(ptr, count, typestr="<f4"):
    """Zero-copy torch view of `count` elements of device memory at ptr."""
    import torch
    return torch.as_tensor(_CudaBuffer(int(ptr), count, typestr), device="cuda")


def dptr(t):
    """Device pointer of a torch CUDA tensor (None -> NULL)."""
    return None if t is None else VP(t.data_ptr())


def default_phys(gamma=1.4, Rgas=None, Cp=None, Prt=0.71, p_inf=None, rho_inf=1.0, Ma=0.1) -> SodPhys:
    if Rgas is None:
        Rgas = 1.0 / (gamma * Ma * Ma)
    if Cp is None:
        Cp = gamma * Rgas / (gamma - 1.0)
    if p_inf is None:
        p_inf = 1.0 / (gamma * Ma * Ma)
    return SodPhys(gamma, Rgas, Cp, Prt, np.float32(0.1), 1.0, 1.0, 1.0, 0.5, 1.0, 0.1, 0.5, p_inf, rho_inf)


def phys_from_ic(ic) -> SodPhys:
    return SodPhys(ic.gamma, ic.Rgas, ic.Cp, ic.Prt, np.float32(0.1), 1.0, 1.0, 1.0, 0.5, 1.0, 0.1, 0.5, ic.P0,
                   ic.rho0)


class Context:
    """Owns a sod_gpu_ctx built from a host.Mesh."""

    def __init__(self, mesh, phys: SodPhys):
        self.mesh = mesh
        self._keep = {k: np.ascontiguousarray(getattr(mesh, k)) for k in (
            "connecWork", "lpoin_w", "invAtoIJK", "gmshAtoI", "gmshAtoJ", "gmshAtoK", "dlxigp_ip", "He", "gpvol",
            "Ml", "invMl", "helem", "helem_l", "lelpn", "Ngp")}
        k = self._keep
        self.sm = SodMesh(mesh.porder, mesh.nelem, mesh.npoin, mesh.npoin_w, _hp(k["connecWork"]), _hp(k["lpoin_w"]),
                          _hp(k["invAtoIJK"]), _hp(k["gmshAtoI"]), _hp(k["gmshAtoJ"]), _hp(k["gmshAtoK"]),
                          _hp(k["dlxigp_ip"]), _hp(k["He"]), _hp(k["gpvol"]), _hp(k["Ml"]), _hp(k["invMl"]),
                          _hp(k["helem"]), _hp(k["helem_l"]), _hp(k["lelpn"]), _hp(k["Ngp"]))
        self.phys = phys
        h = VP()
        check(lib().sod_gpu_init(C.byref(self.sm), C.byref(self.phys), C.byref(h)), "sod_gpu_init")
        self.h = h

    def close(self):
        if self.h:
            lib().sod_gpu_finalize(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def call(self, name, *args):
        rc = getattr(lib(), name)(self.h, *args)
        err = getattr(self, "_halo", {}).pop("err", None)
        if rc != 0 and err is not None:
            raise RuntimeError(f"{name}: halo exchange failed") from err
        check(rc, name)

    def set_halo(self, plan, transport):
        """Attach a halo plan (sod2d_b200.partition.HaloPlan) and a transport
        with exchange(plan, send, recv, width); the send / receive buffers are
        device tensors of 12 floats per entry of nodesToComm."""
        import torch
        n = 12 * max(plan.numNodesToComm, 1)
        h = dict(send=torch.zeros(n, device="cuda"), recv=torch.zeros(n, device="cuda"), plan=plan)
        ints = [np.ascontiguousarray(a, np.int32) for a in (plan.ranksToComm, plan.commsMemPosInLoc,
                                                            plan.commsMemSize, plan.nodesToComm)]
        if ints[3].size == 0:
            ints[3] = np.zeros(1, np.int32)

        def cb(user, send_buf, recv_buf, width, stream):
            try:
                transport.exchange(plan, h["send"], h["recv"], int(width))
                return 0
            except BaseException as e:  # noqa: BLE001 - re-raised by call()
                h["err"] = e
                return -1

        h["fn"], h["ints"] = HALO_FN(cb), ints
        if hasattr(transport, "register"):
            transport.register(plan.rank, h["send"])
        self._halo = h
        self.call("sod_gpu_set_halo", plan.rank, plan.numRanksWithComms, *(a.ctypes.data_as(P_I) for a in ints),
                  dptr(h["send"]), dptr(h["recv"]), h["fn"], None)
        return h

    def set_allreduce(self, transport, rank: int):
        """Global reductions through transport.allreduce(rank, tensor, kind)
        (a collective call: every rank sets it)."""
        import torch
        dtypes = {REDUCE_MIN_F32: (torch.float32, "<f4"), REDUCE_MAX_F32: (torch.float32, "<f4"),
                  REDUCE_SUM_F64: (torch.float64, "<f8")}
        h = self.__dict__.setdefault("_halo", {})

        def cb(user, buf, count, kind, stream):
            try:
                transport.allreduce(rank, device_view(buf, int(count), dtypes[int(kind)][1]), int(kind))
                return 0
            except BaseException as e:  # noqa: BLE001 - re-raised by call()
                h["err"] = e
                return -1

        h["reduce_fn"] = REDUCE_FN(cb)
        self.call("sod_gpu_set_allreduce", h["reduce_fn"], None)

    @property
    def device_bytes(self) -> int:
        return int(lib().sod_gpu_device_bytes(self.h))


class CompSolver:
    """Compressible periodic time loop on the GPU through the C-ABI: the
    driver logic of CFDSolverBase_evalTimeIteration
    (src/lib_mainBaseClass/sources/CFDSolverBase.f90:1929-2164) around
    sod_gpu_comp_rk_ls_step, or sod_gpu_comp_imex_step when imex is set
    (time_integ_imex.f90; the implicit solve's maxIter / tol)."""

    def __init__(self, mesh, ic, stages=4, rk_n=1, fp64_state=True, cfl_conv=0.5, cfl_diff=0.5, imex=False,
                 imex_maxiter=200, imex_tol=1e-3, partition=None):
        """partition = (part, transport): run the rank `part`
        (sod2d_b200.partition.Part of `mesh`) with its halo sums and global
        reductions through transport (a collective constructor)."""
        import torch
        self.torch = torch
        npoin = mesh.npoin
        if partition is not None:
            part, transport = partition
            mesh = part.mesh
            loc = lambda a: np.asarray(a).reshape(-1, npoin)[:, part.nodes].reshape(-1)
        else:
            loc = lambda a: a
        self.ctx = Context(mesh, phys_from_ic(ic))
        if partition is not None:
            self.ctx.set_halo(part.plan, transport)
            self.ctx.set_allreduce(transport, part.rank)
        self.mesh, self.ic = mesh, ic
        self.cfl = (cfl_conv, cfl_diff)
        self.imex = (imex_maxiter, imex_tol) if imex else None
        dv = lambda a: torch.from_numpy(np.ascontiguousarray(loc(a))).cuda()
        self._init = [dv(a) for a in (ic.rho, ic.u, ic.q, ic.pr, ic.E, ic.Tem, ic.csound, ic.machno, ic.eta)]
        cfg = RkCfg(stages, rk_n, int(fp64_state), ic.mu_factor)
        self.ctx.call("sod_gpu_comp_init_state", C.byref(cfg), *(dptr(t) for t in self._init))
        self.time = np.float32(0.0)
        self.dt = self.adapt_dt()

    def adapt_dt(self) -> float:
        v = C.c_float()
        self.ctx.call("sod_gpu_comp_adapt_dt", self.cfl[0], self.cfl[1], C.byref(v))
        return float(v.value)

    def analysis(self):
        out = (C.c_double * 5)()
        self.ctx.call("sod_gpu_comp_analysis", float(self.ic.rho0), out)
        return [float(self.time)] + list(out)

    def step(self):
        if self.imex:
            self.ctx.call("sod_gpu_comp_imex_step", float(self.dt), self.imex[0], self.imex[1])
        else:
            self.ctx.call("sod_gpu_comp_rk_ls_step", float(self.dt))
        self.time = np.float32(self.time + np.float32(self.dt))

    def run(self, nsteps, log_first=1, log_step=10, max_time=None):
        hist = [self.analysis()]
        log_next = log_first
        for istep in range(1, nsteps + 1):
            self.step()
            if istep == log_next:
                hist.append(self.analysis())
                log_next += log_step
            self.dt = self.adapt_dt()
            if max_time is not None and self.time >= np.float32(max_time):
                break
        return np.array(hist)

    def state(self):
        torch = self.torch
        N, n, E = self.mesh.npoin, self.mesh.nnode, self.mesh.nelem
        t = [torch.zeros(k, device="cuda") for k in (N, 3 * N, N, E * n)]
        self.ctx.call("sod_gpu_comp_get_state", *(dptr(x) for x in t))
        return dict(zip(("rho", "q", "E", "mu_e"), (x.cpu().numpy() for x in t)))

    def close(self):
        self.ctx.close()


class IncompSolver:
    """Incompressible periodic time loop on the GPU through the C-ABI: the
    Taylor-Green initial state of TGVSolverIncomp (velocity and pressure),
    the convective CFL dt of CFDSolverPeriodicIncomp_evalDt and one
    sod_gpu_incomp_step (bdfext3_main_incomp) per step.  opts is a
    SolveOpts for the pressure solve (precond 2: the reference's FP32 CG);
    veloc = (maxIter, tol) of the velocity solve."""

    def __init__(self, mesh, Re=1600.0, cfl_conv=0.5, veloc=(20, 1e-2), partition=None):
        """partition = (part, transport): run the rank `part` of `mesh` with
        its halo sums and global reductions (a collective constructor; the
        steps must use the reference's FP32 pressure solve, precond 2)."""
        import torch
        self.torch = torch
        if partition is not None:
            part, transport = partition
            mesh = part.mesh
        self.mesh = mesh
        self.ctx = Context(mesh, default_phys())
        if partition is not None:
            self.ctx.set_halo(part.plan, transport)
            self.ctx.set_allreduce(transport, part.rank)
        N = mesh.npoin
        x, y, z = (mesh.coord[i * N:(i + 1) * N].astype(np.float32) for i in range(3))
        u0 = np.concatenate([np.sin(x) * np.cos(y) * np.cos(z), -np.cos(x) * np.sin(y) * np.cos(z),
                             np.zeros(N, np.float32)]).astype(np.float32)
        p0 = (np.float32(1.0 / 16.0) * (np.cos(np.float32(2) * x) + np.cos(np.float32(2) * y)) *
              (np.cos(np.float32(2) * z) + np.float32(2))).astype(np.float32)
        du = torch.from_numpy(u0).cuda()
        dp = torch.from_numpy(p0.astype(np.float64)).cuda()
        self.nu = float(np.float32(1.0) / np.float32(Re))
        self.ctx.call("sod_gpu_incomp_init", dptr(du), self.nu)
        self.ctx.call("sod_gpu_incomp_set_pressure", dptr(dp))
        self.ctx.call("sod_gpu_incomp_set_veloc_solver", int(veloc[0]), float(veloc[1]))
        self.cfl = cfl_conv
        self.time = np.float32(0.0)
        self.dt = self.adapt_dt()
        self.stats = SolveStats()

    def adapt_dt(self) -> float:
        v = C.c_float()
        self.ctx.call("sod_gpu_incomp_adapt_dt", self.cfl, C.byref(v))
        return float(v.value)

    def analysis(self):
        out = (C.c_double * 4)()
        self.ctx.call("sod_gpu_incomp_analysis", out)
        return [float(self.time)] + list(out) + [0.0]

    def step(self, opts):
        self.ctx.call("sod_gpu_incomp_step", float(self.dt), C.byref(opts), C.byref(self.stats))
        self.time = np.float32(self.time + np.float32(self.dt))

    def run(self, nsteps, opts, log_first=1, log_step=10, max_time=None):
        hist = [self.analysis()]
        log_next = log_first
        for istep in range(1, nsteps + 1):
            self.step(opts)
            if istep == log_next:
                hist.append(self.analysis())
                log_next += log_step
            self.dt = self.adapt_dt()
            if max_time is not None and self.time >= np.float32(max_time):
                break
        return np.array(hist)

    def close(self):
        self.ctx.close()
