"""ctypes binding of the C ABI in include/nsfsi.h (the B200 time-marching path).

The library is 3d-ns-fsi_b200/lib/libnsfsi.so, built in-tree by ``__graft_entry__.build()``. There is no
CPU fallback: if the library is missing or no sm_100 device is present, the calls fail loudly.
"""
import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ROOT = os.path.dirname(PKG)
# NSFSI_LIB overrides the library path (e.g. to compare two builds of the native library).
LIB_PATH = os.environ.get("NSFSI_LIB") or os.path.join(PKG, "lib", "libnsfsi.so")
HEADER = os.path.join(ROOT, "include", "nsfsi.h")
CASES = os.path.join(PKG, "cases")

FIELDS = ["rho", "rho_u", "rho_v", "rho_w", "rho_E", "u", "v", "w", "p", "T", "mu", "kappa"]
STATUS = {0: "NSF_OK", 1: "NSF_ERR_CONFIG", 2: "NSF_ERR_CUDA", 3: "NSF_ERR_NONFINITE", 4: "NSF_ERR_GEOMETRY",
          5: "NSF_ERR_TIMEOUT", 6: "NSF_ERR_ARG", 7: "NSF_ERR_STATE"}
BC = {"periodic": 0, "symmetry": 1, "inlet": 2, "outlet": 3}
IC = {"stagnation": 0, "freestream_noise": 1, "tgv": 2}
MAXF, MAXS, MAXC = 16, 64, 16


class Sphere(ctypes.Structure):
    _fields_ = [("cx", ctypes.c_double), ("cy", ctypes.c_double), ("cz", ctypes.c_double), ("r", ctypes.c_double)]


class Cylinder(ctypes.Structure):
    _fields_ = [("axis", ctypes.c_int32), ("cx", ctypes.c_double), ("cy", ctypes.c_double), ("cz", ctypes.c_double),
                ("r", ctypes.c_double)]


class Config(ctypes.Structure):
    """nsf_config: every ConfigSettings member plus the case description."""
    _i32, _u64, _d = ctypes.c_int32, ctypes.c_uint64, ctypes.c_double
    _fields_ = [("NI", _u64), ("NJ", _u64), ("NK", _u64), ("stop_criterion", _i32), ("stop_time_level", _u64),
                ("t_end", _d), ("conv_stability_limit", _d), ("visc_stability_limit", _d),
                ("n_filter_intervals", _i32), ("filter_intervals", ctypes.c_uint32 * MAXF),
                ("n_filter_change_times", _i32), ("filter_change_times", _d * MAXF), ("status_report_interval", _d),
                ("save_density", _i32), ("save_momentum", _i32), ("save_energy", _i32), ("save_velocity", _i32),
                ("save_pressure", _i32), ("save_temperature", _i32), ("save_viscosity", _i32),
                ("save_thermal_cond", _i32), ("save_ic", _i32), ("save_final", _i32), ("save_intervals", _i32),
                ("save_period", _d), ("save_intervals_start_time", _d), ("save_intervals_end_time", _d),
                ("conv_history", _i32), ("gamma", _d), ("pr", _d), ("r_gas", _d), ("re", _d), ("sutherlands_c1", _d),
                ("sutherlands_c2", _d), ("m0", _d), ("t0", _d), ("lx", _d), ("ly", _d), ("lz", _d),
                ("machine_precision_buffer", _d), ("shipped_case", _i32), ("bc", (_i32 * 2) * 3),
                ("n_spheres", _i32), ("spheres", Sphere * MAXS), ("n_cylinders", _i32),
                ("cylinders", Cylinder * MAXC), ("ic", _i32), ("noise_amp", _d), ("seed", _u64)]


class NsfError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s: %s" % (STATUS.get(code, code), msg))
        self.code = code


_lib = None


def lib():
    """Load libnsfsi.so and declare its signatures (raises if the native library is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("native library %s is missing: run __graft_entry__.build()" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    vp, i32, u32, u64, dp = ctypes.c_void_p, ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER(ctypes.c_double)
    cp = ctypes.POINTER(Config)
    sig = {
        "nsf_abi_version": (i32, []),
        "nsf_config_defaults": (i32, [cp]),
        "nsf_config_load": (i32, [ctypes.c_char_p, cp, ctypes.c_char_p, ctypes.c_size_t]),
        "nsf_config_parse": (i32, [ctypes.c_char_p, cp, ctypes.c_char_p, ctypes.c_size_t]),
        "nsf_create": (i32, [cp, i32, ctypes.POINTER(vp)]),
        "nsf_initialize": (i32, [vp]),
        "nsf_march": (i32, [vp, u64]),
        "nsf_sync": (i32, [vp]),
        "nsf_get_time": (i32, [vp, dp, ctypes.POINTER(u64), dp]),
        "nsf_download": (i32, [vp, u32, dp]),
        "nsf_download_async": (i32, [vp, u32, dp, ctypes.POINTER(u64)]),
        "nsf_download_wait": (i32, [vp, u64]),
        "nsf_download_done": (i32, [vp, u64, ctypes.POINTER(i32)]),
        "nsf_host_alloc": (i32, [ctypes.c_size_t, ctypes.POINTER(vp)]),
        "nsf_host_free": (i32, [vp]),
        "nsf_upload_conserved": (i32, [vp, dp]),
        "nsf_get_node_types": (i32, [vp, ctypes.POINTER(ctypes.c_uint8)]),
        "nsf_get_geometry": (i32, [vp, dp]),
        "nsf_get_num_bodies": (i32, [vp, ctypes.POINTER(u32)]),
        "nsf_get_body_interaction": (i32, [vp, ctypes.POINTER(i32)]),
        "nsf_get_body_counts": (i32, [vp, u32, ctypes.POINTER(u64), ctypes.POINTER(u64), ctypes.POINTER(u64)]),
        "nsf_get_ghosts": (i32, [vp, u32, dp]),
        "nsf_get_filter_nodes": (i32, [vp, u32, ctypes.POINTER(u64)]),
        "nsf_get_history": (i32, [vp, u64, u64, dp, ctypes.POINTER(u64)]),
        "nsf_launches_per_step": (i32, [vp, ctypes.POINTER(u64)]),
        "nsf_march_timed": (i32, [vp, u64, dp]),
        "nsf_profile_steps": (i32, [vp, u64, dp, dp]),
        "nsf_step_metrics_noalloc": (i32, [cp, vp, vp, vp, vp, vp]),
        "nsf_ensemble_create": (i32, [cp, u32, i32, ctypes.c_char_p, ctypes.POINTER(vp)]),
        "nsf_ensemble_march": (i32, [vp, u64]),
        "nsf_ensemble_march_timed": (i32, [vp, u64, dp]),
        "nsf_ensemble_sync": (i32, [vp]),
        "nsf_ensemble_profile_steps": (i32, [vp, u64, dp, dp]),
        "nsf_ensemble_member": (i32, [vp, u32, ctypes.POINTER(vp)]),
        "nsf_ensemble_info": (i32, [vp, ctypes.POINTER(i32), ctypes.POINTER(u64), ctypes.POINTER(u32)]),
        "nsf_ensemble_last_error": (ctypes.c_char_p, [vp]),
        "nsf_ensemble_destroy": (None, [vp]),
        "nsf_autotune": (i32, [cp, i32, ctypes.c_char_p, ctypes.POINTER(i32), dp]),
        "nsf_slab_plan": (i32, [cp, i32, ctypes.POINTER(i32), ctypes.POINTER(i32)]),
        "nsf_slab_group_create": (i32, [cp, i32, i32, ctypes.POINTER(vp)]),
        "nsf_slab_group_march": (i32, [vp, u64]),
        "nsf_slab_group_march_timed": (i32, [vp, u64, dp]),
        "nsf_slab_group_sync": (i32, [vp]),
        "nsf_slab_group_download": (i32, [vp, u32, dp]),
        "nsf_slab_group_solver": (i32, [vp, i32, ctypes.POINTER(vp)]),
        "nsf_slab_group_info": (i32, [vp, ctypes.POINTER(i32), ctypes.POINTER(i32), ctypes.POINTER(u64)]),
        "nsf_slab_group_last_error": (ctypes.c_char_p, [vp]),
        "nsf_slab_group_destroy": (None, [vp]),
        "nsf_slab_nccl_id": (i32, [ctypes.POINTER(ctypes.c_uint8)]),
        "nsf_slab_group_create_ranks": (i32, [cp, i32, i32, i32, ctypes.POINTER(ctypes.c_uint8), i32, i32,
                                              ctypes.POINTER(vp)]),
        "nsf_slab_schedule": (i32, [cp, i32, i32, ctypes.POINTER(i32), ctypes.POINTER(i32), ctypes.POINTER(i32)]),
        "nsf_adj_configure": (i32, [vp, u32, u32]),
        "nsf_adj_forward": (i32, [vp, dp, dp, dp]),
        "nsf_adj_set_tape_limit": (i32, [vp, u64]),
        "nsf_adj_tape_bytes": (i32, [vp, ctypes.POINTER(u64)]),
        "nsf_adj_segment_tape": (i32, [vp, ctypes.POINTER(u64), ctypes.POINTER(u32)]),
        "nsf_adj_backward": (i32, [vp, ctypes.c_double, dp, dp]),
        "nsf_adj_get_dt": (i32, [vp, dp, ctypes.POINTER(u64)]),
        "nsf_adj_profile_step": (i32, [vp, u64, dp]),
        "nsf_math_selftest": (i32, [i32, u64, dp, dp]),
        "nsf_debug_wait_limit": (i32, [vp, u64, i32]),
        "nsf_last_error": (ctypes.c_char_p, [vp]),
        "nsf_destroy": (None, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def config_defaults():
    c = Config()
    lib().nsf_config_defaults(ctypes.byref(c))
    return c


def config_parse(text):
    c = Config()
    err = ctypes.create_string_buffer(1024)
    st = lib().nsf_config_parse(text.encode(), ctypes.byref(c), err, 1024)
    if st:
        raise NsfError(st, err.value.decode())
    return c


def config_load(path):
    c = Config()
    err = ctypes.create_string_buffer(1024)
    st = lib().nsf_config_load(path.encode(), ctypes.byref(c), err, 1024)
    if st:
        raise NsfError(st, err.value.decode())
    return c


def case_path(name):
    return os.path.join(CASES, name + ".cfg")


def math_selftest(x, device=0):
    """(4, n): the device's Newton-Raphson reciprocal, IEEE 1/x, Newton-Raphson square root, IEEE sqrt."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros(4 * x.size)
    st = lib().nsf_math_selftest(device, x.size, _dp(x), _dp(out))
    if st:
        raise NsfError(st, "nsf_math_selftest failed")
    return out.reshape(-1, 4).T


class Snapshot:
    """A download in flight (Solver.download_async): its page-locked host buffer and ticket. The buffer is
    released after the copy has landed, so dropping a Snapshot early is safe."""

    def __init__(self, solver, nfields):
        self.solver, self.ticket, self.shape = solver, 0, (nfields, solver.N)
        self.mem = ctypes.c_void_p()
        st = lib().nsf_host_alloc(8 * nfields * solver.N, ctypes.byref(self.mem))
        if st:
            raise NsfError(st, "nsf_host_alloc of %d bytes failed" % (8 * nfields * solver.N))

    def _ptr(self):
        return ctypes.cast(self.mem, ctypes.POINTER(ctypes.c_double))

    def done(self):
        d = ctypes.c_int32()
        self.solver._check(lib().nsf_download_done(self.solver.h, self.ticket, ctypes.byref(d)))
        return bool(d.value)

    def wait(self):
        """Block until the snapshot has landed; returns a copy of it as a (fields, N) array."""
        st = lib().nsf_download_wait(self.solver.h, self.ticket)
        if st:
            raise NsfError(st, "nsf_download_wait failed")
        n = self.shape[0] * self.shape[1]
        return np.ctypeslib.as_array(self._ptr(), shape=(n,)).reshape(self.shape).copy()

    def release(self):
        if self.mem:
            if self.ticket and self.solver.h:
                lib().nsf_download_wait(self.solver.h, self.ticket)
            lib().nsf_host_free(self.mem)
            self.mem = ctypes.c_void_p()

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class Solver:
    """One solver handle: Solver / Mesh / Simulation state resident on one GPU."""

    def __init__(self, cfg, device=0, initialize=True):
        if isinstance(cfg, str):
            cfg = config_load(cfg) if os.path.exists(cfg) else config_parse(cfg)
        self.cfg = cfg
        self.h = ctypes.c_void_p()
        L = lib()
        st = L.nsf_create(ctypes.byref(cfg), device, ctypes.byref(self.h))
        if st:
            msg = L.nsf_last_error(self.h).decode() if self.h else ""
            self.close()
            raise NsfError(st, msg)
        self.N = int(cfg.NI * cfg.NJ * cfg.NK)
        if initialize:
            self._check(L.nsf_initialize(self.h))

    def _check(self, st):
        if st:
            raise NsfError(st, lib().nsf_last_error(self.h).decode())

    def close(self):
        if self.h:
            lib().nsf_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def march(self, nsteps):
        self._check(lib().nsf_march(self.h, nsteps))

    def sync(self):
        self._check(lib().nsf_sync(self.h))

    def time(self):
        t, lv, dt = ctypes.c_double(), ctypes.c_uint64(), ctypes.c_double()
        self._check(lib().nsf_get_time(self.h, ctypes.byref(t), ctypes.byref(lv), ctypes.byref(dt)))
        return t.value, lv.value, dt.value

    def download(self, fields=range(12)):
        fields = sorted(fields)
        mask = 0
        for f in fields:
            mask |= 1 << f
        out = np.empty((len(fields), self.N))
        self._check(lib().nsf_download(self.h, mask, _dp(out)))
        return out

    def download_async(self, fields=range(12)):
        """Start a snapshot of `fields` that travels to the host while later steps march
        (nsf_download_async); returns a Snapshot whose wait() gives the (len(fields), N) array."""
        fields = sorted(fields)
        mask = 0
        for f in fields:
            mask |= 1 << f
        snap = Snapshot(self, len(fields))
        t = ctypes.c_uint64()
        self._check(lib().nsf_download_async(self.h, mask, snap._ptr(), ctypes.byref(t)))
        snap.ticket = t.value
        return snap

    def debug_wait_limit(self, polls=0, withhold_epilogue=False):
        """Test support: the stage kernel's wait limit in polls (0: default) and the switch that withholds
        its epilogue loads (nsf_debug_wait_limit)."""
        self._check(lib().nsf_debug_wait_limit(self.h, polls, 1 if withhold_epilogue else 0))

    def upload_conserved(self, u5):
        a = np.ascontiguousarray(u5, dtype=np.float64)
        self._check(lib().nsf_upload_conserved(self.h, _dp(a)))

    def node_types(self):
        out = np.empty(self.N, np.uint8)
        self._check(lib().nsf_get_node_types(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))
        return out

    def bodies(self):
        L = lib()
        nb = ctypes.c_uint32()
        self._check(L.nsf_get_num_bodies(self.h, ctypes.byref(nb)))
        res = []
        for b in range(nb.value):
            ng, nf, cl = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
            self._check(L.nsf_get_body_counts(self.h, b, ctypes.byref(ng), ctypes.byref(nf), ctypes.byref(cl)))
            g = np.zeros((ng.value, 9))
            f = np.zeros(nf.value, np.uint64)
            if ng.value:
                self._check(L.nsf_get_ghosts(self.h, b, _dp(g)))
            if nf.value:
                self._check(L.nsf_get_filter_nodes(self.h, b, f.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
            res.append((g, f, cl.value))
        return res

    def bodies_interact(self):
        """True if immersed bodies reach each other's nodes (nsf_get_body_interaction)."""
        v = ctypes.c_int32()
        self._check(lib().nsf_get_body_interaction(self.h, ctypes.byref(v)))
        return bool(v.value)

    def history(self, first=0, count=None):
        avail = ctypes.c_uint64()
        self._check(lib().nsf_get_history(self.h, 0, 0, None, ctypes.byref(avail)))
        count = avail.value - first if count is None else count
        out = np.zeros((count, 7))
        if count:
            self._check(lib().nsf_get_history(self.h, first, count, _dp(out), ctypes.byref(avail)))
        return out

    def march_timed(self, nsteps):
        """March nsteps; device time (ms) from CUDA events on the solver's own stream."""
        ms = ctypes.c_double()
        self._check(lib().nsf_march_timed(self.h, nsteps, ctypes.byref(ms)))
        return ms.value

    def profile_steps(self, nsteps):
        """March nsteps launched eagerly; returns (mean ms of each stage kernel [4], mean ms per step)."""
        st = np.zeros(4)
        step = ctypes.c_double()
        self._check(lib().nsf_profile_steps(self.h, nsteps, _dp(st), ctypes.byref(step)))
        return st, step.value

    def launches_per_step(self):
        n = ctypes.c_uint64()
        self._check(lib().nsf_launches_per_step(self.h, ctypes.byref(n)))
        return n.value

    # ---------------------------------------------------------------- discrete adjoint
    def adj_configure(self, avg_last_steps=50, snapshots=20):
        self._check(lib().nsf_adj_configure(self.h, avg_last_steps, snapshots))

    def adj_tape_limit(self, nbytes):
        """Device memory the adjoint's tape may take (0: checkpointing only; None: the default, half the
        free device memory)."""
        self._check(lib().nsf_adj_set_tape_limit(self.h, (1 << 64) - 1 if nbytes is None else int(nbytes)))

    def adj_tape_bytes(self):
        n = ctypes.c_uint64()
        self._check(lib().nsf_adj_tape_bytes(self.h, ctypes.byref(n)))
        return n.value

    def adj_segment_tape(self):
        """(bytes, steps per segment) of the segment tape the last forward run left for the backward run
        ((0, 0): none)."""
        n, L = ctypes.c_uint64(), ctypes.c_uint32()
        self._check(lib().nsf_adj_segment_tape(self.h, ctypes.byref(n), ctypes.byref(L)))
        return n.value, L.value

    def adj_forward(self, u0=None, inflow=None):
        """J of a run from level 0 (u0: (5, N) conserved field or None for the case's IC; inflow: (NJ, NK)
        inlet profile factor or None for 1)."""
        J = ctypes.c_double()
        a = None if u0 is None else np.ascontiguousarray(u0, dtype=np.float64)
        b = None if inflow is None else np.ascontiguousarray(inflow, dtype=np.float64)
        self._check(lib().nsf_adj_forward(self.h, None if a is None else _dp(a), None if b is None else _dp(b),
                                          ctypes.byref(J)))
        return J.value

    def adj_backward(self, dJ=1.0):
        """(gradient w.r.t. the inflow profile factor (NJ, NK), gradient w.r.t. the level-0 field (5, N))."""
        c = self.cfg
        gi = np.zeros((int(c.NJ), int(c.NK)))
        gu = np.zeros((5, self.N))
        self._check(lib().nsf_adj_backward(self.h, dJ, _dp(gi), _dp(gu)))
        return gi, gu

    # slots of nsf_adj_profile_step's result (None: unused)
    ADJ_PHASES = ("recompute", None, "boundary_combine", None, None, None, None, "rhs", "density_filter")

    def adj_profile_step(self, step=0):
        """{phase: device ms} of one eagerly launched adjoint step (after adj_forward)."""
        ms = np.zeros(len(self.ADJ_PHASES))
        self._check(lib().nsf_adj_profile_step(self.h, step, _dp(ms)))
        return {k: v for k, v in zip(self.ADJ_PHASES, ms.tolist()) if k}

    def adj_dt(self):
        n = ctypes.c_uint64()
        self._check(lib().nsf_adj_get_dt(self.h, None, ctypes.byref(n)))
        out = np.zeros(n.value)
        self._check(lib().nsf_adj_get_dt(self.h, _dp(out), ctypes.byref(n)))
        return out

    def geometry(self):
        """dx, dy, dz and Mesh::positionOffset x, y, z."""
        g = np.zeros(6)
        self._check(lib().nsf_get_geometry(self.h, _dp(g)))
        return g


class Member(Solver):
    """Read-only view of one ensemble member (owned by its Ensemble: never destroyed or marched here)."""

    def __init__(self, handle, cfg):
        self.cfg = cfg
        self.h = handle
        self.N = int(cfg.NI * cfg.NJ * cfg.NK)

    def close(self):
        self.h = ctypes.c_void_p()


class Ensemble:
    """Independent grids advanced together: one CUDA graph per RK4 step for all members."""

    def __init__(self, cfgs, device=0, tune_cache=None):
        self.cfgs = [config_load(c) if isinstance(c, str) and os.path.exists(c) else
                     (config_parse(c) if isinstance(c, str) else c) for c in cfgs]
        arr = (Config * len(self.cfgs))(*self.cfgs)
        self.h = ctypes.c_void_p()
        st = lib().nsf_ensemble_create(arr, len(self.cfgs), device, tune_cache.encode() if tune_cache else None,
                                       ctypes.byref(self.h))
        if st:
            msg = lib().nsf_ensemble_last_error(self.h).decode() if self.h else ""
            self.close()
            raise NsfError(st, msg)

    def _check(self, st):
        if st:
            raise NsfError(st, lib().nsf_ensemble_last_error(self.h).decode())

    def close(self):
        if self.h:
            lib().nsf_ensemble_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def march(self, nsteps):
        self._check(lib().nsf_ensemble_march(self.h, nsteps))

    def march_timed(self, nsteps):
        ms = ctypes.c_double()
        self._check(lib().nsf_ensemble_march_timed(self.h, nsteps, ctypes.byref(ms)))
        return ms.value

    def sync(self):
        self._check(lib().nsf_ensemble_sync(self.h))

    def profile_steps(self, nsteps):
        """(mean ms of each stage launch [4], mean ms per step), kernels launched one by one."""
        st = np.zeros(4)
        step = ctypes.c_double()
        self._check(lib().nsf_ensemble_profile_steps(self.h, nsteps, _dp(st), ctypes.byref(step)))
        return st, step.value

    def member(self, m):
        h = ctypes.c_void_p()
        self._check(lib().nsf_ensemble_member(self.h, m, ctypes.byref(h)))
        return Member(h, self.cfgs[m])

    def info(self):
        """(tile shape, launches per step, stage work items)."""
        tile, lps, items = ctypes.c_int32(), ctypes.c_uint64(), ctypes.c_uint32()
        self._check(lib().nsf_ensemble_info(self.h, ctypes.byref(tile), ctypes.byref(lps), ctypes.byref(items)))
        return tile.value, lps.value, items.value


def slab_plan(cfg, nslabs):
    """[(first, last)] interior planes each of nslabs x-slabs computes (nsf_slab_plan)."""
    if isinstance(cfg, str):
        cfg = config_load(cfg) if os.path.exists(cfg) else config_parse(cfg)
    a = (ctypes.c_int32 * nslabs)()
    b = (ctypes.c_int32 * nslabs)()
    st = lib().nsf_slab_plan(ctypes.byref(cfg), nslabs, a, b)
    if st:
        raise NsfError(st, "nsf_slab_plan")
    return list(zip(list(a), list(b)))


NCCL_ID_BYTES = 128
SLAB_NCCL_ALL = 1


def slab_nccl_id():
    """The NCCL communicator id (bytes) for nsf_slab_group_create_ranks, made on one process of the group."""
    buf = (ctypes.c_uint8 * NCCL_ID_BYTES)()
    st = lib().nsf_slab_nccl_id(buf)
    if st:
        raise NsfError(st, "nsf_slab_nccl_id: NCCL (libnccl.so.2) unavailable")
    return bytes(buf)


def slab_schedule(cfg, nslabs, world):
    """(owner per slab, [(list, from slab, from plane, to slab, to plane)]) of nslabs x-slabs over `world`
    processes, transfers in the order every process issues them (nsf_slab_schedule; host only)."""
    if isinstance(cfg, str):
        cfg = config_load(cfg) if os.path.exists(cfg) else config_parse(cfg)
    owner = (ctypes.c_int32 * nslabs)()
    n = ctypes.c_int32(0)
    st = lib().nsf_slab_schedule(ctypes.byref(cfg), nslabs, world, owner, None, ctypes.byref(n))
    if st:
        raise NsfError(st, "nsf_slab_schedule")
    t = (ctypes.c_int32 * (5 * n.value))()
    st = lib().nsf_slab_schedule(ctypes.byref(cfg), nslabs, world, owner, t, ctypes.byref(n))
    if st:
        raise NsfError(st, "nsf_slab_schedule")
    return list(owner), [tuple(t[5 * q:5 * q + 5]) for q in range(n.value)]


class SlabGroup:
    """One grid split into x-slabs (nsf_slab_group_*): all slabs on one device, or (rank, world, nccl_id
    given) this process's share of a group spread over `world` processes that exchange planes by NCCL.
    With torch.distributed, e.g.: ids = [nsfsi.slab_nccl_id() if rank == 0 else None];
    dist.broadcast_object_list(ids, src=0); SlabGroup(cfg, n, device, rank, world, ids[0])."""

    def __init__(self, cfg, nslabs, device=0, rank=None, world=None, nccl_id=None, flags=0):
        if isinstance(cfg, str):
            cfg = config_load(cfg) if os.path.exists(cfg) else config_parse(cfg)
        self.cfg = cfg
        self.N = int(cfg.NI * cfg.NJ * cfg.NK)
        self.h = ctypes.c_void_p()
        if nccl_id is None:
            st = lib().nsf_slab_group_create(ctypes.byref(cfg), nslabs, device, ctypes.byref(self.h))
        else:
            idb = (ctypes.c_uint8 * NCCL_ID_BYTES).from_buffer_copy(bytes(nccl_id))
            st = lib().nsf_slab_group_create_ranks(ctypes.byref(cfg), nslabs, int(rank or 0), int(world or 1), idb,
                                                   int(flags), device, ctypes.byref(self.h))
        if st:
            msg = lib().nsf_slab_group_last_error(self.h).decode() if self.h else ""
            self.close()
            raise NsfError(st, msg)

    def _check(self, st):
        if st:
            raise NsfError(st, lib().nsf_slab_group_last_error(self.h).decode())

    def close(self):
        if self.h:
            lib().nsf_slab_group_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def march(self, nsteps):
        self._check(lib().nsf_slab_group_march(self.h, nsteps))

    def march_timed(self, nsteps):
        ms = ctypes.c_double()
        self._check(lib().nsf_slab_group_march_timed(self.h, nsteps, ctypes.byref(ms)))
        return ms.value

    def sync(self):
        self._check(lib().nsf_slab_group_sync(self.h))

    def download(self, fields=range(12)):
        fields = sorted(fields)
        mask = 0
        for f in fields:
            mask |= 1 << f
        out = np.zeros((len(fields), self.N))  # a process of a multi-process group fills its own planes
        self._check(lib().nsf_slab_group_download(self.h, mask, _dp(out)))
        return out

    def slab(self, p):
        """Slab p's solver (read-only view: time, history)."""
        h = ctypes.c_void_p()
        self._check(lib().nsf_slab_group_solver(self.h, p, ctypes.byref(h)))
        return Member(h, self.cfg)

    def info(self):
        n = ctypes.c_int32()
        self._check(lib().nsf_slab_group_info(self.h, ctypes.byref(n), None, None))
        first = (ctypes.c_int32 * n.value)()
        lps = ctypes.c_uint64()
        self._check(lib().nsf_slab_group_info(self.h, None, first, ctypes.byref(lps)))
        return n.value, list(first), lps.value


def autotune(cfg, device=0, cache=None):
    """(faster tile shape: 0 = 32x8, 1 = 16x16; ns per node and stage for both)."""
    tile = ctypes.c_int32()
    ns = np.zeros(2)
    st = lib().nsf_autotune(ctypes.byref(cfg), device, cache.encode() if cache else None, ctypes.byref(tile), _dp(ns))
    if st:
        raise NsfError(st, "autotune failed")
    return tile.value, ns


ENSEMBLE_SHAPES = [(32, 32, 32), (48, 48, 48), (64, 64, 64), (96, 64, 64), (128, 64, 64)]


def ensemble_configs(n=64, seed=20240301, steps=200):
    """The batched-ensemble workload: n single-sphere flows (inflow/outflow in x, periodic y and z) with
    grid shapes drawn from ENSEMBLE_SHAPES, Mach from U[0.2, 0.4], Re from U[50, 300] on the diameter,
    sphere diameter from U[0.15, 0.25] of the domain width (L_y = L_z = 1), centre at 40 % of the domain
    length; L_x makes dx equal to dy. Freestream + seeded 1e-4 noise, `steps` RK4 steps each."""
    rng = np.random.default_rng(seed)
    base = config_load(case_path("sphere48"))
    out = []
    for m in range(n):
        NI, NJ, NK = ENSEMBLE_SHAPES[int(rng.integers(len(ENSEMBLE_SHAPES)))]
        mach = float(rng.uniform(0.2, 0.4))
        re_d = float(rng.uniform(50.0, 300.0))
        d = float(rng.uniform(0.15, 0.25))
        c = Config()
        ctypes.memmove(ctypes.byref(c), ctypes.byref(base), ctypes.sizeof(Config))
        c.NI, c.NJ, c.NK = NI, NJ, NK
        c.stop_time_level = steps
        c.lx = float(NI - 1) / float(NJ - 2)
        c.ly = c.lz = 1.0
        c.m0 = mach
        c.re = re_d / (mach * d)
        c.machine_precision_buffer = np.finfo(np.float64).eps * (c.lx + c.ly + c.lz)
        c.n_spheres = 1
        c.spheres[0] = Sphere(0.4 * c.lx, 0.5, 0.5, d / 2)
        c.seed = seed + m
        out.append(c)
    return out
