"""Oracle test infrastructure only: Python access to the CPU oracle.

* ``Oracle`` wraps ``oracle/liboracle.so`` (the C++ restatement in ``nsf_oracle.hpp``) through ctypes.
* ``run_reference`` runs ``oracle/_ref/ref_runner`` (the reference solver itself, built by
  ``oracle/Makefile.ref``) and ``read_ref_setup`` / ``read_ref_fields`` / ``read_ref_history`` parse its dumps.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use this module, as the checker.
"""
import ctypes
import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_RUNNER = os.path.join(HERE, "_ref", "ref_runner")
FIELD_NAMES = ["rho", "rho_u", "rho_v", "rho_w", "rho_E", "u", "v", "w", "p", "T", "mu", "kappa"]

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("oracle/liboracle.so is not built (run __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        vp, u64, dbl = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_double
        L.nsfo_create.restype = vp
        L.nsfo_create.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        L.nsfo_initialize.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
        L.nsfo_set_frozen_dt.argtypes = [vp, ctypes.POINTER(dbl), u64]
        L.nsfo_set_exact_image_solve.argtypes = [vp, ctypes.c_int]
        L.nsfo_march.restype = dbl
        L.nsfo_march.argtypes = [vp, u64]
        L.nsfo_last_error.restype = ctypes.c_int
        L.nsfo_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
        for name, rt in [("nsfo_num_nodes", u64), ("nsfo_time", dbl), ("nsfo_time_level", u64), ("nsfo_dt", dbl),
                         ("nsfo_non_finite", ctypes.c_int), ("nsfo_num_bodies", u64)]:
            getattr(L, name).restype = rt
            getattr(L, name).argtypes = [vp]
        L.nsfo_geometry.argtypes = [vp, ctypes.POINTER(dbl)]
        L.nsfo_get_fields.argtypes = [vp, ctypes.POINTER(dbl)]
        L.nsfo_get_old.argtypes = [vp, ctypes.POINTER(dbl)]
        L.nsfo_rhs.argtypes = [vp, ctypes.POINTER(dbl)]
        L.nsfo_set_conserved.argtypes = [vp, ctypes.POINTER(dbl)]
        L.nsfo_get_types.argtypes = [vp, ctypes.POINTER(ctypes.c_uint8)]
        for name in ("nsfo_num_ghosts", "nsfo_num_filter", "nsfo_closure_added"):
            getattr(L, name).restype = u64
            getattr(L, name).argtypes = [vp, u64]
        L.nsfo_get_ghosts.argtypes = [vp, u64, ctypes.POINTER(dbl)]
        L.nsfo_get_filter.argtypes = [vp, u64, ctypes.POINTER(ctypes.c_uint64)]
        L.nsfo_history.restype = u64
        L.nsfo_history.argtypes = [vp, ctypes.POINTER(dbl)]
        L.nsfo_destroy.argtypes = [vp]
        L.nsfo_dual_objective.argtypes = [ctypes.c_char_p] + [ctypes.POINTER(dbl)] * 5 + [u64, u64] + \
            [ctypes.POINTER(dbl)] * 2 + [ctypes.c_char_p, ctypes.c_int]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def dual_objective(cfg_text, dts, navg, u0=None, du0=None, inflow=None, dinflow=None):
    """(J, dJ): the adjoint's objective (the bodies' x-force averaged over the last navg steps of a run of
    len(dts) steps with that frozen dt sequence) and its exact directional derivative along (du0, dinflow)
    by dual-number differentiation of the oracle (nsfo_dual_objective)."""
    keep = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
            for a in (u0, du0, inflow, dinflow)]
    dts = np.ascontiguousarray(dts, dtype=np.float64)
    J, dJ = ctypes.c_double(), ctypes.c_double()
    err = ctypes.create_string_buffer(512)
    st = lib().nsfo_dual_objective(cfg_text.encode(), *[None if a is None else _dp(a) for a in keep], _dp(dts),
                                   len(dts), navg, ctypes.byref(J), ctypes.byref(dJ), err, 512)
    if st:
        raise RuntimeError(err.value.decode())
    return J.value, dJ.value


class Oracle:
    """The CPU restatement of the reference solver, driven like Solver/Simulation."""

    def __init__(self, cfg_text, exact_image_solve=False):
        """exact_image_solve: solve the image-point systems in extended precision (see nsf_oracle.hpp)."""
        L = lib()
        err = ctypes.create_string_buffer(512)
        self.h = L.nsfo_create(cfg_text.encode(), 1, err, 512)
        if not self.h:
            raise RuntimeError("oracle config error: " + err.value.decode())
        if exact_image_solve:
            L.nsfo_set_exact_image_solve(self.h, 1)
        if L.nsfo_initialize(self.h, err, 512) != 0:
            raise RuntimeError("oracle initialize error: " + err.value.decode())
        self.N = int(L.nsfo_num_nodes(self.h))

    def close(self):
        if self.h:
            lib().nsfo_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_frozen_dt(self, dts):
        a = np.ascontiguousarray(dts, dtype=np.float64)
        lib().nsfo_set_frozen_dt(self.h, _dp(a), len(a))

    def march(self, nsteps):
        """Wall seconds of nsteps steps; RuntimeError if the reference algorithm throws on the way."""
        sec = lib().nsfo_march(self.h, nsteps)
        if sec < 0:
            buf = ctypes.create_string_buffer(512)
            lib().nsfo_last_error(self.h, buf, 512)
            raise RuntimeError("oracle march error: " + buf.value.decode())
        return sec

    @property
    def t(self):
        return lib().nsfo_time(self.h)

    @property
    def time_level(self):
        return int(lib().nsfo_time_level(self.h))

    @property
    def dt(self):
        return lib().nsfo_dt(self.h)

    @property
    def non_finite(self):
        return bool(lib().nsfo_non_finite(self.h))

    def geometry(self):
        g = np.zeros(6)
        lib().nsfo_geometry(self.h, _dp(g))
        return g

    def fields(self):
        out = np.empty((12, self.N))
        lib().nsfo_get_fields(self.h, _dp(out))
        return out

    def rhs(self):
        """RHS (5, N) of the current state at the interior nodes (zero elsewhere)."""
        out = np.zeros((5, self.N))
        lib().nsfo_rhs(self.h, _dp(out))
        return out

    def old_conserved(self):
        out = np.empty((5, self.N))
        lib().nsfo_get_old(self.h, _dp(out))
        return out

    def set_conserved(self, u5):
        a = np.ascontiguousarray(u5, dtype=np.float64)
        lib().nsfo_set_conserved(self.h, _dp(a))

    def node_types(self):
        out = np.empty(self.N, np.uint8)
        lib().nsfo_get_types(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
        return out

    def bodies(self):
        """[(ghosts[n,9] = i,j,k,bi_xyz,ip_xyz ; filter[m] ; closure_added)] per body."""
        L = lib()
        res = []
        for b in range(int(L.nsfo_num_bodies(self.h))):
            ng, nf = int(L.nsfo_num_ghosts(self.h, b)), int(L.nsfo_num_filter(self.h, b))
            g = np.zeros((ng, 9))
            f = np.zeros(nf, np.uint64)
            if ng:
                L.nsfo_get_ghosts(self.h, b, _dp(g))
            if nf:
                L.nsfo_get_filter(self.h, b, f.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
            res.append((g, f, int(L.nsfo_closure_added(self.h, b))))
        return res

    def history(self):
        """rows: t after step, dt used, norms(5) (-1 where not recorded)."""
        n = int(lib().nsfo_history(self.h, None))
        out = np.zeros((n, 7))
        if n:
            lib().nsfo_history(self.h, _dp(out))
        return out


# ------------------------------------------------------------------ reference runner dumps
def ref_available():
    return os.path.exists(REF_RUNNER)


def run_reference(cfg_path, dumps, outdir=None, final=False):
    outdir = outdir or tempfile.mkdtemp(prefix="nsf_ref_")
    cmd = [REF_RUNNER, cfg_path, outdir, "--dump", ",".join(str(d) for d in dumps)]
    if final:
        cmd.append("--final")
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
    return outdir


def time_reference(cfg_path, warm, steps):
    import json
    out = subprocess.run([REF_RUNNER, cfg_path, tempfile.gettempdir(), "--time", str(warm), str(steps)],
                         check=True, capture_output=True, text=True).stdout
    return json.loads(out.strip().splitlines()[-1])


def read_ref_setup(outdir):
    b = open(os.path.join(outdir, "setup.bin"), "rb").read()
    magic, NI, NJ, NK = struct.unpack_from("<4Q", b, 0)
    o = 32
    geo = struct.unpack_from("<6d", b, o)
    o += 48
    N = NI * NJ * NK
    types = np.frombuffer(b, np.uint8, N, o).copy()
    o += N
    (nb,) = struct.unpack_from("<Q", b, o)
    o += 8
    bodies = []
    for _ in range(nb):
        (ng,) = struct.unpack_from("<Q", b, o)
        o += 8
        raw = np.frombuffer(b, np.uint8, ng * 72, o).reshape(ng, 72)
        o += ng * 72
        ijk = raw[:, :24].copy().view(np.uint64).reshape(ng, 3).astype(np.float64)
        pts = raw[:, 24:].copy().view(np.float64).reshape(ng, 6)
        g = np.concatenate([ijk, pts], axis=1) if ng else np.zeros((0, 9))
        (nf,) = struct.unpack_from("<Q", b, o)
        o += 8
        f = np.frombuffer(b, np.uint64, nf, o).copy()
        o += 8 * nf
        bodies.append((g, f))
    (dt0,) = struct.unpack_from("<d", b, o)
    return dict(shape=(NI, NJ, NK), geometry=np.array(geo), types=types, bodies=bodies, dt0=dt0)


def read_ref_fields(outdir, level):
    path = os.path.join(outdir, "fields_final.bin" if level == "final" else "fields_%06d.bin" % level)
    raw = np.fromfile(path, dtype=np.float64)
    t, lvl, dt = raw[0], raw[1:2].view(np.uint64)[0], raw[2]
    return dict(t=t, level=int(lvl), dt=dt, fields=raw[3:].reshape(12, -1))


def read_ref_history(outdir):
    """rows: t after step, dt used, dt next, norms(5)."""
    return np.fromfile(os.path.join(outdir, "history.bin"), dtype=np.float64).reshape(-1, 8)
