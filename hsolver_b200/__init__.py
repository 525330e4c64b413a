"""hsolver_b200: B200-native SIMPLE conjugate-heat-transfer step.

Python mirror of the C ABI in include/hsolver_b200.h (ctypes over the in-tree
libhsolver_b200.so).  `Solver` follows the reference's driver sequence
(main.cpp:18-45, solver.h:44-158): build the case from a `.in` deck, `init()`
(FluidSolver::init + MobSolver::init), then `step(n)` outer iterations.

The CUDA library is the only compute path: if it is missing or no GPU is
present, constructing a Solver raises; there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhsolver_b200.so")

HS_OK = 0
ERRORS = {-1: "HS_ERR_ARG", -2: "HS_ERR_DECK", -3: "HS_ERR_UNSUPPORTED", -4: "HS_ERR_CUDA", -5: "HS_ERR_NOMEM",
          -6: "HS_ERR_STATE", -7: "HS_ERR_DIVERGED", -8: "HS_ERR_INTERNAL", -9: "HS_ERR_MAXITER"}
FIELDS = {"u_star": 0, "v_star": 1, "w_star": 2, "p_temp": 3, "t_temp": 4, "up": 5, "vp": 6, "wp": 7,
          "ux": 8, "uy": 9, "uz": 10, "p": 11, "t": 12, "p_prime": 13}
PSOLVE_CG, PSOLVE_MGCG = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
CH_SKIP_PRESSURE, CH_SKIP_ENERGY = 1, 2
CONV_UPWIND, CONV_HYBRID, CONV_QUICK = 0, 1, 2
CH_FIELDS = {"u": 0, "v": 1, "w": 2, "p": 3, "T": 4, "u_star": 5, "v_star": 6, "w_star": 7, "d_u": 8, "d_v": 9,
             "d_w": 10, "p_prime": 11}


class HsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s: %s" % (ERRORS.get(code, code), msg))
        self.code = code


class Params(ctypes.Structure):
    """hs_params: the reference's macros as runtime values."""
    _fields_ = [("nu", ctypes.c_double), ("rho", ctypes.c_double), ("alpha", ctypes.c_double),
                ("u_lid", ctypes.c_double), ("relax", ctypes.c_double), ("relax_solid", ctypes.c_double),
                ("mom_tol", ctypes.c_double), ("energy_tol", ctypes.c_double), ("solid_tol", ctypes.c_double),
                ("gs_max", ctypes.c_int), ("t_fluid0", ctypes.c_double), ("t_wall", ctypes.c_double),
                ("t_solid0", ctypes.c_double), ("pcg_tol", ctypes.c_double), ("pcg_maxiter", ctypes.c_int),
                ("frozen_matrix", ctypes.c_int), ("pressure_solver", ctypes.c_int),
                ("reserved", ctypes.c_int * 7)]


class Stats(ctypes.Structure):
    _fields_ = [("sweeps_u", ctypes.c_int), ("sweeps_v", ctypes.c_int), ("sweeps_w", ctypes.c_int),
                ("sweeps_t", ctypes.c_int), ("sweeps_solid_max", ctypes.c_int), ("pcg_iters", ctypes.c_int),
                ("res_u", ctypes.c_double), ("res_v", ctypes.c_double), ("res_w", ctypes.c_double),
                ("res_t", ctypes.c_double), ("pcg_relres", ctypes.c_double), ("steps", ctypes.c_longlong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def load(path=LIB_PATH):
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError("hsolver_b200 CUDA library not built: %s (run __graft_entry__.build())" % path)
    L = ctypes.CDLL(path)
    vp, ll, llp = ctypes.c_void_p, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)
    dp = ctypes.POINTER(ctypes.c_double)
    L.hs_params_default.argtypes = [ctypes.POINTER(Params)]
    L.hs_params_default.restype = None
    L.hs_create.argtypes = [ctypes.c_char_p, ctypes.POINTER(Params), ctypes.c_int, ctypes.POINTER(vp)]
    L.hs_init.argtypes = [vp]
    L.hs_step.argtypes = [vp, ctypes.c_int, ctypes.POINTER(Stats)]
    L.hs_sync.argtypes = [vp]
    L.hs_field_size.argtypes = [vp, ctypes.c_int, llp]
    L.hs_get_field.argtypes = [vp, ctypes.c_int, dp, ll]
    L.hs_set_field.argtypes = [vp, ctypes.c_int, dp, ll]
    L.hs_field_device_ptr.argtypes = [vp, ctypes.c_int, ctypes.POINTER(dp), llp]
    L.hs_fluid_meta.argtypes = [vp, llp]
    L.hs_grid_dims.argtypes = [vp, llp]
    L.hs_num_solids.argtypes = [vp]
    L.hs_solid_meta.argtypes = [vp, ctypes.c_int, llp]
    L.hs_get_solid.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, ll]
    L.hs_get_fluid_mask.argtypes = [vp, ctypes.POINTER(ctypes.c_uint8), ll]
    L.hs_get_cell_types.argtypes = [vp, ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_int), ll]
    L.hs_get_row_ids.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ll]
    L.hs_destroy.argtypes = [vp]
    L.hs_destroy.restype = None
    L.hs_last_error.argtypes = [vp]
    L.hs_last_error.restype = ctypes.c_char_p
    L.hs_stream.argtypes = [vp, ctypes.POINTER(vp)]
    L.hs_profile.argtypes = [vp, ctypes.c_int]
    L.hs_profile_read.argtypes = [vp, dp, ctypes.POINTER(ctypes.c_int)]
    L.hs_counters.argtypes = [vp, llp]
    _lib = L
    return L


def default_params(**over):
    p = Params()
    load().hs_params_default(ctypes.byref(p))
    for k, v in over.items():
        setattr(p, k, v)
    return p


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Solver:
    """One case on one GPU: the fluid region plus every solid region."""

    def __init__(self, deck_text, params=None, device=0):
        L = load()
        self._L = L
        self.h = None
        h = ctypes.c_void_p()
        p = params if params is not None else default_params()
        rc = L.hs_create(deck_text.encode() if isinstance(deck_text, str) else deck_text, ctypes.byref(p), device,
                         ctypes.byref(h))
        if rc != HS_OK:
            raise HsError(rc, L.hs_last_error(None).decode())
        self.h = h
        m = (ctypes.c_longlong * 9)()
        self._check(L.hs_fluid_meta(h, m))
        self.meta = tuple(m)
        d = (ctypes.c_longlong * 3)()
        self._check(L.hs_grid_dims(h, d))
        self.dims = tuple(d)
        self.nsolid = L.hs_num_solids(h)

    def _check(self, rc):
        if rc < 0:
            raise HsError(rc, self._L.hs_last_error(self.h).decode())
        return rc

    def close(self):
        if self.h:
            self._L.hs_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init(self):
        self._check(self._L.hs_init(self.h))

    def step(self, n=1, stats=False):
        st = Stats() if stats else None
        self._check(self._L.hs_step(self.h, n, ctypes.byref(st) if st is not None else None))
        return st.as_dict() if st is not None else None

    def sync(self):
        self._check(self._L.hs_sync(self.h))

    def field_size(self, name):
        n = ctypes.c_longlong()
        self._check(self._L.hs_field_size(self.h, FIELDS[name], ctypes.byref(n)))
        return n.value

    def field(self, name, out=None):
        n = self.field_size(name)
        out = np.empty(n, np.float64) if out is None else out
        self._check(self._L.hs_get_field(self.h, FIELDS[name], _dptr(out), n))
        return out

    def set_field(self, name, arr):
        arr = np.ascontiguousarray(arr, np.float64)
        self._check(self._L.hs_set_field(self.h, FIELDS[name], _dptr(arr), arr.size))

    def device_ptr(self, name):
        p = ctypes.POINTER(ctypes.c_double)()
        n = ctypes.c_longlong()
        self._check(self._L.hs_field_device_ptr(self.h, FIELDS[name], ctypes.byref(p), ctypes.byref(n)))
        return ctypes.cast(p, ctypes.c_void_p).value, n.value

    def solid_meta(self, r):
        m = (ctypes.c_longlong * 9)()
        self._check(self._L.hs_solid_meta(self.h, r, m))
        return tuple(m)

    def solid(self, r, which="t_temp"):
        md = self.solid_meta(r)
        n = (md[0] + 2) * (md[1] + 2) * (md[2] + 2) if which == "t_temp" else md[0] * md[1] * md[2]
        out = np.empty(n, np.float64)
        self._check(self._L.hs_get_solid(self.h, r, 0 if which == "t_temp" else 1, _dptr(out), n))
        return out

    def fluid_empty(self):
        cx, cy, cz = self.meta[:3]
        out = np.empty(cx * cy * cz, np.uint8)
        self._check(self._L.hs_get_fluid_mask(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), out.size))
        return out

    def cell_types(self):
        n = self.dims[0] * self.dims[1] * self.dims[2]
        t = np.empty(n, np.uint8)
        r = np.empty(n, np.int32)
        self._check(self._L.hs_get_cell_types(self.h, t.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                                              r.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n))
        return t, r

    def row_ids(self):
        cx, cy, cz = self.meta[:3]
        out = np.empty(cx * cy * cz, np.int32)
        self._check(self._L.hs_get_row_ids(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), out.size))
        return out

    PHASES = ["mom_u", "mom_v", "mom_w", "pressure", "correct", "energy", "solid", "swap_setfornext"]

    def profile(self, on=True):
        self._check(self._L.hs_profile(self.h, 1 if on else 0))

    def profile_read(self):
        ms = (ctypes.c_double * 8)()
        n = ctypes.c_int()
        self._check(self._L.hs_profile_read(self.h, ms, ctypes.byref(n)))
        return dict(zip(self.PHASES, list(ms))), n.value

    def counters(self):
        c = (ctypes.c_longlong * 8)()
        self._check(self._L.hs_counters(self.h, c))
        keys = ["sweeps_u", "sweeps_v", "sweeps_w", "sweeps_t", "solid_cell_sweeps", "pcg_iters", "pcg_solves", "steps"]
        return dict(zip(keys, list(c)))

    def stream(self):
        p = ctypes.c_void_p()
        self._check(self._L.hs_stream(self.h, ctypes.byref(p)))
        return p.value

    def solve(self, n_outer=100):
        """Solver::solve (solver.h:44-158): init, then n_outer outer steps."""
        self.init()
        return self.step(n_outer, stats=True)


class Case:
    """Host-only case model (no GPU): deck parse, cell types, regions, local
    boxes and interface pairs -- the reference's decompose step for one rank."""

    def __init__(self, deck_text):
        L = load()
        for name, args, res in [("hs_case_create", [ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
                                ("hs_case_dims", [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)], ctypes.c_int),
                                ("hs_case_fluid_meta", [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)], ctypes.c_int),
                                ("hs_case_num_solids", [ctypes.c_void_p], ctypes.c_int),
                                ("hs_case_solid_meta", [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)], ctypes.c_int),
                                ("hs_case_cell_types", [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_int), ctypes.c_longlong], ctypes.c_int),
                                ("hs_case_fluid_mask", [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint8), ctypes.c_longlong], ctypes.c_int),
                                ("hs_case_num_interface", [ctypes.c_void_p], ctypes.c_longlong),
                                ("hs_case_interface", [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong), ctypes.c_longlong], ctypes.c_int),
                                ("hs_case_geometry", [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_longlong], ctypes.c_int),
                                ("hs_case_destroy", [ctypes.c_void_p], None)]:
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        self._L = L
        self.h = None
        h = ctypes.c_void_p()
        rc = L.hs_case_create(deck_text.encode() if isinstance(deck_text, str) else deck_text, ctypes.byref(h))
        if rc != HS_OK:
            raise HsError(rc, L.hs_last_error(None).decode())
        self.h = h
        d = (ctypes.c_longlong * 3)()
        L.hs_case_dims(h, d)
        self.dims = tuple(d)
        m = (ctypes.c_longlong * 9)()
        L.hs_case_fluid_meta(h, m)
        self.meta = tuple(m)
        self.nsolid = L.hs_case_num_solids(h)

    def __del__(self):
        if getattr(self, "h", None):
            self._L.hs_case_destroy(self.h)
            self.h = None

    def solid_meta(self, r):
        m = (ctypes.c_longlong * 9)()
        if self._L.hs_case_solid_meta(self.h, r, m) != HS_OK:
            raise HsError(-1, "bad region")
        return tuple(m)

    def cell_types(self):
        n = self.dims[0] * self.dims[1] * self.dims[2]
        t = np.empty(n, np.uint8)
        r = np.empty(n, np.int32)
        assert self._L.hs_case_cell_types(self.h, t.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                                          r.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n) == HS_OK
        return t, r

    def fluid_empty(self):
        n = self.meta[0] * self.meta[1] * self.meta[2]
        out = np.empty(n, np.uint8)
        assert self._L.hs_case_fluid_mask(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), n) == HS_OK
        return out

    def interface(self):
        n = self._L.hs_case_num_interface(self.h)
        out = np.empty(5 * n, np.int64)
        assert self._L.hs_case_interface(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)), n) == HS_OK
        return out.reshape(n, 5)

    def geometry(self, axis):
        n = self.meta[axis] + 2
        out = np.empty(3 * n, np.float64)
        assert self._L.hs_case_geometry(self.h, axis, _dptr(out), 3 * n) == HS_OK
        return out.reshape(3, n)


class ChannelParams(ctypes.Structure):
    """hs_channel_params (include/hsolver_b200.h)."""
    _fields_ = [("re", ctypes.c_double), ("pr", ctypes.c_double), ("u_in", ctypes.c_double), ("t_in", ctypes.c_double),
                ("alpha_u", ctypes.c_double), ("alpha_p", ctypes.c_double), ("alpha_t", ctypes.c_double),
                ("mom_sweeps", ctypes.c_int), ("p_tol", ctypes.c_double), ("p_maxiter", ctypes.c_int),
                ("t_tol", ctypes.c_double), ("t_maxiter", ctypes.c_int), ("precision", ctypes.c_int),
                ("p_precond", ctypes.c_int), ("p_mg_sweeps", ctypes.c_int), ("p_level0", ctypes.c_int),
                ("conv", ctypes.c_int), ("g_axis", ctypes.c_int), ("ri", ctypes.c_double),
                ("reserved", ctypes.c_double * 3)]


class ChannelStats(ctypes.Structure):
    _fields_ = [("res", ctypes.c_double * 5), ("norm", ctypes.c_double * 5), ("global_", ctypes.c_double),
                ("iter", ctypes.c_int), ("pcg_iters", ctypes.c_int), ("t_iters", ctypes.c_int),
                ("pcg_relres", ctypes.c_double), ("t_relres", ctypes.c_double)]

    def as_dict(self):
        return {"res": list(self.res), "norm": list(self.norm), "global": self.global_, "iter": self.iter,
                "pcg_iters": self.pcg_iters, "t_iters": self.t_iters, "pcg_relres": self.pcg_relres,
                "t_relres": self.t_relres}


class AdjointInfo(ctypes.Structure):
    _fields_ = [("fwd_iters", ctypes.c_int), ("adj_iters", ctypes.c_int), ("fwd_ms", ctypes.c_double),
                ("adj_ms", ctypes.c_double)]


def _channel_api(L):
    if getattr(L, "_channel_ready", False):
        return
    vp, ll = ctypes.c_void_p, ctypes.c_longlong
    dp = ctypes.POINTER(ctypes.c_double)
    sig = {
        "hs_channel_params_default": ([ctypes.POINTER(ChannelParams)], None),
        "hs_channel_create": ([ctypes.c_char_p, ctypes.POINTER(ChannelParams), ctypes.c_int, ctypes.POINTER(vp)], ctypes.c_int),
        "hs_channel_num_blocks": ([vp, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
        "hs_channel_set_solid": ([vp, dp, ctypes.c_int, dp, ll], ctypes.c_int),
        "hs_channel_init": ([vp], ctypes.c_int),
        "hs_channel_step": ([vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ChannelStats)], ctypes.c_int),
        "hs_channel_solve_to": ([vp, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                 ctypes.POINTER(ChannelStats)], ctypes.c_int),
        "hs_channel_field_size": ([vp, ctypes.c_int, ctypes.POINTER(ll)], ctypes.c_int),
        "hs_channel_get_field": ([vp, ctypes.c_int, dp, ll], ctypes.c_int),
        "hs_channel_set_field": ([vp, ctypes.c_int, dp, ll], ctypes.c_int),
        "hs_channel_stream": ([vp, ctypes.POINTER(vp)], ctypes.c_int),
        "hs_channel_sync": ([vp], ctypes.c_int),
        "hs_channel_device_bytes": ([vp, ctypes.POINTER(ll)], ctypes.c_int),
        "hs_channel_adjoint": ([vp, ctypes.c_double, ctypes.c_int, dp, dp, ll, dp, ctypes.c_int,
                                ctypes.POINTER(AdjointInfo)], ctypes.c_int),
        "hs_channel_profile": ([vp, ctypes.c_int], ctypes.c_int),
        "hs_channel_balance": ([vp, dp], ctypes.c_int),
        "hs_channel_profile_read": ([vp, dp, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
        "hs_channel_destroy": ([vp], None),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    L._channel_ready = True


def channel_params(**over):
    L = load()
    _channel_api(L)
    p = ChannelParams()
    L.hs_channel_params_default(ctypes.byref(p))
    for k, v in over.items():
        setattr(p, k, v)
    return p


class Channel:
    """Channel conjugate-heat-transfer case on one GPU (hs_channel_*): inlet
    plug flow, zero-gradient outlet, the deck's mobs boxes as heated solid
    blocks; SIMPLE outer steps until a global residual tolerance."""

    def __init__(self, deck_text, params=None, device=0, **over):
        L = load()
        _channel_api(L)
        self._L = L
        self.h = None
        p = params if params is not None else channel_params(**over)
        h = ctypes.c_void_p()
        rc = L.hs_channel_create(deck_text.encode() if isinstance(deck_text, str) else deck_text, ctypes.byref(p), device,
                                 ctypes.byref(h))
        if rc != HS_OK:
            raise HsError(rc, L.hs_last_error(None).decode())
        self.h = h
        self.params = p
        n = ctypes.c_int()
        self._check(L.hs_channel_num_blocks(h, ctypes.byref(n)))
        self.nblocks = n.value
        self.ncell = self.field_size("p")

    def _check(self, rc):
        if rc < 0:
            raise HsError(rc, self._L.hs_last_error(None).decode())
        return rc

    def close(self):
        if self.h:
            self._L.hs_channel_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_solid(self, k_ratio, q_cell):
        k = np.ascontiguousarray(k_ratio, np.float64)
        q = np.ascontiguousarray(q_cell, np.float64)
        self._check(self._L.hs_channel_set_solid(self.h, _dptr(k), k.size, _dptr(q), q.size))

    def init(self):
        self._check(self._L.hs_channel_init(self.h))

    def step(self, n=1, flags=0):
        st = ChannelStats()
        self._check(self._L.hs_channel_step(self.h, n, flags, ctypes.byref(st)))
        return st.as_dict()

    def solve_to(self, tol=1e-6, max_outer=500):
        """Outer steps until the global residual <= tol; returns (converged, steps, stats)."""
        st = ChannelStats()
        steps = ctypes.c_int()
        rc = self._L.hs_channel_solve_to(self.h, tol, max_outer, ctypes.byref(steps), ctypes.byref(st))
        if rc < 0 and rc != -9:
            self._check(rc)
        return rc == HS_OK, steps.value, st.as_dict()

    def field_size(self, name):
        n = ctypes.c_longlong()
        self._check(self._L.hs_channel_field_size(self.h, CH_FIELDS[name], ctypes.byref(n)))
        return n.value

    def field(self, name, out=None):
        n = self.field_size(name)
        out = np.empty(n, np.float64) if out is None else out
        self._check(self._L.hs_channel_get_field(self.h, CH_FIELDS[name], _dptr(out), n))
        return out

    def set_field(self, name, arr):
        arr = np.ascontiguousarray(arr, np.float64)
        self._check(self._L.hs_channel_set_field(self.h, CH_FIELDS[name], _dptr(arr), arr.size))

    def stream(self):
        p = ctypes.c_void_p()
        self._check(self._L.hs_channel_stream(self.h, ctypes.byref(p)))
        return p.value

    def sync(self):
        self._check(self._L.hs_channel_sync(self.h))

    PHASES = ["momentum", "p_assembly", "p_solve", "correction", "energy"]

    def profile(self, on=True):
        self._check(self._L.hs_channel_profile(self.h, 1 if on else 0))

    def profile_read(self):
        ms = (ctypes.c_double * 5)()
        n = ctypes.c_int()
        self._check(self._L.hs_channel_profile_read(self.h, ms, ctypes.byref(n)))
        return dict(zip(self.PHASES, list(ms))), n.value

    def balance(self):
        """FP64 global balances of the current state (hs_channel_balance):
        volume flux in and out, heat source, heat leaving through the
        boundary."""
        out = np.empty(4)
        self._check(self._L.hs_channel_balance(self.h, _dptr(out)))
        return {"flow_in": out[0], "flow_out": out[1], "heat_source": out[2], "heat_out": out[3]}

    def device_bytes(self):
        b = ctypes.c_longlong()
        self._check(self._L.hs_channel_device_bytes(self.h, ctypes.byref(b)))
        return b.value

    def adjoint(self, tol=1e-10, maxiter=20000):
        """Energy forward + adjoint on the current flow: (J, dJdq per cell, dJdk per block, info dict)."""
        J = ctypes.c_double()
        dq = np.empty(self.ncell)
        dk = np.empty(max(self.nblocks, 1))
        info = AdjointInfo()
        self._check(self._L.hs_channel_adjoint(self.h, tol, maxiter, ctypes.byref(J), _dptr(dq), dq.size, _dptr(dk),
                                               self.nblocks, ctypes.byref(info)))
        return J.value, dq, dk[:self.nblocks], {k: getattr(info, k) for k, _ in AdjointInfo._fields_}
