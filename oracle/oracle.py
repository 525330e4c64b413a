"""ctypes harness over oracle/liboracle.so, the plain-C FP64 restatement of
hsolver's SIMPLE conjugate-heat-transfer outer step (hs_oracle.c).

Test infrastructure: the parity checker and the CPU baseline, never the product.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")

FIELDS = {"u_star": 0, "v_star": 1, "w_star": 2, "p_temp": 3, "t_temp": 4, "up": 5, "vp": 6, "wp": 7,
          "ux": 8, "uy": 9, "uz": 10, "p": 11, "t": 12, "p_prime": 13}


class Params(ctypes.Structure):
    """Mirror of or_params (reference macros, fluid_solver.h:21-37, mobs_solver.h:15-29)."""
    _fields_ = [("nu", ctypes.c_double), ("rho", ctypes.c_double), ("alpha", ctypes.c_double),
                ("u_lid", ctypes.c_double), ("relax", ctypes.c_double), ("relax_solid", ctypes.c_double),
                ("mom_tol", ctypes.c_double), ("energy_tol", ctypes.c_double), ("solid_tol", ctypes.c_double),
                ("gs_max", ctypes.c_int), ("t_fluid0", ctypes.c_double), ("t_wall", ctypes.c_double),
                ("t_solid0", ctypes.c_double), ("pcg_tol", ctypes.c_double), ("pcg_maxiter", ctypes.c_int),
                ("frozen_matrix", ctypes.c_int)]


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = ctypes.CDLL(_LIB)
        vp, i64, i64p = ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)
        dp = ctypes.POINTER(ctypes.c_double)
        L.or_create.restype = vp
        L.or_create.argtypes = [ctypes.c_char_p, ctypes.POINTER(Params)]
        L.or_params_default.argtypes = [ctypes.POINTER(Params)]
        L.or_last_error.restype = ctypes.c_char_p
        L.or_init.argtypes = [vp]
        L.or_step.argtypes = [vp, ctypes.c_int]
        L.or_destroy.argtypes = [vp]
        L.or_fluid_meta.argtypes = [vp, i64p]
        L.or_solid_meta.argtypes = [vp, ctypes.c_int, i64p]
        L.or_num_solids.argtypes = [vp]
        L.or_grid_dims.argtypes = [vp, i64p]
        L.or_field_size.restype = i64
        L.or_field_size.argtypes = [vp, ctypes.c_int]
        L.or_get_field.argtypes = [vp, ctypes.c_int, dp, i64]
        L.or_set_field.argtypes = [vp, ctypes.c_int, dp, i64]
        L.or_solid_size.restype = i64
        L.or_solid_size.argtypes = [vp, ctypes.c_int]
        L.or_get_solid.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, i64]
        L.or_get_fluid_mask.argtypes = [vp, ctypes.POINTER(ctypes.c_uint8), i64]
        L.or_get_cell_types.argtypes = [vp, ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_int), i64]
        L.or_get_grid.argtypes = [vp, ctypes.c_int, dp, i64]
        L.or_num_swap.restype = i64
        L.or_num_swap.argtypes = [vp]
        L.or_get_swap.argtypes = [vp, i64p, i64]
        L.or_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_int), dp]
        L.or_solid_sweeps.argtypes = [vp, ctypes.c_int]
        L.or_get_row_ids.argtypes = [vp, ctypes.POINTER(ctypes.c_int), i64]
        _lib = L
    return _lib


def default_params():
    p = Params()
    lib().or_params_default(ctypes.byref(p))
    return p


class OracleCase:
    """One case: fluid region 0 plus every solid region of a `.in` deck."""

    def __init__(self, deck_text, params=None):
        L = lib()
        self._p = params if params is not None else default_params()
        h = L.or_create(deck_text.encode() if isinstance(deck_text, str) else deck_text, ctypes.byref(self._p))
        if not h:
            raise ValueError(L.or_last_error().decode())
        self.h = h
        m = (ctypes.c_int64 * 9)()
        L.or_fluid_meta(h, m)
        self.meta = tuple(m)
        d = (ctypes.c_int64 * 3)()
        L.or_grid_dims(h, d)
        self.dims = tuple(d)
        self.nsolid = L.or_num_solids(h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_destroy(self.h)
            self.h = None

    def init(self):
        lib().or_init(self.h)

    def step(self, n=1):
        lib().or_step(self.h, n)

    def field(self, name):
        L = lib()
        f = FIELDS[name]
        n = L.or_field_size(self.h, f)
        out = np.empty(n, np.float64)
        assert L.or_get_field(self.h, f, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n) == 0
        return out

    def set_field(self, name, arr):
        L = lib()
        arr = np.ascontiguousarray(arr, np.float64)
        assert L.or_set_field(self.h, FIELDS[name], arr.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), arr.size) == 0

    def solid_meta(self, r):
        m = (ctypes.c_int64 * 9)()
        lib().or_solid_meta(self.h, r, m)
        return tuple(m)

    def solid(self, r, which="t_temp"):
        L = lib()
        md = self.solid_meta(r)
        n = L.or_solid_size(self.h, r) if which == "t_temp" else md[0] * md[1] * md[2]
        out = np.empty(n, np.float64)
        assert L.or_get_solid(self.h, r, 0 if which == "t_temp" else 1,
                              out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n) == 0
        return out

    def fluid_empty(self):
        cx, cy, cz = self.meta[:3]
        out = np.empty(cx * cy * cz, np.uint8)
        assert lib().or_get_fluid_mask(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), out.size) == 0
        return out

    def cell_types(self):
        n = self.dims[0] * self.dims[1] * self.dims[2]
        t = np.empty(n, np.uint8)
        r = np.empty(n, np.int32)
        assert lib().or_get_cell_types(self.h, t.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                                       r.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n) == 0
        return t, r

    def swap_pairs(self):
        n = lib().or_num_swap(self.h)
        out = np.empty(5 * n, np.int64)
        assert lib().or_get_swap(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), n) == 0
        return out.reshape(n, 5)

    def row_ids(self):
        cx, cy, cz = self.meta[:3]
        out = np.empty(cx * cy * cz, np.int32)
        assert lib().or_get_row_ids(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), out.size) == 0
        return out

    def stats(self):
        i = (ctypes.c_int * 5)()
        d = (ctypes.c_double * 5)()
        lib().or_stats(self.h, i, d)
        return {"sweeps_u": i[0], "sweeps_v": i[1], "sweeps_w": i[2], "sweeps_t": i[3], "pcg_iters": i[4],
                "res_u": d[0], "res_v": d[1], "res_w": d[2], "res_t": d[3], "pcg_relres": d[4],
                "sweeps_solid": [lib().or_solid_sweeps(self.h, r) for r in range(self.nsolid)]}


def read_dump(path):
    """Parse a record file written by oracle/ref/ref_driver (or tests/golden)."""
    out = {}
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    while pos < len(data):
        name = data[pos:pos + 32].split(b"\0", 1)[0].decode()
        kind = int.from_bytes(data[pos + 32:pos + 36], "little", signed=True)
        n = int.from_bytes(data[pos + 36:pos + 44], "little", signed=True)
        pos += 44
        dt = np.float64 if kind == 0 else np.int32
        nb = n * (8 if kind == 0 else 4)
        arr = np.frombuffer(data[pos:pos + nb], dt).copy()
        pos += nb
        key = name
        k = 1
        while key in out:
            key = "%s#%d" % (name, k)
            k += 1
        out[key] = arr
    return out


def pcg_solve(nx, ny, nz, acx, acy, acz, b, tol=1e-5, maxiter=1000):
    """or_pcg_solve: the oracle's HYPRE-rule CG on padded arrays; returns
    (x, iterations, final relative residual)."""
    L = lib()
    dp = ctypes.POINTER(ctypes.c_double)
    L.or_pcg_solve.restype = ctypes.c_int
    L.or_pcg_solve.argtypes = [ctypes.c_int64] * 3 + [dp] * 5 + [ctypes.c_double, ctypes.c_int, dp]
    arrs = [np.ascontiguousarray(a, np.float64) for a in (acx, acy, acz, b)]
    x = np.zeros_like(arrs[3])
    rr = ctypes.c_double()
    it = L.or_pcg_solve(nx, ny, nz, *[a.ctypes.data_as(dp) for a in arrs], x.ctypes.data_as(dp), tol, maxiter,
                        ctypes.byref(rr))
    return x, it, rr.value


class _Cht(ctypes.Structure):
    _fields_ = [("Nx", ctypes.c_int64), ("Ny", ctypes.c_int64), ("Nz", ctypes.c_int64),
                ("xs", ctypes.c_void_p), ("ys", ctypes.c_void_p), ("zs", ctypes.c_void_p),
                ("solid", ctypes.c_void_p), ("region", ctypes.c_void_p), ("kcell", ctypes.c_void_p),
                ("qcell", ctypes.c_void_p), ("ug", ctypes.c_void_p), ("vg", ctypes.c_void_p), ("wg", ctypes.c_void_p),
                ("Tb", ctypes.c_double), ("bc", ctypes.c_int)]


def cht_solve(xs, ys, zs, ctype, region, kcell, qcell, ug, vg, wg, Tb=293.0, tol=1e-13, maxiter=20000, nreg=0, bc=0):
    """Oracle forward + adjoint of the monolithic conjugate-heat-transfer
    energy equation (hs_oracle.c: or_cht_forward / or_cht_adjoint).
    Returns dict(T, J, dJdq, dJdk, iters)."""
    L = lib()
    keep = [np.ascontiguousarray(a, dt) for a, dt in [(xs, np.float64), (ys, np.float64), (zs, np.float64),
                                                      (ctype, np.uint8), (region, np.int32), (kcell, np.float64),
                                                      (qcell, np.float64), (ug, np.float64), (vg, np.float64),
                                                      (wg, np.float64)]]
    Nx, Ny, Nz = len(xs) - 1, len(ys) - 1, len(zs) - 1
    H = _Cht(Nx, Ny, Nz, *[a.ctypes.data for a in keep], Tb, bc)
    dp = ctypes.POINTER(ctypes.c_double)
    L.or_cht_forward.restype = ctypes.c_int
    L.or_cht_forward.argtypes = [ctypes.POINTER(_Cht), dp, ctypes.c_double, ctypes.c_int, dp, dp]
    L.or_cht_adjoint.restype = ctypes.c_int
    L.or_cht_adjoint.argtypes = [ctypes.POINTER(_Cht), dp, dp, dp, dp, ctypes.c_int, ctypes.c_double, ctypes.c_int, dp]
    N = Nx * Ny * Nz
    T = np.empty(N)
    J = ctypes.c_double()
    rr = ctypes.c_double()
    it1 = L.or_cht_forward(ctypes.byref(H), T.ctypes.data_as(dp), tol, maxiter, ctypes.byref(J), ctypes.byref(rr))
    lam = np.empty(N)
    dJdq = np.empty(N)
    dJdk = np.zeros(max(nreg, 1))
    it2 = L.or_cht_adjoint(ctypes.byref(H), T.ctypes.data_as(dp), lam.ctypes.data_as(dp), dJdq.ctypes.data_as(dp),
                           dJdk.ctypes.data_as(dp), nreg, tol, maxiter, ctypes.byref(rr))
    return {"T": T, "J": J.value, "dJdq": dJdq, "dJdk": dJdk[:nreg], "iters": (it1, it2)}


class ChParams(ctypes.Structure):
    """or_ch_params (hs_oracle.c): the channel conjugate-heat-transfer case."""
    _fields_ = [("re", ctypes.c_double), ("pr", ctypes.c_double), ("u_in", ctypes.c_double), ("t_in", ctypes.c_double),
                ("alpha_u", ctypes.c_double), ("alpha_p", ctypes.c_double), ("alpha_t", ctypes.c_double),
                ("mom_sweeps", ctypes.c_int), ("p_tol", ctypes.c_double), ("p_maxiter", ctypes.c_int),
                ("t_tol", ctypes.c_double), ("t_maxiter", ctypes.c_int),
                ("conv", ctypes.c_int), ("g_axis", ctypes.c_int), ("ri", ctypes.c_double)]

    @classmethod
    def default(cls, **kw):
        P = cls()
        lib().or_ch_params_default(ctypes.byref(P))
        for k, v in kw.items():
            setattr(P, k, v)
        return P


CH_FIELDS = {"u": 0, "v": 1, "w": 2, "p": 3, "T": 4, "u_star": 5, "v_star": 6, "w_star": 7, "d_u": 8, "d_v": 9,
             "d_w": 10, "p_prime": 11}


class ChannelCase:
    """Oracle of the channel conjugate-heat-transfer SIMPLE iteration
    (hs_oracle.c: or_ch_*): inlet plug flow, zero-gradient outlet, solid
    blocks with a heat source and a conductivity ratio."""

    def __init__(self, deck, **params):
        L = lib()
        L.or_ch_create.restype = ctypes.c_void_p
        L.or_ch_create.argtypes = [ctypes.c_char_p, ctypes.POINTER(ChParams)]
        L.or_ch_nreg.argtypes = [ctypes.c_void_p]
        L.or_ch_set_solid.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.or_ch_init.argtypes = [ctypes.c_void_p]
        L.or_ch_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.or_ch_get.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64]
        L.or_ch_set.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64]
        L.or_ch_stats.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.or_ch_destroy.argtypes = [ctypes.c_void_p]
        self.L = L
        self.params = ChParams.default(**params)
        self.h = L.or_ch_create(deck.encode(), ctypes.byref(self.params))
        if not self.h:
            raise ValueError("deck rejected")
        d = np.zeros(3, np.int64)
        L.or_ch_dims.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.or_ch_dims(self.h, d.ctypes.data)
        self.dims = tuple(int(v) for v in d)
        self.nreg = L.or_ch_nreg(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.or_ch_destroy(self.h)
            self.h = None

    def size(self, name):
        Nx, Ny, Nz = self.dims
        f = CH_FIELDS[name]
        if f in (3, 4, 11):
            return Nx * Ny * Nz
        a = f % 3 if f < 3 else (f - 5) % 3
        return (Nx + (a == 0)) * (Ny + (a == 1)) * (Nz + (a == 2))

    def set_solid(self, k_region, q_cell):
        k = np.ascontiguousarray(k_region, np.float64)
        q = np.ascontiguousarray(q_cell, np.float64)
        assert k.size == self.nreg and q.size == self.dims[0] * self.dims[1] * self.dims[2]
        self.L.or_ch_set_solid(self.h, k.ctypes.data, q.ctypes.data)

    def init(self):
        self.L.or_ch_init(self.h)

    def step(self, n=1, pressure=True, energy=True):
        self.L.or_ch_step(self.h, n, int(pressure), int(energy))

    def field(self, name):
        out = np.empty(self.size(name))
        assert self.L.or_ch_get(self.h, CH_FIELDS[name], out.ctypes.data, out.size) == 0
        return out

    def set_field(self, name, arr):
        a = np.ascontiguousarray(arr, np.float64)
        assert self.L.or_ch_set(self.h, CH_FIELDS[name], a.ctypes.data, a.size) == 0

    def stats(self):
        res, norm, glob, it = np.zeros(5), np.zeros(5), ctypes.c_double(), np.zeros(3, np.int32)
        self.L.or_ch_stats(self.h, res.ctypes.data, norm.ctypes.data, ctypes.byref(glob), it.ctypes.data)
        return {"res": res, "norm": norm, "global": glob.value, "iter": int(it[0]), "pcg_iters": int(it[1]),
                "t_iters": int(it[2])}


def set_threads(n):
    """The thread count of the oracle's OpenMP loops (the tests run one: every
    sum in loop order); returns the previous count."""
    L = lib()
    L.or_threads.restype = ctypes.c_int
    L.or_set_threads.argtypes = [ctypes.c_int]
    prev = int(L.or_threads())
    L.or_set_threads(int(n))
    return prev


def _channel_extra(L):
    L.or_ch_step_given.restype = ctypes.c_double
    L.or_ch_step_given.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.or_ch_energy_residual.restype = ctypes.c_double
    L.or_ch_energy_residual.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]


def channel_step_given(case, pprime):
    """One outer step of a ChannelCase with p' given instead of solved (no
    energy): returns ||b - A p'|| / ||b|| on the step's own p' system."""
    _channel_extra(case.L)
    a = np.ascontiguousarray(pprime, np.float64)
    return case.L.or_ch_step_given(case.h, a.ctypes.data)


def channel_energy_residual(case, T):
    """(||b - A T||, ||b||) of a ChannelCase's energy system on its current
    face velocities."""
    _channel_extra(case.L)
    a = np.ascontiguousarray(T, np.float64)
    bn = ctypes.c_double()
    r = case.L.or_ch_energy_residual(case.h, a.ctypes.data, ctypes.byref(bn))
    return r, bn.value


def quick_weights(pts, kind, e):
    """The QUICK weights (far upwind, upwind, downwind) of control-volume face
    e along an axis with grid points `pts` (hs_oracle.c: ch_quick_w): six
    values, for a flux in the + direction then against it; node kind 1 = the
    faces of that axis, 0 = cell centres."""
    L = lib()
    L.or_ch_quick_weights.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int64, ctypes.c_void_p]
    p = np.ascontiguousarray(pts, np.float64)
    w = np.zeros(6)
    L.or_ch_quick_weights(p.ctypes.data, p.size - 1, int(kind), int(e), w.ctypes.data)
    return w


def neighbour_coefficient(conv, D, F, hi):
    """a_nb of the momentum convection scheme `conv` for a control-volume face
    of conductance D and flux F (+ direction), neighbour on the high side when
    hi (hs_oracle.c: ch_anb)."""
    L = lib()
    L.or_ch_anb.restype = ctypes.c_double
    L.or_ch_anb.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int]
    return L.or_ch_anb(int(conv), float(D), float(F), int(hi))
