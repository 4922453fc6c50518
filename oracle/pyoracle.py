"""ctypes binding of oracle/liboracle.so (test infrastructure only).

The oracle restates app/rk2_serial_driver.F90 and src/serial/*.F90 of the
reference in C; this module exposes it to numpy for the parity tests.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}

INIT_REF, INIT_CFG = 0, 1

# field ids (same numbering as mom6b.h / mom6_oracle.h)
FIELDS = ["u", "v", "h", "h0", "uh", "vh", "up", "vp", "eta", "ubt", "vbt",
          "ubt_av", "vbt_av", "eta_av", "hu_bt", "FA_u_W0", "FA_u_WW",
          "FA_u_E0", "FA_u_EE", "uBT_WW", "uBT_EE", "du_cor", "taux_bot",
          "tauy_bot", "taux", "tauy", "Ray_u", "Ray_v", "CAu", "CAv",
          "diffu", "diffv", "hv_bt", "FA_v_S0", "FA_v_SS", "FA_v_N0", "FA_v_NN",
          "vBT_SS", "vBT_NN", "dv_cor", "visc_rem_u", "visc_rem_v"]
FID = {n: i for i, n in enumerate(FIELDS)}
FIELDS_3D = {"u", "v", "h", "h0", "uh", "vh", "up", "vp", "hu_bt", "Ray_u",
             "Ray_v", "CAu", "CAv", "diffu", "diffv", "hv_bt", "visc_rem_u", "visc_rem_v"}


class HorViscOpts(ctypes.Structure):
    """hor_visc_init's scheme options (mom6_hor_visc_serial.F90:160-193)."""
    _fields_ = [("laplacian", ctypes.c_int), ("biharmonic", ctypes.c_int),
                ("smagorinsky", ctypes.c_int), ("leith", ctypes.c_int),
                ("no_slip", ctypes.c_int), ("better_bound", ctypes.c_int),
                ("modified_leith", ctypes.c_int), ("Ah", ctypes.c_double)]


def hor_visc_opts(laplacian=True, biharmonic=False, smagorinsky=False, leith=False,
                  no_slip=False, better_bound=False, modified_leith=False, Ah=1.0e10):
    return HorViscOpts(int(bool(laplacian)), int(bool(biharmonic)), int(bool(smagorinsky)),
                       int(bool(leith)), int(bool(no_slip)), int(bool(better_bound)),
                       int(bool(modified_leith)), float(Ah))


class Config(ctypes.Structure):
    _fields_ = [("ni", ctypes.c_int), ("nj", ctypes.c_int), ("nk", ctypes.c_int),
                ("bt_nsteps", ctypes.c_int), ("init_mode", ctypes.c_int),
                ("seed", ctypes.c_uint64), ("dt", ctypes.c_double),
                ("dx_km", ctypes.c_double), ("lat_deg", ctypes.c_double),
                ("Kh", ctypes.c_double), ("Kv", ctypes.c_double),
                ("Kv_ml", ctypes.c_double), ("Kv_extra_bbl", ctypes.c_double),
                ("Hmix", ctypes.c_double), ("Hbbl", ctypes.c_double),
                ("bc_fill", ctypes.c_int),
                ("ni_global", ctypes.c_int), ("nj_global", ctypes.c_int),
                ("i_offset", ctypes.c_int), ("j_offset", ctypes.c_int), ("cuts", ctypes.c_int)]

CUT_W, CUT_E, CUT_S, CUT_N = 1, 2, 4, 8
# void (*)(void *ctx, double *field, int nz, int kind)
ExchangeFn = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                              ctypes.c_int, ctypes.c_int)


def build():
    """Compile liboracle.so with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib(parallel=False):
    """The single-threaded oracle, or (parallel=True) the same source built with
    its row-parallel loops on OpenMP threads; the two give identical results."""
    if parallel not in _LIBS:
        path = os.path.join(_HERE, "liboracle_omp.so" if parallel else "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        P = ctypes.POINTER
        d = ctypes.c_double
        vp = ctypes.c_void_p
        L.oracle_config_default.argtypes = [P(Config), ctypes.c_int]
        L.oracle_create.argtypes = [P(Config)]
        L.oracle_create.restype = vp
        L.oracle_destroy.argtypes = [vp]
        L.oracle_step.argtypes = [vp, ctypes.c_int]
        L.oracle_field_size.argtypes = [vp, ctypes.c_int]
        L.oracle_field_size.restype = ctypes.c_size_t
        L.oracle_get.argtypes = [vp, ctypes.c_int, P(d)]
        L.oracle_set.argtypes = [vp, ctypes.c_int, P(d)]
        L.oracle_dims.argtypes = [vp, P(ctypes.c_int)]
        L.oracle_verify.argtypes = [vp, P(d)]
        for name in ("oracle_compute_transports",):
            getattr(L, name).argtypes = [vp] + [P(d)] * 5
        L.oracle_hor_visc.argtypes = [vp] + [P(d)] * 5
        L.oracle_coriolis.argtypes = [vp] + [P(d)] * 7
        L.oracle_vert_visc.argtypes = [vp, P(d), P(d), P(d), d]
        L.oracle_btstep.argtypes = [vp] + [P(d)] * 6
        L.oracle_continuity.argtypes = [vp, P(d), P(d), P(d), P(d), d]
        L.oracle_continuity_merid.argtypes = [vp, P(d), P(d), P(d), P(d), d]
        L.oracle_set_merid.argtypes = [vp, ctypes.c_int]
        L.oracle_set_coriolis_scheme.argtypes = [vp, ctypes.c_int]
        L.oracle_set_remnant.argtypes = [vp, ctypes.c_int]
        L.oracle_vert_visc_remnant.argtypes = [vp, d]
        L.oracle_set_coriolis_scheme.restype = ctypes.c_int
        L.oracle_set_hor_visc.argtypes = [vp, ctypes.POINTER(HorViscOpts)]
        L.oracle_set_hor_visc.restype = ctypes.c_int
        L.oracle_halo_fill.argtypes = [vp, P(d), ctypes.c_int, ctypes.c_int]
        L.oracle_normal.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64]
        L.oracle_normal.restype = d
        L.oracle_set_bt_extended.argtypes = [vp, ctypes.c_int]
        L.oracle_set_bt_first_direction.argtypes = [vp, ctypes.c_int]
        L.oracle_set_exchange.argtypes = [vp, ExchangeFn, vp]
        L.oracle_array.argtypes = [vp, ctypes.c_char_p, P(d), ctypes.c_size_t]
        L.oracle_array.restype = ctypes.c_int
        L.oracle_set_threads.argtypes = [ctypes.c_int]
        L.oracle_set_threads.restype = ctypes.c_int
        L.oracle_diag_enable.argtypes = [vp, ctypes.c_int]
        L.oracle_diag_get.argtypes = [vp, ctypes.c_int, P(d)]
        L.oracle_diag_get.restype = ctypes.c_int
        _LIBS[parallel] = L
    return _LIBS[parallel]


def _ptr(a):
    assert a.dtype == np.float64 and a.flags["F_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Oracle:
    """One oracle model (grid + state + persistent module work arrays)."""

    def __init__(self, ni, nj, nk, bt_nsteps, init_mode=INIT_CFG, seed=0,
                 dt=None, Kh=None, bc_fill=None, threads=None, dx_km=None,
                 subdomain=None):
        """threads: None for the single-threaded build, else the OpenMP build
        on that many threads (0: all the runtime offers).  subdomain: (ni_global,
        nj_global, i_offset, j_offset, cuts) for one subdomain of a decomposed
        run, ni and nj then being the local sizes (compute width + 4)."""
        L = lib(parallel=threads is not None)
        self._L = L
        self.threads = 1 if threads is None else L.oracle_set_threads(int(threads))
        c = Config()
        L.oracle_config_default(ctypes.byref(c), init_mode)
        c.ni, c.nj, c.nk, c.bt_nsteps, c.seed = ni, nj, nk, bt_nsteps, seed
        if dt is not None:
            c.dt = dt
        if Kh is not None:
            c.Kh = Kh
        if bc_fill is not None:
            c.bc_fill = int(bc_fill)
        if dx_km is not None:
            c.dx_km = dx_km
        if subdomain is not None:
            c.ni_global, c.nj_global, c.i_offset, c.j_offset, c.cuts = map(int, subdomain)
        self.cfg = c
        self._xfn = None
        self._m = L.oracle_create(ctypes.byref(c))
        if not self._m:
            raise ValueError("oracle_create rejected the configuration")
        dims = (ctypes.c_int * 8)()
        L.oracle_dims(self._m, dims)
        self.n1, self.n2, self.nk, self.is_, self.ie, self.js, self.je, _ = list(dims)

    def close(self):
        if self._m:
            self._L.oracle_destroy(self._m)
            self._m = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def shape(self, name):
        return (self.n1, self.n2, self.nk) if name in FIELDS_3D else (self.n1, self.n2)

    def empty(self, name):
        return np.zeros(self.shape(name), dtype=np.float64, order="F")

    def get(self, name):
        a = self.empty(name)
        if self._L.oracle_get(self._m, FID[name], _ptr(a)) != 0:
            raise KeyError(name)
        return a

    def set(self, name, a):
        a = np.asfortranarray(a, dtype=np.float64)
        assert a.shape == self.shape(name)
        if self._L.oracle_set(self._m, FID[name], _ptr(a)) != 0:
            raise KeyError(name)

    def step(self, n=1):
        self._L.oracle_step(self._m, int(n))

    DIAG_FIELDS = {"diffu_sum": 0, "diffv_sum": 1, "KE": 2, "mass": 3}

    def diag_enable(self, on=True):
        """Record the driver's diagnostics (rk2_serial_driver.F90 with
        diag_mode = 1) from the next step on."""
        self._L.oracle_diag_enable(self._m, int(bool(on)))

    def diag_get(self, name):
        """The field the last post of diagnostic `name` carried (full array;
        the posts use its computational domain)."""
        a = self.empty("h" if name == "KE" else "eta")
        if self._L.oracle_diag_get(self._m, self.DIAG_FIELDS[name], _ptr(a)) != 0:
            raise RuntimeError("diagnostics are not enabled")
        return a

    def verify(self):
        out = (ctypes.c_double * 7)()
        self._L.oracle_verify(self._m, out)
        keys = ["mass_init", "mass_final", "rel_error", "max_u", "max_v",
                "max_eta", "ke_total"]
        return dict(zip(keys, list(out)))

    # single phases -------------------------------------------------------
    def continuity(self, u, hin, dt):
        h = self.get("h")
        uh = self.get("uh")
        self._L.oracle_continuity(self._m, _ptr(u), _ptr(hin), _ptr(h), _ptr(uh), dt)
        return h, uh

    def continuity_merid(self, v, hin, dt):
        """The meridional pass alone: (h, vh) from v and hin (h starts as
        the model's h; only the computational domain is written)."""
        h = self.get("h")
        vh = self.empty("vh")
        self._L.oracle_continuity_merid(self._m, _ptr(v), _ptr(hin), _ptr(h), _ptr(vh), dt)
        return h, vh

    def set_coriolis_scheme(self, scheme):
        """1 SADOURNY75_ENERGY, 2 ARAKAWA_HSU90, 3 ARAKAWA_LAMB81."""
        if self._L.oracle_set_coriolis_scheme(self._m, int(scheme)) != 0:
            raise ValueError(scheme)

    def set_hor_visc(self, **opts):
        """hor_visc_init's options: laplacian, biharmonic, smagorinsky, leith,
        no_slip, better_bound, modified_leith (bools) and Ah."""
        o = hor_visc_opts(**opts)
        if self._L.oracle_set_hor_visc(self._m, ctypes.byref(o)) != 0:
            raise ValueError(opts)

    def set_remnant(self, on=True):
        """Feed the vertical-viscosity remnant to continuity from now on."""
        self._L.oracle_set_remnant(self._m, int(bool(on)))

    def vert_visc_remnant(self, dt):
        """vert_visc_remnant after the last vert_visc; (visc_rem_u, visc_rem_v)."""
        self._L.oracle_vert_visc_remnant(self._m, float(dt))
        return self.get("visc_rem_u"), self.get("visc_rem_v")

    def set_merid(self, on=True):
        """Zonal then meridional continuity in every step from now on."""
        self._L.oracle_set_merid(self._m, int(bool(on)))

    def vert_visc(self, u, v, h, dt):
        u = u.copy(order="F")
        v = v.copy(order="F")
        self._L.oracle_vert_visc(self._m, _ptr(u), _ptr(v), _ptr(h), dt)
        return u, v

    def btstep(self, eta, ubt, vbt):
        ua, va, ea = self.empty("ubt"), self.empty("vbt"), self.empty("eta")
        self._L.oracle_btstep(self._m, _ptr(eta), _ptr(ubt), _ptr(vbt), _ptr(ua),
                            _ptr(va), _ptr(ea))
        return ua, va, ea

    def hor_visc(self, u, v, h):
        du, dv = self.empty("u"), self.empty("v")
        self._L.oracle_hor_visc(self._m, _ptr(u), _ptr(v), _ptr(h), _ptr(du), _ptr(dv))
        return du, dv

    def coriolis(self, u, v, h, uh, vh):
        cu, cv = self.empty("u"), self.empty("v")
        self._L.oracle_coriolis(self._m, _ptr(u), _ptr(v), _ptr(h), _ptr(uh),
                              _ptr(vh), _ptr(cu), _ptr(cv))
        return cu, cv

    def transports(self, u, v, h):
        uh, vh = self.empty("u"), self.empty("v")
        self._L.oracle_compute_transports(self._m, _ptr(u), _ptr(v), _ptr(h),
                                        _ptr(uh), _ptr(vh))
        return uh, vh

    def array(self, name):
        """A named grid / control-structure array, (n1, n2) or (4, n1, n2)."""
        n1, n2 = self.shape("eta")
        four = name in ("f_4_u", "f_4_v")
        out = np.zeros((4, n1, n2) if four else (n1, n2), order="F")
        rc = self._L.oracle_array(self._m, name.encode(), _ptr(out), out.size)
        if rc != 0:
            raise KeyError(name)
        return out

    def set_bt_extended(self, on):
        self._L.oracle_set_bt_extended(self._m, 1 if on else 0)

    def set_bt_first_direction(self, d):
        self._L.oracle_set_bt_first_direction(self._m, int(d))

    def set_exchange(self, fn):
        """fn(a, kind) refreshes the halo of a, a Fortran-ordered (n1, n2, nz)
        view of the model's field, in place; None removes the exchange."""
        if fn is None:
            self._xfn = None
            self._L.oracle_set_exchange(self._m, ExchangeFn(), None)
            return
        n1, n2 = self.n1, self.n2

        def cb(_ctx, ptr, nz, kind):
            a = np.ctypeslib.as_array(ptr, shape=(n1 * n2 * nz,)).reshape((n1, n2, nz),
                                                                           order="F")
            fn(a, kind)

        self._xfn = ExchangeFn(cb)
        self._L.oracle_set_exchange(self._m, self._xfn, None)

    def halo_fill(self, f, kind):
        f = np.asfortranarray(f.copy())
        nz = f.shape[2] if f.ndim == 3 else 1
        self._L.oracle_halo_fill(self._m, _ptr(f), nz, kind)
        return f
