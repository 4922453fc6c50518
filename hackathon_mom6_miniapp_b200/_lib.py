"""ctypes binding of libmom6b.so (the product library)."""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

INIT_REF, INIT_CFG = 0, 1
FP64, MIXED = 0, 1

FIELDS = ["u", "v", "h", "h0", "uh", "vh", "up", "vp", "eta", "ubt", "vbt",
          "ubt_av", "vbt_av", "eta_av", "hu_bt", "FA_u_W0", "FA_u_WW",
          "FA_u_E0", "FA_u_EE", "uBT_WW", "uBT_EE", "du_cor", "taux_bot",
          "tauy_bot", "taux", "tauy", "Ray_u", "Ray_v",
          # ids 28..31: the oracle's Coriolis and viscosity fields (no model buffer)
          "CAu", "CAv", "diffu", "diffv",
          # the meridional continuity's outputs (Model.set_continuity_merid)
          "hv_bt", "FA_v_S0", "FA_v_SS", "FA_v_N0", "FA_v_NN", "vBT_SS", "vBT_NN", "dv_cor",
          # the vertical-viscosity remnant (Model.set_visc_remnant)
          "visc_rem_u", "visc_rem_v"]
FID = {n: i for i, n in enumerate(FIELDS)}
FIELDS_3D = {"u", "v", "h", "h0", "uh", "vh", "up", "vp", "hu_bt", "Ray_u", "Ray_v", "CAu",
             "CAv", "diffu", "diffv", "hv_bt", "visc_rem_u", "visc_rem_v"}

STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of memory",
          4: "grid barrier timeout", 5: "invalid state"}


class HorVisc(ctypes.Structure):
    """mom6b_hor_visc: hor_visc_init's scheme options."""
    _fields_ = [("laplacian", ctypes.c_int), ("biharmonic", ctypes.c_int),
                ("smagorinsky", ctypes.c_int), ("leith", ctypes.c_int),
                ("no_slip", ctypes.c_int), ("better_bound", ctypes.c_int),
                ("modified_leith", ctypes.c_int), ("Ah", ctypes.c_double)]


class Mom6bError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"mom6b error {code} ({STATUS.get(code, '?')}): {msg}")
        self.code = code


class MixedNotBuilt(Mom6bError):
    pass


class Config(ctypes.Structure):
    _fields_ = [("ni", ctypes.c_int), ("nj", ctypes.c_int), ("nk", ctypes.c_int),
                ("bt_nsteps", ctypes.c_int), ("init_mode", ctypes.c_int),
                ("seed", ctypes.c_uint64), ("dt", ctypes.c_double),
                ("dx_km", ctypes.c_double), ("lat_deg", ctypes.c_double),
                ("Kh", ctypes.c_double), ("Kv", ctypes.c_double),
                ("Kv_ml", ctypes.c_double), ("Kv_extra_bbl", ctypes.c_double),
                ("Hmix", ctypes.c_double), ("Hbbl", ctypes.c_double),
                ("bc_fill", ctypes.c_int), ("precision", ctypes.c_int),
                ("device", ctypes.c_int), ("use_graph", ctypes.c_int),
                ("exact", ctypes.c_int), ("bt_untiled", ctypes.c_int),
                ("general_metrics", ctypes.c_int), ("wait_cycles", ctypes.c_longlong),
                ("mixed_f32_vertvisc", ctypes.c_int),
                ("ni_global", ctypes.c_int), ("nj_global", ctypes.c_int),
                ("i_offset", ctypes.c_int), ("j_offset", ctypes.c_int), ("cuts", ctypes.c_int)]

CUT_W, CUT_E, CUT_S, CUT_N = 1, 2, 4, 8
# int (*)(void *ctx, double *field, int nz, int kind, int more, void *stream)
_ExchangeFn = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                               ctypes.c_int, ctypes.c_int, ctypes.c_void_p)


def library_path():
    return os.path.join(_HERE, "libmom6b.so")


def library():
    """Load libmom6b.so; raises OSError when it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not os.path.exists(path):
        raise OSError(f"{path} is missing: run __graft_entry__.build() first")
    L = ctypes.CDLL(path)
    P, d, vp, i64 = ctypes.POINTER, ctypes.c_double, ctypes.c_void_p, ctypes.c_int64
    L.mom6b_config_default.argtypes = [P(Config), ctypes.c_int]
    L.mom6b_create.argtypes = [P(Config), P(vp)]
    L.mom6b_destroy.argtypes = [vp]
    L.mom6b_step.argtypes = [vp, ctypes.c_int]
    L.mom6b_synchronize.argtypes = [vp]
    L.mom6b_field_size.argtypes = [vp, ctypes.c_int]
    L.mom6b_field_size.restype = ctypes.c_size_t
    L.mom6b_get_field.argtypes = [vp, ctypes.c_int, P(d), ctypes.c_size_t]
    L.mom6b_set_field.argtypes = [vp, ctypes.c_int, P(d), ctypes.c_size_t]
    L.mom6b_field_device_ptr.argtypes = [vp, ctypes.c_int, P(vp)]
    L.mom6b_dims.argtypes = [vp, P(ctypes.c_int)]
    L.mom6b_stream.argtypes = [vp, P(vp)]
    L.mom6b_step_host.argtypes = [vp, ctypes.c_int, P(d), P(d), P(d), P(d)]
    L.mom6b_step_host_io.argtypes = [vp, ctypes.c_int] + [P(d)] * 7
    L.mom6b_verify.argtypes = [vp, P(d)]
    L.mom6b_launch_count.argtypes = [vp]
    L.mom6b_launch_count.restype = i64
    L.mom6b_reset_launch_count.argtypes = [vp]
    L.mom6b_reset_launch_count.restype = None
    L.mom6b_kernel_timing.argtypes = [vp, ctypes.c_int]
    L.mom6b_kernel_time_ms.argtypes = [vp, ctypes.c_char_p, P(d), P(i64)]
    L.mom6b_cudac_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_double, ctypes.c_char_p, P(vp)]
    L.mom6b_cudac_create_cfg.argtypes = [P(Config), ctypes.c_char_p, P(vp)]
    L.mom6b_cudac_step.argtypes = [vp, ctypes.c_int]
    L.mom6b_cudac_field_size.argtypes = [vp, ctypes.c_int]
    L.mom6b_cudac_field_size.restype = ctypes.c_size_t
    L.mom6b_cudac_get_field.argtypes = [vp, ctypes.c_int, P(d), ctypes.c_size_t]
    L.mom6b_cudac_destroy.argtypes = [vp]
    L.mom6b_ensemble_create.argtypes = [ctypes.c_int, P(Config), P(vp)]
    L.mom6b_ensemble_destroy.argtypes = [vp]
    L.mom6b_ensemble_size.argtypes = [vp]
    L.mom6b_ensemble_step.argtypes = [vp, ctypes.c_int]
    L.mom6b_ensemble_synchronize.argtypes = [vp]
    L.mom6b_ensemble_stream.argtypes = [vp, P(vp)]
    L.mom6b_ensemble_launch_count.argtypes = [vp]
    L.mom6b_ensemble_launch_count.restype = i64
    L.mom6b_ensemble_member.argtypes = [vp, ctypes.c_int]
    L.mom6b_ensemble_member.restype = vp
    L.mom6b_ensemble_get_field.argtypes = [vp, ctypes.c_int, ctypes.c_int, P(d),
                                           ctypes.c_size_t]
    L.mom6b_ensemble_autotune.argtypes = [vp, ctypes.c_int, P(d)]
    L.mom6b_ensemble_get_tuning.argtypes = [vp, P(ctypes.c_int)]
    L.mom6b_ensemble_set_tuning.argtypes = [vp, P(ctypes.c_int)]
    f32p, u64 = P(ctypes.c_float), ctypes.c_uint64
    L.mom6b_surrogate_train.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, d, u64,
                                        P(d)]
    L.mom6b_surrogate_enable.argtypes = [vp, ctypes.c_int, ctypes.c_int, d]
    L.mom6b_surrogate_eval.argtypes = [vp, u64, ctypes.c_int, ctypes.c_int, P(d)]
    L.mom6b_surrogate_status.argtypes = [vp, P(d)]
    L.mom6b_surrogate_param_count.restype = ctypes.c_size_t
    L.mom6b_surrogate_get_params.argtypes = [vp, f32p, ctypes.c_size_t]
    L.mom6b_surrogate_set_params.argtypes = [vp, f32p, ctypes.c_size_t]
    L.mom6b_mlp_param_count.restype = ctypes.c_int
    L.mom6b_mlp_create.argtypes = [ctypes.c_int, u64, P(vp)]
    L.mom6b_mlp_destroy.argtypes = [vp]
    L.mom6b_mlp_get_params.argtypes = [vp, f32p, ctypes.c_size_t]
    L.mom6b_mlp_set_params.argtypes = [vp, f32p, ctypes.c_size_t]
    L.mom6b_mlp_gradients.argtypes = [vp, f32p, f32p, ctypes.c_int, f32p, f32p, f32p]
    L.mom6b_mlp_train.argtypes = [vp, f32p, f32p, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                  f32p]
    L.mom6b_mlp_predict.argtypes = [vp, f32p, ctypes.c_int, f32p]
    cp, ip = ctypes.c_char_p, P(ctypes.c_int)
    L.mom6b_diag_init.argtypes = [vp, cp, ctypes.c_int]
    L.mom6b_diag_end.argtypes = [vp]
    L.mom6b_diag_register.argtypes = [vp, cp, cp, cp, ctypes.c_int, cp, ctypes.c_int, ip]
    L.mom6b_diag_post_2d.argtypes = [vp, ctypes.c_int, vp]
    L.mom6b_diag_post_3d.argtypes = [vp, ctypes.c_int, vp]
    L.mom6b_diag_post_product_sum_u.argtypes = [vp, ctypes.c_int, vp, vp]
    L.mom6b_diag_post_product_sum_v.argtypes = [vp, ctypes.c_int, vp, vp]
    L.mom6b_diag_stats.argtypes = [vp, ctypes.c_int, P(d)]
    L.mom6b_diag_report.argtypes = [vp, ip]
    L.mom6b_diag_driver.argtypes = [vp, ctypes.c_int]
    L.mom6b_write_field_bin.argtypes = [vp, ctypes.c_int, cp]
    L.mom6b_set_continuity_merid.argtypes = [vp, ctypes.c_int]
    L.mom6b_set_visc_remnant.argtypes = [vp, ctypes.c_int]
    L.mom6b_set_hor_visc.argtypes = [vp, ctypes.POINTER(HorVisc)]
    L.mom6b_set_bt_overlap.argtypes = [vp, ctypes.c_int]
    L.mom6b_set_wait_limit.argtypes = [vp, ctypes.c_longlong, ctypes.c_int]
    L.mom6b_set_exchange.argtypes = [vp, vp, vp]
    L.mom6b_halo_group_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                          ctypes.POINTER(vp)]
    L.mom6b_halo_group_join.argtypes = [vp, vp, ctypes.c_int]
    L.mom6b_halo_group_destroy.argtypes = [vp]
    L.mom6b_halo_group_destroy.restype = None
    L.mom6b_abi_set_deferral.argtypes = [ctypes.c_int]
    L.mom6b_btstep_noalloc_status.argtypes = [vp]
    L.mom6b_btstep_noalloc_set_wait.argtypes = [ctypes.c_longlong, ctypes.c_int]
    L.mom6b_continuity_pass.argtypes = [vp, ctypes.c_int, ctypes.c_double]
    L.mom6b_set_coriolis_scheme.argtypes = [vp, ctypes.c_int]
    L.mom6b_read_field_bin.argtypes = [vp, ctypes.c_int, cp]
    L.mom6b_last_error.restype = ctypes.c_char_p
    L.mom6b_version.restype = ctypes.c_char_p
    _LIB = L
    return L


def _check(rc):
    if rc != 0:
        msg = library().mom6b_last_error().decode()
        raise Mom6bError(rc, msg)


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Model:
    """A split RK2 model resident on one GPU (mirrors rk2_serial_driver's
    state: u, v, h, h0, eta, ubt, vbt, ...)."""

    def __init__(self, ni=180, nj=180, nk=75, bt_nsteps=30, init_mode=INIT_CFG,
                 seed=0, dt=None, Kh=None, bc_fill=None, precision=FP64,
                 device=0, use_graph=False, dx_km=None, exact=False, bt_untiled=False,
                 general_metrics=False, wait_cycles=0, mixed_f32_vertvisc=False,
                 subdomain=None):
        """exact=True: the bit-identical FP64 kernels (the serial driver's
        roundings); False: the fast FP64 kernels (within 1e-12 relative L2).
        subdomain: (ni_global, nj_global, i_offset, j_offset, cuts) for one
        subdomain of a decomposed run (ni, nj then its own sizes; see
        HaloGroup)."""
        L = library()
        c = Config()
        _check(L.mom6b_config_default(ctypes.byref(c), init_mode))
        c.ni, c.nj, c.nk, c.bt_nsteps, c.seed = ni, nj, nk, bt_nsteps, seed
        if dt is not None:
            c.dt = dt
        if Kh is not None:
            c.Kh = Kh
        if bc_fill is not None:
            c.bc_fill = int(bc_fill)
        if dx_km is not None:
            c.dx_km = dx_km
        c.precision, c.device, c.use_graph = precision, device, int(use_graph)
        c.exact, c.bt_untiled = int(bool(exact)), int(bool(bt_untiled))
        c.general_metrics, c.wait_cycles = int(bool(general_metrics)), int(wait_cycles)
        c.mixed_f32_vertvisc = int(bool(mixed_f32_vertvisc))
        if subdomain is not None:
            c.ni_global, c.nj_global, c.i_offset, c.j_offset, c.cuts = map(int, subdomain)
        self.cfg = c
        h = ctypes.c_void_p()
        rc = L.mom6b_create(ctypes.byref(c), ctypes.byref(h))
        if rc != 0:
            msg = L.mom6b_last_error().decode()
            if precision == MIXED and "not built" in msg:
                raise MixedNotBuilt(rc, msg)
            raise Mom6bError(rc, msg)
        self._m = h
        dims = (ctypes.c_int * 8)()
        _check(L.mom6b_dims(self._m, dims))
        self.n1, self.n2, self.nk, self.is_, self.ie, self.js, self.je, _ = list(dims)

    def close(self):
        if getattr(self, "_m", None):
            library().mom6b_destroy(self._m)
            self._m = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def shape(self, name):
        return (self.n1, self.n2, self.nk) if name in FIELDS_3D else (self.n1, self.n2)

    def get(self, name):
        a = np.zeros(self.shape(name), dtype=np.float64, order="F")
        _check(library().mom6b_get_field(self._m, FID[name], _dptr(a), a.size))
        return a

    def set(self, name, a):
        a = np.asfortranarray(a, dtype=np.float64)
        if a.shape != self.shape(name):
            raise ValueError(f"{name}: expected shape {self.shape(name)}, got {a.shape}")
        _check(library().mom6b_set_field(self._m, FID[name], _dptr(a), a.size))

    def step(self, n=1):
        _check(library().mom6b_step(self._m, int(n)))

    def synchronize(self):
        _check(library().mom6b_synchronize(self._m))

    def set_exchange(self, fn, batch=False):
        """The halo exchange of a decomposed run, from Python (mom6b_set_exchange):
        fn(t, kind) refreshes in place the halo of t, a torch CUDA tensor viewing
        the model's device field as (nz, n2, n1) (the Fortran array's memory),
        with the model's stream current, so work fn enqueues there is ordered
        with the step; kind 0 h points, 1 u faces, 2 v faces.  batch=True: fn
        receives the list of (t, kind) of one exchange point at once (e.g.
        HaloExchange.exchange_many, one round of messages for all of them).
        With one process per GPU, fn = decomp.HaloExchange(d).exchange over
        torch.distributed (NCCL); within one process, decomp.LocalHaloExchange.
        None removes it."""
        L = library()
        if fn is None:
            self._xfn = None
            _check(L.mom6b_set_exchange(self._m, None, None))
            return
        import torch
        dev = torch.device("cuda", int(self.cfg.device))
        n1, n2 = self.n1, self.n2

        class _View:
            def __init__(self, ptr, nz):
                self.__cuda_array_interface__ = {"shape": (nz, n2, n1), "typestr": "<f8",
                                                 "data": (ptr, False), "version": 2}

        held = []

        def cb(_ctx, ptr, nz, kind, more, stream):
            try:
                t = torch.as_tensor(_View(ptr, nz), device=dev)
                if batch:
                    held.append((t, kind))
                    if more:
                        return 0
                with torch.cuda.stream(torch.cuda.ExternalStream(stream, device=dev)):
                    if batch:
                        fn(list(held))
                    else:
                        fn(t, kind)
                held.clear()
                return 0
            except Exception as e:   # the step reports the failure
                held.clear()
                self.exchange_error = e
                return 1

        self._xfn = _ExchangeFn(cb)
        _check(L.mom6b_set_exchange(self._m, ctypes.cast(self._xfn, ctypes.c_void_p), None))

    def step_host(self, n, u=None, v=None, h=None, eta=None):
        """End-to-end: upload the given host arrays, run n steps, download them."""
        def p(a):
            if a is None:
                return None
            assert a.dtype == np.float64 and a.flags["F_CONTIGUOUS"]
            return _dptr(a)
        _check(library().mom6b_step_host(self._m, int(n), p(u), p(v), p(h), p(eta)))

    def step_host_io(self, n, u_in=None, v_in=None, eta_in=None, u_out=None, v_out=None,
                     h_out=None, eta_out=None):
        """End-to-end with the step's inputs (u, v, eta) and outputs (u, v, h, eta)
        apart (mom6b_step_host_io); an input and an output may be the same array."""
        def p(a):
            if a is None:
                return None
            assert a.dtype == np.float64 and a.flags["F_CONTIGUOUS"]
            return _dptr(a)
        _check(library().mom6b_step_host_io(self._m, int(n), p(u_in), p(v_in), p(eta_in),
                                            p(u_out), p(v_out), p(h_out), p(eta_out)))

    def verify(self):
        out = (ctypes.c_double * 7)()
        _check(library().mom6b_verify(self._m, out))
        keys = ["mass_init", "mass_final", "rel_error", "max_u", "max_v",
                "max_eta", "ke_total"]
        return dict(zip(keys, list(out)))

    def device_ptr(self, name):
        p = ctypes.c_void_p()
        _check(library().mom6b_field_device_ptr(self._m, FID[name], ctypes.byref(p)))
        return p.value

    def stream(self):
        p = ctypes.c_void_p()
        _check(library().mom6b_stream(self._m, ctypes.byref(p)))
        return p.value

    def launch_count(self):
        return int(library().mom6b_launch_count(self._m))

    def reset_launch_count(self):
        library().mom6b_reset_launch_count(self._m)

    def kernel_timing(self, enable=True):
        _check(library().mom6b_kernel_timing(self._m, int(enable)))

    def kernel_time_ms(self, name):
        ms = ctypes.c_double()
        n = ctypes.c_int64()
        _check(library().mom6b_kernel_time_ms(self._m, name.encode(), ctypes.byref(ms),
                                              ctypes.byref(n)))
        return ms.value, n.value

    def set_coriolis_scheme(self, scheme):
        """1 SADOURNY75_ENERGY (default), 2 ARAKAWA_HSU90, 3 ARAKAWA_LAMB81."""
        _check(library().mom6b_set_coriolis_scheme(self._m, int(scheme)))

    def set_continuity_merid(self, on=True):
        """Zonal then meridional continuity in every step (FP64 form)."""
        _check(library().mom6b_set_continuity_merid(self._m, int(bool(on))))

    def set_hor_visc(self, laplacian=True, biharmonic=False, smagorinsky=False, leith=False,
                     no_slip=False, better_bound=False, modified_leith=False, Ah=1.0e10):
        """hor_visc_init's scheme options (FP64 form for any but the default)."""
        o = HorVisc(int(bool(laplacian)), int(bool(biharmonic)), int(bool(smagorinsky)),
                    int(bool(leith)), int(bool(no_slip)), int(bool(better_bound)),
                    int(bool(modified_leith)), float(Ah))
        _check(library().mom6b_set_hor_visc(self._m, ctypes.byref(o)))

    def set_bt_overlap(self, on=True):
        """Run the barotropic chain on a second stream beside the 3-D chain."""
        _check(library().mom6b_set_bt_overlap(self._m, int(bool(on))))

    def set_wait_limit(self, cycles=0, stall_test=False):
        """Bound of the barotropic barrier waits (clock64 cycles, 0: default);
        stall_test=True makes the next steps' first barrier wait for an
        arrival that never comes (a testing aid for the timeout path)."""
        _check(library().mom6b_set_wait_limit(self._m, int(cycles), int(bool(stall_test))))

    def set_visc_remnant(self, on=True):
        """Every vertvisc also writes visc_rem_u / visc_rem_v and the continuity
        after it runs with them (zonal_mass_flux's use_visc_rem form; FP64)."""
        _check(library().mom6b_set_visc_remnant(self._m, int(bool(on))))

    def continuity_pass(self, direction, dt):
        """One continuity pass ("x" or "y") from (u or v, h0) into h."""
        _check(library().mom6b_continuity_pass(self._m, {"x": 0, "y": 1}[direction],
                                               float(dt)))

    # ---- diagnostics (mom6_diag.F90) and binary dumps ----
    def diag_init(self, output_dir="./", output_freq=1):
        _check(library().mom6b_diag_init(self._m, str(output_dir).encode(), int(output_freq)))

    def diag_end(self):
        _check(library().mom6b_diag_end(self._m))

    def diag_register(self, name, long_name, units, ndims, position, output_mode):
        """register_diag_field: the id, -1 when inactive."""
        i = ctypes.c_int()
        _check(library().mom6b_diag_register(self._m, name.encode(), long_name.encode(),
                                             units.encode(), int(ndims), position.encode(),
                                             int(output_mode), ctypes.byref(i)))
        return i.value

    def diag_post(self, diag_id, field):
        """post_data_2d / post_data_3d of a device field: a model field name
        or a CUDA tensor of the model's 2-D or 3-D shape (float64)."""
        ptr, nd = self._device_field(field)
        fn = library().mom6b_diag_post_3d if nd == 3 else library().mom6b_diag_post_2d
        _check(fn(self._m, int(diag_id), ptr))

    def diag_post_product_sum(self, diag_id, a, b, position="u"):
        """post_product_sum_u / _v of two device 3-D fields."""
        pa, _ = self._device_field(a)
        pb, _ = self._device_field(b)
        fn = (library().mom6b_diag_post_product_sum_u if position == "u"
              else library().mom6b_diag_post_product_sum_v)
        _check(fn(self._m, int(diag_id), pa, pb))

    def _device_field(self, f):
        """(device pointer, 2 or 3) of a model field name, or of a contiguous
        float64 CUDA tensor of n1*n2 or n1*n2*nk elements whose memory holds
        the field in the reference (column-major) layout."""
        if isinstance(f, str):
            return ctypes.c_void_p(self.device_ptr(f)), len(self.shape(f))
        n2d = self.n1 * self.n2
        if not (f.is_cuda and f.dtype.is_floating_point and f.element_size() == 8
                and f.is_contiguous() and f.numel() in (n2d, n2d * self.nk)):
            raise ValueError("a contiguous float64 CUDA tensor of the model's 2-D or 3-D size")
        return ctypes.c_void_p(f.data_ptr()), 2 if f.numel() == n2d else 3

    def diag_stats(self, diag_id):
        """(min, max, mean, rms) of the last post of diag_id."""
        out = (ctypes.c_double * 4)()
        _check(library().mom6b_diag_stats(self._m, int(diag_id), out))
        return tuple(out)

    def diag_report(self):
        out = (ctypes.c_int * 3)()
        _check(library().mom6b_diag_report(self._m, out))
        return dict(zip(["registered", "post_calls", "call_count"], list(out)))

    def diag_driver(self, output_mode=1):
        """The diagnostics of rk2_serial_driver with diag_mode = 1 (KE,
        diffu_sum, diffv_sum, mass), posted by every later step call."""
        _check(library().mom6b_diag_driver(self._m, int(output_mode)))

    def write_field_bin(self, name, path):
        _check(library().mom6b_write_field_bin(self._m, FID[name], str(path).encode()))

    def read_field_bin(self, name, path):
        _check(library().mom6b_read_field_bin(self._m, FID[name], str(path).encode()))

    # ---- learned barotropic surrogate ----
    def surrogate_train(self, nstates=8, nsteps=2000, batch=65536, lr=1e-3, seed=1):
        out = (ctypes.c_double * 4)()
        _check(library().mom6b_surrogate_train(self._m, int(nstates), int(nsteps), int(batch),
                                               float(lr), int(seed), out))
        return dict(zip(["loss_first", "loss_last", "batches", "seconds"], list(out)))

    def surrogate_eval(self, seed=1, state=100, nsteps=10):
        """Transport error of the network on a held-out state of the seeded
        family (see mom6b_surrogate_eval)."""
        out = (ctypes.c_double * 3)()
        _check(library().mom6b_surrogate_eval(self._m, int(seed), int(state), int(nsteps), out))
        return dict(zip(["rel_error", "zero_prediction_error", "calls"], list(out)))

    def surrogate_enable(self, on=True, shadow_every=10, threshold=1e-3):
        _check(library().mom6b_surrogate_enable(self._m, int(on), int(shadow_every),
                                                float(threshold)))

    def surrogate_status(self):
        out = (ctypes.c_double * 10)()
        _check(library().mom6b_surrogate_status(self._m, out))
        keys = ["enabled", "fallen_back", "steps", "shadow_checks", "fallbacks",
                "last_shadow_error", "max_shadow_error", "loss_first", "loss_last",
                "train_batches"]
        return dict(zip(keys, list(out)))

    def surrogate_params(self):
        n = int(library().mom6b_surrogate_param_count())
        a = np.zeros(n, dtype=np.float32)
        _check(library().mom6b_surrogate_get_params(
            self._m, a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n))
        return a

    def set_surrogate_params(self, a):
        a = np.ascontiguousarray(a, dtype=np.float32)
        _check(library().mom6b_surrogate_set_params(
            self._m, a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), a.size))


def abi_set_deferral(on=True):
    """Defer the launch_bt_* substep calls of one btstep_cuda_c into one
    persistent loop (mom6b_abi_set_deferral; on by default)."""
    _check(library().mom6b_abi_set_deferral(int(bool(on))))


class HaloGroup:
    """The library's in-process halo exchange among npes_x * npes_y subdomain
    models (mom6b_halo_group_*): join each model at its rank (pos_x * npes_y
    + pos_y), then step every model from its own host thread."""

    def __init__(self, npes_x, npes_y, timeout_s=60.0):
        h = ctypes.c_void_p()
        _check(library().mom6b_halo_group_create(int(npes_x), int(npes_y), float(timeout_s),
                                                 ctypes.byref(h)))
        self._g = h
        self.members = {}

    def join(self, model, rank):
        _check(library().mom6b_halo_group_join(self._g, model._m, int(rank)))
        self.members[int(rank)] = model

    def close(self):
        if getattr(self, "_g", None):
            library().mom6b_halo_group_destroy(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def subdomain_config(ni_global, nj_global, npes_x, npes_y, rank):
    """(ni, nj, subdomain) of one rank's model: the global compute domain
    (ni_global - 4 by nj_global - 4 points) split as mpi_domain_init splits
    it (mom6_mpi_domain.F90:57-137, remainder to the first positions)."""
    from .decomp import Decomposition
    d = Decomposition(ni_global - 4, nj_global - 4, npes_x, npes_y, rank)
    cuts = sum(bit for side, bit in (("W", CUT_W), ("E", CUT_E), ("S", CUT_S), ("N", CUT_N))
               if d.neighbour(side) is not None)
    return d.ni_local + 4, d.nj_local + 4, (ni_global, nj_global, d.i_offset, d.j_offset, cuts)


def make_config(ni=180, nj=180, nk=75, bt_nsteps=30, init_mode=INIT_CFG, seed=0, dt=None,
                Kh=None, bc_fill=None, precision=FP64, device=0, use_graph=False):
    """A mom6b_config with the defaults of init_mode and the given overrides."""
    c = Config()
    _check(library().mom6b_config_default(ctypes.byref(c), init_mode))
    c.ni, c.nj, c.nk, c.bt_nsteps, c.seed = ni, nj, nk, bt_nsteps, seed
    if dt is not None:
        c.dt = dt
    if Kh is not None:
        c.Kh = Kh
    if bc_fill is not None:
        c.bc_fill = int(bc_fill)
    c.precision, c.device, c.use_graph = precision, device, int(use_graph)
    return c


TUNING_KEYS = ["tend_tile", "tend_kc", "vv_nb", "vv_ch", "ppm_nb", "faces_nb", "bt_tile"]


class Ensemble:
    """Many independent domains of any sizes advanced together in the mixed
    form, one launch per phase for all of them (mom6b_ensemble_*).

    domains: list of dicts of make_config arguments (ni, nj, nk, bt_nsteps,
    seed, init_mode, dt, ...); precision is MIXED for every domain."""

    def __init__(self, domains, device=0, use_graph=True):
        L = library()
        n = len(domains)
        arr = (Config * n)()
        for q, kw in enumerate(domains):
            kw = dict(kw)
            kw["precision"] = MIXED
            kw["device"] = device
            arr[q] = make_config(**kw)
        self.cfgs = [arr[q] for q in range(n)]
        h = ctypes.c_void_p()
        _check(L.mom6b_ensemble_create(n, arr, ctypes.byref(h)))
        self._e = h
        self.n = n
        self.dims = []
        for q in range(n):
            dims = (ctypes.c_int * 8)()
            _check(L.mom6b_dims(L.mom6b_ensemble_member(self._e, q), dims))
            self.dims.append(tuple(dims))
        if not use_graph:
            raise ValueError("the ensemble always steps through its CUDA graph")

    def close(self):
        if getattr(self, "_e", None):
            library().mom6b_ensemble_destroy(self._e)
            self._e = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return self.n

    def step(self, n=1):
        _check(library().mom6b_ensemble_step(self._e, int(n)))

    def synchronize(self):
        _check(library().mom6b_ensemble_synchronize(self._e))

    def stream(self):
        p = ctypes.c_void_p()
        _check(library().mom6b_ensemble_stream(self._e, ctypes.byref(p)))
        return p.value

    def launch_count(self):
        return int(library().mom6b_ensemble_launch_count(self._e))

    def shape(self, d, name):
        n1, n2, nk = self.dims[d][0], self.dims[d][1], self.dims[d][2]
        return (n1, n2, nk) if name in FIELDS_3D else (n1, n2)

    def get(self, d, name):
        a = np.zeros(self.shape(d, name), dtype=np.float64, order="F")
        _check(library().mom6b_ensemble_get_field(self._e, int(d), FID[name], _dptr(a), a.size))
        return a

    def cell_layers(self):
        """Compute cells x layers of all domains (the unit of the ensemble rate)."""
        tot = 0
        for c in self.cfgs:
            tot += c.ni * c.nj * c.nk
        return tot

    def autotune(self, reps=3):
        out = (ctypes.c_double * 5)()
        _check(library().mom6b_ensemble_autotune(self._e, int(reps), out))
        return dict(zip(["tendency", "vertvisc", "ppm", "faces", "btstep"], list(out)))

    def tuning(self):
        out = (ctypes.c_int * 7)()
        _check(library().mom6b_ensemble_get_tuning(self._e, out))
        return dict(zip(TUNING_KEYS, list(out)))

    def set_tuning(self, t):
        vals = (ctypes.c_int * 7)(*[int(t[k]) for k in TUNING_KEYS])
        _check(library().mom6b_ensemble_set_tuning(self._e, vals))


def _fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class Mlp:
    """The surrogate network alone (mom6b_mlp_*): gradients, Adam steps and
    predictions of batches of 175 fp32 features."""

    def __init__(self, batch=1024, seed=0):
        h = ctypes.c_void_p()
        _check(library().mom6b_mlp_create(int(batch), int(seed), ctypes.byref(h)))
        self._p = h
        self.nparams = int(library().mom6b_mlp_param_count())

    def close(self):
        if getattr(self, "_p", None):
            library().mom6b_mlp_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        a = np.zeros(self.nparams, dtype=np.float32)
        _check(library().mom6b_mlp_get_params(self._p, _fptr(a), a.size))
        return a

    def set_params(self, a):
        a = np.ascontiguousarray(a, dtype=np.float32)
        _check(library().mom6b_mlp_set_params(self._p, _fptr(a), a.size))

    def gradients(self, X, Y):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        B = X.shape[0]
        g = np.zeros(self.nparams, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        out = np.zeros((B, 2), dtype=np.float32)
        _check(library().mom6b_mlp_gradients(self._p, _fptr(X), _fptr(Y), B, _fptr(g),
                                             _fptr(loss), _fptr(out)))
        return g, float(loss[0]), out

    def train(self, X, Y, lr=1e-3, nsteps=1):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        losses = np.zeros(max(nsteps, 1), dtype=np.float32)
        _check(library().mom6b_mlp_train(self._p, _fptr(X), _fptr(Y), X.shape[0], float(lr),
                                         int(nsteps), _fptr(losses)))
        return losses[:nsteps]

    def predict(self, X):
        X = np.ascontiguousarray(X, dtype=np.float32)
        out = np.zeros((X.shape[0], 2), dtype=np.float32)
        _check(library().mom6b_mlp_predict(self._p, _fptr(X), X.shape[0], _fptr(out)))
        return out


class CudaCDriver:
    """The reference's CUDA C host side (rk2_cuda_c_driver + the src/cuda_c
    Fortran wrappers) restated in C++ and driven through the launch_* ABI.

    kernel_lib=None runs this library's own entry points; a path runs the
    entry points of another shared object with the same symbols."""

    def __init__(self, ni=180, nj=180, nk=75, bt_nsteps=30, dt=300.0, kernel_lib=None,
                 init_mode=INIT_REF, seed=0):
        """init_mode INIT_REF: the driver's analytic state (dt as given);
        INIT_CFG: the seeded beta-plane state a Model of the same arguments
        builds (its Kh and viscosity defaults)."""
        L = library()
        h = ctypes.c_void_p()
        lib = kernel_lib.encode() if kernel_lib else None
        c = make_config(ni, nj, nk, bt_nsteps, init_mode, seed, dt=dt)
        _check(L.mom6b_cudac_create_cfg(ctypes.byref(c), lib, ctypes.byref(h)))
        self._h = h
        self.n1, self.n2, self.nk = ni + 2, nj + 2, nk

    def close(self):
        if getattr(self, "_h", None):
            library().mom6b_cudac_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n=1):
        _check(library().mom6b_cudac_step(self._h, n))

    def get(self, name):
        L = library()
        fid = FID[name]
        n = L.mom6b_cudac_field_size(self._h, fid)
        if n == 0:
            raise KeyError(name)
        a = np.empty(n, dtype=np.float64)
        _check(L.mom6b_cudac_get_field(self._h, fid, _dptr(a), n))
        shp = (self.n1, self.n2, self.nk) if n == self.n1 * self.n2 * self.nk else (self.n1, self.n2)
        return a.reshape(shp, order="F")
