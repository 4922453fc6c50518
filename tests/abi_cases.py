"""Shared helpers for the reference-ABI tests.

`declarations()` parses include/*.h into {name: [(kind, arg_name), ...]}
with kind 'p' (double*), 'i' (int), 'd' (double), 'z' (size_t) or 'v'
(void* / const void*), so the ctypes signatures used by the tests come from
the headers the library ships.

`make_case()` builds seeded inputs for one launch_* entry point of the
reference's CUDA C backend: every array argument gets a shape and a value
distribution from its name and the kernel family it belongs to (thicknesses
positive, velocities of O(0.1 m/s), metrics of a 10 km grid, masks mostly 1
with a few land points), and every scalar its value in the reference driver.
"""
import ctypes
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")

_TYPE = [(re.compile(r"^(const\s+)?double\s*\*"), "p"), (re.compile(r"^(const\s+)?void\s*\*"), "v"),
         (re.compile(r"^int\b"), "i"), (re.compile(r"^double\b"), "d"),
         (re.compile(r"^size_t\b"), "z")]


def _strip_comments(text):
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    return re.sub(r"//[^\n]*", " ", text)


def declarations(header=None):
    """{function name: [(kind, arg name), ...], ...} for every prototype."""
    files = [header] if header else sorted(
        os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h"))
    out = {}
    for path in files:
        text = _strip_comments(open(path).read())
        text = re.sub(r"^\s*#[^\n]*", " ", text, flags=re.M)
        for stmt in re.split(r"[;{}]", text):
            m = re.match(r"\s*([A-Za-z_][\w\s\*]*?)\b(\w+)\s*\(([^()]*)\)\s*$", stmt, flags=re.S)
            if not m:
                continue
            name, args = m.group(2), m.group(3).strip()
            if name in ("if", "while", "for", "return", "sizeof"):
                continue
            parsed = []
            if args and args != "void":
                for a in args.split(","):
                    a = " ".join(a.split())
                    kind = None
                    for rx, k in _TYPE:
                        if rx.search(a):
                            kind = k
                            break
                    if kind is None:
                        kind = "x"  # struct pointers and other types of the high-level ABI
                    arg = re.sub(r"[\*\s]", " ", a).split()[-1]
                    parsed.append((kind, arg))
            out[name] = parsed
    return out


_CT = {"p": ctypes.c_void_p, "v": ctypes.c_void_p, "i": ctypes.c_int, "d": ctypes.c_double,
       "z": ctypes.c_size_t}


def bind(lib, name, decl):
    f = getattr(lib, name)
    f.argtypes = [_CT[k] for k, _ in decl]
    f.restype = None
    return f


# ---------------------------------------------------------------------------
# grid and value generators
# ---------------------------------------------------------------------------
class Grid:
    """A (n1, n2, n3) block with the reference's halo: is = js = 4 (1-based),
    ie = n1 - 3, je = n2 - 3, as init_ocean_grid lays them out."""

    def __init__(self, n1=38, n2=32, n3=8):
        self.n1, self.n2, self.n3 = n1, n2, n3
        self.is_l, self.js_l = 4, 4
        self.ie_l, self.je_l = n1 - 3, n2 - 3


FAMILY = {
    "bt": ("launch_bt_",),
    "cont": ("launch_ppm_", "launch_zonal_", "launch_visc_rem_max", "launch_uh_duhdu",
             "launch_set_zonal", "launch_u_cor"),
    "cor": ("launch_phase1", "launch_vorticity", "launch_arakawa", "launch_coriolis"),
    "hv": ("launch_stress", "launch_divergence"),
    "vv": ("launch_vert_visc",),
}


def family(name):
    for fam, prefixes in FAMILY.items():
        if name.startswith(prefixes):
            return fam
    raise KeyError(name)


_2D = {"bt": None,  # every array of the barotropic kernels is 2-D
       "cont": {"mask2dT", "mask2dCu", "dy_Cu", "IdxT", "IareaT", "dxT", "areaT", "dxCu",
                "uhbt", "du_out", "du", "du_max_CFL_out", "du_min_CFL_out", "du_max_CFL_in",
                "du_min_CFL_in", "uh_tot_0", "duhdu_tot_0", "uh_tot_0_in", "duhdu_tot_0_in",
                "visc_rem_max_out", "visc_rem_max_in", "FA_u_W0", "FA_u_WW", "uBT_WW",
                "FA_u_E0", "FA_u_EE", "uBT_EE"},
       "cor": {"dyCv", "dxCu", "dyCu", "dxCv", "areaT", "IareaBu", "CoriolisBu", "mask2dBu",
               "IdxCu", "IdyCv"},
       "hv": {"DY_dxT", "DX_dyT", "DY_dxBu", "DX_dyBu", "IdyCu", "IdxCu", "IdyCv", "IdxCv",
              "mask2dBu", "reduction_xx", "reduction_xy", "mask2dT", "IareaCu", "IareaCv",
              "dy2h", "dx2h", "dy2q", "dx2q"},
       "vv": {"mask2dCu", "mask2dCv", "taux_bot", "tauy_bot", "taux", "tauy"}}


def _shape(fam, name, g):
    if name in ("f_4_u", "f_4_v"):
        return (4, g.n1, g.n2)
    if fam == "vv" and name == "z_i":
        return (g.n1, g.n2, g.n3 + 1)
    two = _2D[fam]
    if two is None or name in two:
        return (g.n1, g.n2)
    return (g.n1, g.n2, g.n3)


def _values(fam, name, shape, rng):
    """Seeded values for an array argument, by name."""
    n = int(np.prod(shape))
    U = lambda lo, hi: rng.uniform(lo, hi, n)
    if name.startswith("mask"):
        v = np.ones(n)
        v[rng.random(n) < 0.04] = 0.0
        return v
    if name in ("h", "h_in", "hin", "h_W", "h_E"):
        return U(5.0, 80.0)
    if name in ("u", "v", "ubt", "vbt", "ubt_in", "vbt_in", "ubt_prev", "vbt_prev"):
        return U(-0.3, 0.3)
    if name in ("uh", "vh") and fam == "cor":
        return U(-1.0e5, 1.0e5)
    if name in ("eta", "eta_in", "eta_pred"):
        return U(-0.2, 0.2)
    if name in ("dxT", "dyCu", "dxCu", "dy_Cu", "dyCv", "dxCv", "dxCu"):
        return U(0.95e4, 1.05e4)
    if name in ("IdxT", "IdxCu", "IdyCu", "IdxCv", "IdyCv"):
        return 1.0 / U(0.95e4, 1.05e4)
    if name in ("areaT",):
        return U(0.95e8, 1.05e8)
    if name in ("IareaT", "IareaBu", "IareaCu", "IareaCv"):
        return 1.0 / U(0.95e8, 1.05e8)
    if name == "Area_q":
        return U(3.8e8, 4.2e8)
    if name in ("DY_dxT", "DX_dyT", "DY_dxBu", "DX_dyBu", "reduction_xx", "reduction_xy"):
        return U(0.9, 1.1)
    if name in ("dy2h", "dx2h", "dy2q", "dx2q"):
        return U(0.9e8, 1.1e8)
    if name == "CoriolisBu":
        return U(0.9e-4, 1.1e-4)
    if name in ("f_4_u", "f_4_v"):
        return U(2.0e-5, 3.0e-5)
    if name in ("bt_rem_u", "bt_rem_v"):
        return np.full(n, 0.999)
    if name in ("Datu", "Datv"):
        return U(3.5e7, 4.5e7)
    if name.startswith("gtot"):
        return U(4.8, 5.0)
    if name in ("taux", "tauy"):
        return U(-0.1, 0.1)
    if name in ("visc_rem_u", "visc_rem_v") and fam == "cont":
        return U(0.2, 1.0)
    if name == "por_face_areaU":
        return U(0.5, 1.0)
    if name in ("visc_rem_max_in",):
        return U(0.5, 1.0)
    if name == "uhbt":
        v = U(-2.0e5, 2.0e5)
        v[rng.random(n) < 0.3] = 0.0
        return v
    if name in ("uh_tot_0_in",):
        return U(-3.0e5, 3.0e5)
    if name in ("duhdu_tot_0_in",):
        return U(1.0e6, 4.0e6)
    if name == "du_max_CFL_in":
        return U(0.05, 0.5)
    if name == "du_min_CFL_in":
        return U(-0.5, -0.05)
    if name == "du":
        return U(-0.05, 0.05)
    if name in ("duhdu",):
        return U(1.0e4, 8.0e5)
    if name in ("q",) and fam == "cor":
        return U(-2e-5, 2e-5) + 1e-4
    if name in ("KE",):
        return U(0.0, 0.05)
    if name in ("dvdx", "dudy"):
        return U(-3.0e3, 3.0e3)
    if name in ("hArea_u", "hArea_v"):
        return U(1.0e9, 8.0e9)
    if name in ("str_xx", "str_xy"):
        return U(-50.0, 50.0)
    if name in ("a", "b", "c", "d"):
        return U(0.5e-5, 1.5e-5)
    # outputs and scratch: garbage that must not leak into a result
    return rng.standard_normal(n) * 1.0e3


SCALARS = {"dt": 600.0, "dtbt": 12.0, "dgeo_de": 1.0, "trans_wt1": 1.2, "trans_wt2": -0.2,
           "inv_nstep": 1.0 / 50.0, "h_min": 2.0e-10, "Kh_bg": 100.0, "Kv": 1.0e-4,
           "Kv_ml": 1.0e-2, "Kv_extra_bbl": 1.0e-2, "Hmix": 50.0, "Hbbl": 10.0,
           "I_Hbbl": 1.0 / (10.0 + 1.0e-10), "tol_eta_base": 1.0e-12, "tol_vel_val": 3.0e8}


def scalar(fam, name):
    if name == "h_neglect":
        return 1.0e-30 if fam == "vv" else 1.0e-3
    if name == "dt_Rho0":
        return 600.0 / 1035.0
    if name == "CFL_dt":
        return 0.5 / 600.0
    if name == "I_dt":
        return 1.0 / 600.0
    return SCALARS[name]


FLAG_NAMES = ("monotonic", "upwind_1st_flag", "simple_2nd_flag", "vol_CFL_flag",
              "use_visc_rem_flag", "use_por_face_flag", "aggress_flag", "better_iter_flag",
              "marginal_flag", "has_visc_rem_flag", "use_vrm_max_flag")

# flags as the reference wrappers pass them (mom6_continuity_cuda_c.F90:292-303,
# rk2_cuda_c_driver.F90:145)
DRIVER_FLAGS = {"monotonic": 1, "upwind_1st_flag": 0, "simple_2nd_flag": 0, "vol_CFL_flag": 0,
                "use_visc_rem_flag": 0, "use_por_face_flag": 0, "aggress_flag": 0,
                "better_iter_flag": 1, "marginal_flag": 1, "has_visc_rem_flag": 0,
                "use_vrm_max_flag": 0}


def flag_variants(decl):
    """The driver's flag setting, then each flag of the kernel flipped alone."""
    names = [a for k, a in decl if k == "i" and a in FLAG_NAMES]
    base = {a: DRIVER_FLAGS[a] for a in names}
    out = [dict(base)]
    for a in names:
        v = dict(base)
        v[a] = 1 - v[a]
        out.append(v)
    return out


def make_case(name, decl, g, seed, flags=None):
    """Arrays (name -> numpy array, Fortran order) and the scalar/int values."""
    fam = family(name)
    rng = np.random.default_rng(seed)
    arrays, values = {}, {}
    flags = flags or {}
    for kind, a in decl:
        if kind == "p":
            if a in arrays:
                continue
            shp = _shape(fam, a, g)
            arrays[a] = np.asfortranarray(_values(fam, a, shp, rng).reshape(shp, order="F"))
        elif kind == "d":
            values[a] = scalar(fam, a)
        elif kind == "i":
            if a in flags:
                values[a] = flags[a]
            elif a in ("n1", "n2", "n3", "nz", "is_l", "ie_l", "js_l", "je_l"):
                values[a] = {"n1": g.n1, "n2": g.n2, "n3": g.n3, "nz": g.n3, "is_l": g.is_l,
                             "ie_l": g.ie_l, "js_l": g.js_l, "je_l": g.je_l}[a]
            elif a in FLAG_NAMES:
                values[a] = DRIVER_FLAGS[a]
    # launch geometry as the wrappers compute it (bx = 32, by = 4)
    bx, by = 32, 4
    values.update({"grid_x": (g.n1 + bx - 1) // bx, "grid_y": (g.n2 + by - 1) // by,
                   "grid_z": g.n3 if fam != "bt" else 1, "block_x": bx, "block_y": by,
                   "block_z": 1})
    return arrays, values


# Arrays a kernel of the reference writes as scratch that this library
# intentionally leaves untouched.
SCRATCH = {"launch_vert_visc_cra_u_kernel": {"hvel", "z_i"},
           "launch_vert_visc_cra_v_kernel": {"hvel", "z_i"}}
