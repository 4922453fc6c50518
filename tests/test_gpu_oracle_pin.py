"""Pin the oracle against the reference's own compiled code.

The reference has no golden vectors and its serial Fortran does not compile
here, but its CUDA C kernels (src/cuda_c/*.cu) build from their sources into
oracle/_ref.  Where the serial semantics the oracle restates and those
kernels coincide, both are run on the same inputs (the oracle's grid and a
perturbed state) and compared:

  horizontal viscosity        stress + divergence kernels
  Coriolis (Sadourny)         phase1 + vorticity_pv + sadourny kernels
  barotropic loop             the 11 bt kernels, nstep substeps, with the
                              oracle switched to the extended transport ranges
  vertical viscosity          the fused cra kernels, Rayleigh drag set to zero
  continuity                  PPM (positive-definite limiter) + fluxes + Newton
                              adjustment + convergence

Coriolis and the barotropic loop agree bit for bit.  The other three carry
rounding-level differences between the serial and the CUDA C sources, so
they are compared to 1e-13 relative: horizontal viscosity associates the
stress products differently (serial -(Kh sh) (h red), CUDA C
((-Kh sh) h) red), vertical viscosity associates z**6 in botfn differently,
and continuity differs in the real(4) locals of PPM_limit_pos and the
single-precision tolerance literals of the serial Newton loop.
"""
import ctypes
import os

import numpy as np
import pytest

from oracle.pyoracle import INIT_REF, Oracle
from tests.abi_cases import bind, declarations

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "libref_cuda_c_nofma.so")
DECLS = declarations(os.path.join(ROOT, "include", "mom6_cuda_c.h"))


class RefKernels:
    """Call the reference's launch_* entry points with named device arrays."""

    def __init__(self):
        import torch
        if not os.path.exists(REF):
            pytest.skip("oracle/_ref not built (make -C oracle ref)")
        self.lib = ctypes.CDLL(REF)
        self.torch = torch
        self.dev = {}

    def put(self, name, a):
        self.dev[name] = self.torch.from_numpy(np.ravel(a, order="F").copy()).cuda()

    def zeros(self, name, shape):
        self.dev[name] = self.torch.zeros(int(np.prod(shape)), dtype=self.torch.float64,
                                          device="cuda")

    def get(self, name, shape):
        self.torch.cuda.synchronize()
        return self.dev[name].cpu().numpy().reshape(shape, order="F")

    def call(self, fn, **kw):
        decl = DECLS[fn]
        args = []
        for kind, a in decl:
            v = kw.get(a, None)
            if kind == "p":
                args.append(ctypes.c_void_p(self.dev[v if isinstance(v, str) else a].data_ptr()))
            elif kind == "v":
                args.append(None)
            else:
                args.append(v)
        bind(self.lib, fn, decl)(*args)


def _setup(ni=36, nj=30, nk=8, seed=3):
    o = Oracle(ni, nj, nk, 30, INIT_REF, dt=300.0)
    o.step(1)
    rng = np.random.default_rng(seed)
    st = {}
    for f in ("u", "v", "h", "eta", "ubt", "vbt"):
        a = o.get(f)
        scale = 0.05 if f in ("u", "v", "ubt", "vbt") else (1.0 if f == "h" else 0.05)
        st[f] = np.asfortranarray(a + scale * rng.standard_normal(a.shape))
    st["uh"], st["vh"] = o.transports(st["u"], st["v"], st["h"])
    return o, st


def _geom(o, fam="3d"):
    n1, n2, nk = o.shape("u")
    d = o.dims if hasattr(o, "dims") else None
    is_, ie, js, je = o.is_, o.ie, o.js, o.je
    bx, by = 32, 4
    return dict(n1=n1, n2=n2, n3=nk, nz=nk, is_l=is_, ie_l=ie, js_l=js, je_l=je,
                grid_x=(n1 + bx - 1) // bx, grid_y=(n2 + by - 1) // by,
                grid_z=nk if fam == "3d" else 1, block_x=bx, block_y=by, block_z=1)


def _relmax(a, b):
    den = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / den)


@pytest.mark.gpu
def test_oracle_hor_visc_matches_reference_kernels():
    o, st = _setup()
    R = RefKernels()
    g = _geom(o)
    n1, n2, nk = g["n1"], g["n2"], g["n3"]
    for f in ("u", "v", "h"):
        R.put(f, st[f])
    for m in ("DY_dxT", "DX_dyT", "DY_dxBu", "DX_dyBu", "IdyCu", "IdxCu", "IdyCv", "IdxCv",
              "mask2dBu", "reduction_xx", "reduction_xy", "mask2dT", "IareaCu", "IareaCv",
              "dy2h", "dx2h", "dy2q", "dx2q"):
        R.put(m, o.array(m))
    for s in ("str_xx", "str_xy", "diffu", "diffv"):
        R.zeros(s, (n1, n2, nk))
    R.call("launch_stress_kernel", Kh_bg=100.0, **g)
    R.call("launch_divergence_kernel", h_neglect=1.0e-3, **g)
    du, dv = o.hor_visc(st["u"], st["v"], st["h"])
    ru, rv = R.get("diffu", (n1, n2, nk)), R.get("diffv", (n1, n2, nk))
    # The serial hor_visc keeps Kh in one persistent array written only on
    # the interior h points and the q-point ranges, so the last h column and
    # row (i = ie+1, j = je+1) keep Kh = 0 and str_xx = 0 there
    # (mom6_hor_visc_serial.F90, STEP 8 / STEP 11); the CUDA C kernel applies
    # Kh everywhere.  The faces that read those h points (u faces I = ie, v
    # faces J = je) differ by that definition and are left out.
    iu = (slice(o.is_ - 2, o.ie - 1), slice(o.js - 1, o.je))
    iv = (slice(o.is_ - 1, o.ie), slice(o.js - 2, o.je - 1))
    assert _relmax(du[iu], ru[iu]) < 1e-13
    assert _relmax(dv[iv], rv[iv]) < 1e-13


@pytest.mark.gpu
def test_oracle_coriolis_matches_reference_kernels():
    o, st = _setup()
    R = RefKernels()
    g = _geom(o)
    n1, n2, nk = g["n1"], g["n2"], g["n3"]
    for f in ("u", "v", "h", "uh", "vh"):
        R.put(f, st[f])
    for m in ("dyCv", "dxCu", "dyCu", "dxCv", "areaT", "IareaBu", "CoriolisBu", "mask2dBu",
              "IdxCu", "IdyCv"):
        R.put(m, o.array(m))
    R.put("Area_q", np.repeat(o.array("Area_q")[:, :, None], nk, axis=2))
    for s in ("dvdx", "dudy", "hArea_u", "hArea_v", "KE", "rel_vort", "abs_vort", "q", "Ih_q",
              "CAu", "CAv"):
        R.zeros(s, (n1, n2, nk))
    R.call("launch_phase1_kernel", **g)
    R.call("launch_vorticity_pv_kernel", **g)
    R.call("launch_coriolis_sadourny_kernel", **g)
    cu, cv = o.coriolis(st["u"], st["v"], st["h"], st["uh"], st["vh"])
    ru, rv = R.get("CAu", (n1, n2, nk)), R.get("CAv", (n1, n2, nk))
    iu = (slice(o.is_ - 1, o.ie - 1), slice(o.js - 1, o.je))
    iv = (slice(o.is_ - 1, o.ie), slice(o.js - 1, o.je - 1))
    assert np.array_equal(cu[iu], ru[iu]) and np.array_equal(cv[iv], rv[iv])


@pytest.mark.gpu
@pytest.mark.parametrize("scheme,coef", [(2, "launch_arakawa_hsu90_coef_kernel"),
                                         (3, "launch_arakawa_lamb81_coef_kernel")])
def test_oracle_arakawa_coriolis_matches_reference_kernels(scheme, coef):
    """The Arakawa HSU90 / LAMB81 branches of CorAdCalc (serial :171-193,
    :228-248), which the driver does not exercise, against the reference's
    coefficient and Arakawa kernels."""
    o, st = _setup()
    o.set_coriolis_scheme(scheme)
    R = RefKernels()
    g = _geom(o)
    n1, n2, nk = g["n1"], g["n2"], g["n3"]
    for f in ("u", "v", "h", "uh", "vh"):
        R.put(f, st[f])
    for m in ("dyCv", "dxCu", "dyCu", "dxCv", "areaT", "IareaBu", "CoriolisBu", "mask2dBu",
              "IdxCu", "IdyCv"):
        R.put(m, o.array(m))
    R.put("Area_q", np.repeat(o.array("Area_q")[:, :, None], nk, axis=2))
    for s in ("dvdx", "dudy", "hArea_u", "hArea_v", "KE", "rel_vort", "abs_vort", "q", "Ih_q",
              "a", "b", "c", "d", "CAu", "CAv"):
        R.zeros(s, (n1, n2, nk))
    R.call("launch_phase1_kernel", **g)
    R.call("launch_vorticity_pv_kernel", **g)
    R.call(coef, **g)
    R.call("launch_coriolis_arakawa_kernel", **g)
    cu, cv = o.coriolis(st["u"], st["v"], st["h"], st["uh"], st["vh"])
    ru, rv = R.get("CAu", (n1, n2, nk)), R.get("CAv", (n1, n2, nk))
    iu = (slice(o.is_ - 1, o.ie - 1), slice(o.js - 1, o.je))
    iv = (slice(o.is_ - 1, o.ie), slice(o.js - 1, o.je - 1))
    assert np.any(cu[iu] != 0)
    assert np.array_equal(cu[iu], ru[iu]), _relmax(cu[iu], ru[iu])
    assert np.array_equal(cv[iv], rv[iv]), _relmax(cv[iv], rv[iv])


@pytest.mark.gpu
def test_oracle_btstep_extended_matches_reference_kernels():
    o, st = _setup()
    o.set_bt_extended(True)
    R = RefKernels()
    g = _geom(o, "2d")
    n1, n2 = g["n1"], g["n2"]
    nstep, dtbt = 30, 300.0 / 30
    for f in ("eta", "ubt", "vbt"):
        R.put(f + "_in", st[f])
    for m in ("Datu", "Datv", "gtot_E", "gtot_W", "gtot_N", "gtot_S", "f_4_u", "f_4_v",
              "bt_rem_u", "bt_rem_v", "IareaT", "IdxCu", "IdyCv"):
        R.put(m, o.array(m))
    for s in ("eta", "eta_pred", "ubt", "vbt", "ubt_prev", "vbt_prev", "uhbt", "vhbt",
              "ubt_av", "vbt_av", "uhbt_av", "vhbt_av", "PFu", "PFv", "Cor_u", "Cor_v",
              "u_av_out", "v_av_out", "eta_out"):
        R.zeros(s, (n1, n2))
    c = dict(dtbt=dtbt, dgeo_de=1.0, trans_wt1=1.2, trans_wt2=-0.2, inv_nstep=1.0 / nstep, **g)
    R.call("launch_bt_init_kernel", **c)
    for n in range(1, nstep + 1):
        R.call("launch_bt_store_prev_u_kernel", **c)
        R.call("launch_bt_store_prev_v_kernel", **c)
        R.call("launch_bt_eta_pred_kernel", **c)
        R.call("launch_bt_pressure_force_u_kernel", **c)
        R.call("launch_bt_pressure_force_v_kernel", **c)
        order = ["v", "u"] if n % 2 == 1 else ["u", "v"]
        for w in order:
            R.call(f"launch_bt_coriolis_update_{w}_kernel", **c)
        R.call("launch_bt_transport_eta_accum_kernel", **c)
        R.call("launch_bt_eta_update_kernel", **c)
    R.call("launch_bt_copy_output_kernel", **c)
    ua, va, ea = o.btstep(st["eta"], st["ubt"], st["vbt"])
    assert np.array_equal(ua, R.get("u_av_out", (n1, n2)))
    assert np.array_equal(va, R.get("v_av_out", (n1, n2)))
    assert np.array_equal(ea, R.get("eta_out", (n1, n2)))


@pytest.mark.gpu
def test_oracle_vert_visc_matches_reference_kernels_without_rayleigh():
    o, st = _setup()
    n1, n2, nk = o.shape("u")
    o.set("Ray_u", np.zeros((n1, n2, nk), order="F"))
    o.set("Ray_v", np.zeros((n1, n2, nk), order="F"))
    R = RefKernels()
    g = _geom(o, "2d")
    dt, hn = 300.0, 1.0e-10
    for f in ("u", "v", "h"):
        R.put(f, st[f])
    R.put("taux", o.get("taux"))
    R.put("tauy", o.get("tauy"))
    for m in ("mask2dCu", "mask2dCv"):
        R.put(m, o.array(m))
    for s in ("visc_rem", "hvel"):
        R.zeros(s, (n1, n2, nk))
    R.zeros("z_i", (n1, n2, nk + 1))
    R.zeros("tau_bot", (n1, n2))
    c = dict(Kv=1.0e-4, Kv_ml=1.0e-2, Kv_extra_bbl=1.0e-2, Hmix=50.0, Hbbl=10.0, dt=dt,
             dt_Rho0=dt / 1035.0, h_neglect=hn, I_Hbbl=1.0 / (10.0 + hn), **g)
    R.call("launch_vert_visc_cra_u_kernel", visc_rem_u="visc_rem", taux_bot="tau_bot", **c)
    R.call("launch_vert_visc_cra_v_kernel", visc_rem_v="visc_rem", tauy_bot="tau_bot", **c)
    uo, vo = o.vert_visc(st["u"], st["v"], st["h"], dt)
    ru, rv = R.get("u", (n1, n2, nk)), R.get("v", (n1, n2, nk))
    iu = (slice(o.is_ - 2, o.ie), slice(o.js - 1, o.je))
    iv = (slice(o.is_ - 1, o.ie), slice(o.js - 2, o.je))
    assert _relmax(uo[iu], ru[iu]) < 1e-13
    assert _relmax(vo[iv], rv[iv]) < 1e-13


@pytest.mark.gpu
def test_oracle_continuity_matches_reference_kernels():
    o, st = _setup()
    R = RefKernels()
    g = _geom(o)
    n1, n2, nk = g["n1"], g["n2"], g["n3"]
    dt = 300.0
    hin = np.asfortranarray(np.maximum(st["h"], 1.0))
    R.put("u", st["u"])
    R.put("h_in", hin)
    for m in ("mask2dT", "dy_Cu", "IdxT", "IareaT", "dxT", "areaT", "mask2dCu", "dxCu"):
        R.put(m, o.array(m))
    for s in ("h_W", "h_E", "uh", "duhdu", "h"):
        R.zeros(s, (n1, n2, nk))
    for s in ("vrm", "uh_tot_0", "duhdu_tot_0", "du_max", "du_min", "du", "uhbt"):
        R.zeros(s, (n1, n2))
    fl = dict(monotonic=0, upwind_1st_flag=0, simple_2nd_flag=0, vol_CFL_flag=0,
              use_visc_rem_flag=0, use_por_face_flag=0, aggress_flag=0, better_iter_flag=1,
              use_vrm_max_flag=0)
    c = dict(h_min=2.0e-10, dt=dt, CFL_dt=0.5 / dt, I_dt=1.0 / dt, tol_eta_base=1.0e-12,
             tol_vel_val=3.0e8, **fl, **g)
    R.call("launch_ppm_reconstruction_3d_kernel", **c)
    R.call("launch_zonal_flux_layer_3d_kernel", por_face_areaU="h_W", visc_rem_u="h_W", **c)
    R.call("launch_visc_rem_max_kernel", visc_rem_max_out="vrm", visc_rem_u="h_W", **c)
    R.call("launch_uh_duhdu_tot_kernel", **c)
    R.call("launch_zonal_CFL_limits_kernel", du_max_CFL_out="du_max", du_min_CFL_out="du_min",
           visc_rem_u="h_W", visc_rem_max_in="vrm", **c)
    R.call("launch_zonal_flux_adjust_kernel", du_out="du", visc_rem_u="h_W",
           por_face_areaU="h_W", du_max_CFL_in="du_max", du_min_CFL_in="du_min",
           uh_tot_0_in="uh_tot_0", duhdu_tot_0_in="duhdu_tot_0", **c)
    R.call("launch_zonal_convergence_kernel", hin="h_in", **c)
    ho, uho = o.continuity(st["u"], hin, dt)
    rh, ruh = R.get("h", (n1, n2, nk)), R.get("uh", (n1, n2, nk))
    ih = (slice(o.is_ - 1, o.ie), slice(o.js - 1, o.je))
    iu = (slice(o.is_ - 2, o.ie), slice(o.js - 1, o.je))
    assert _relmax(ho[ih], rh[ih]) < 1e-13
    assert _relmax(uho[iu], ruh[iu]) < 1e-13


@pytest.mark.gpu
def test_oracle_remnant_matches_reference_kernels_without_rayleigh():
    """vert_visc_remnant (mom6_vert_visc_serial.F90:295-387) against the
    remnant half of the fused cra kernels (mom6_vert_visc_kernels.cu:69-157).
    Both start from the same coefficients, which differ by the z**6
    association of botfn (1e-13 relative); 1 - visc_rem carries that error
    and the cancellation of its subtraction (an ulp of 1 over 1 - visc_rem)."""
    o, st = _setup()
    n1, n2, nk = o.shape("u")
    o.set("Ray_u", np.zeros((n1, n2, nk), order="F"))
    o.set("Ray_v", np.zeros((n1, n2, nk), order="F"))
    R = RefKernels()
    g = _geom(o, "2d")
    dt, hn = 300.0, 1.0e-10
    for f in ("u", "v", "h"):
        R.put(f, st[f])
    R.put("taux", o.get("taux"))
    R.put("tauy", o.get("tauy"))
    for m in ("mask2dCu", "mask2dCv"):
        R.put(m, o.array(m))
    for s in ("vr_u", "vr_v", "hvel"):
        R.zeros(s, (n1, n2, nk))
    R.zeros("z_i", (n1, n2, nk + 1))
    R.zeros("tau_bot", (n1, n2))
    c = dict(Kv=1.0e-4, Kv_ml=1.0e-2, Kv_extra_bbl=1.0e-2, Hmix=50.0, Hbbl=10.0, dt=dt,
             dt_Rho0=dt / 1035.0, h_neglect=hn, I_Hbbl=1.0 / (10.0 + hn), **g)
    R.call("launch_vert_visc_cra_u_kernel", visc_rem_u="vr_u", taux_bot="tau_bot", **c)
    R.call("launch_vert_visc_cra_v_kernel", visc_rem_v="vr_v", tauy_bot="tau_bot", **c)
    o.vert_visc(st["u"], st["v"], st["h"], dt)
    ou, ov = o.vert_visc_remnant(dt)
    ru, rv = R.get("vr_u", (n1, n2, nk)), R.get("vr_v", (n1, n2, nk))
    iu = (slice(o.is_ - 2, o.ie), slice(o.js - 1, o.je))
    iv = (slice(o.is_ - 1, o.ie), slice(o.js - 2, o.je))
    for a, b in ((ou[iu], ru[iu]), (ov[iv], rv[iv])):
        assert (b < 1.0).any() and (b > 0.0).all()
        assert _relmax(a, b) < 1e-14
        assert _relmax(1.0 - a, 1.0 - b) < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("low", [False, True])
def test_oracle_continuity_with_remnant_matches_reference_kernels(low):
    """zonal_mass_flux with visc_rem_u present and use_visc_rem_max (the CFL
    limits, the Newton velocities u + du visc_rem, the marginal areas),
    set_zonal_BT_cont with visc_rem_lim, u_cor and zonal_flux_thickness
    scaled by visc_rem, against the reference's CUDA C chain with
    use_visc_rem_flag = use_vrm_max_flag = 1.  visc_rem is random in
    [0.3, 1]; with low, one layer in ten is 0.02, below 0.1 of the column
    maximum, so visc_rem_lim = min_visc_rem * visc_rem_max there.  The serial
    code assigns min_visc_rem the default-real literal 0.1
    (mom6_continuity_serial.F90:993), the CUDA C code the double 0.1
    (mom6_continuity_kernels.cu:693): 1.5e-8 relative in visc_rem_lim, which
    duL and duR take at such faces, so BT_cont's fields then agree to 1e-7
    only.  uBT_WW and uBT_EE divide by FAmt - FA_0, a difference of two
    nearly equal column areas, which magnifies the chains' 1e-13 rounding
    differences in the areas; they are held to 1e-8.  Everything else agrees
    as the plain chain does."""
    o, st = _setup()
    R = RefKernels()
    g = _geom(o)
    n1, n2, nk = g["n1"], g["n2"], g["n3"]
    dt = 300.0
    hin = np.asfortranarray(np.maximum(st["h"], 1.0))
    rng = np.random.default_rng(17)
    vr = rng.uniform(0.3, 1.0, (n1, n2, nk))
    if low:
        vr[rng.random((n1, n2, nk)) < 0.1] = 0.02
    vr = np.asfortranarray(vr)
    o.set("visc_rem_u", vr)
    R.put("u", st["u"])
    R.put("h_in", hin)
    R.put("vr", vr)
    for m in ("mask2dT", "dy_Cu", "IdxT", "IareaT", "dxT", "areaT", "mask2dCu", "dxCu"):
        R.put(m, o.array(m))
    for s in ("h_W", "h_E", "uh", "duhdu", "h", "h_u", "u_cor"):
        R.zeros(s, (n1, n2, nk))
    bt = ("FA_u_W0", "FA_u_WW", "uBT_WW", "FA_u_E0", "FA_u_EE", "uBT_EE")
    for s in ("vrm", "uh_tot_0", "duhdu_tot_0", "du_max", "du_min", "du", "uhbt") + bt:
        R.zeros(s, (n1, n2))
    fl = dict(monotonic=0, upwind_1st_flag=0, simple_2nd_flag=0, vol_CFL_flag=0,
              use_visc_rem_flag=1, use_por_face_flag=0, aggress_flag=0, better_iter_flag=1,
              use_vrm_max_flag=1)
    c = dict(h_min=2.0e-10, dt=dt, CFL_dt=0.5 / dt, I_dt=1.0 / dt, tol_eta_base=1.0e-12,
             tol_vel_val=3.0e8, **fl, **g)
    R.call("launch_ppm_reconstruction_3d_kernel", **c)
    R.call("launch_zonal_flux_layer_3d_kernel", por_face_areaU="h_W", visc_rem_u="vr", **c)
    R.call("launch_visc_rem_max_kernel", visc_rem_max_out="vrm", visc_rem_u="vr", **c)
    R.call("launch_uh_duhdu_tot_kernel", **c)
    R.call("launch_zonal_CFL_limits_kernel", du_max_CFL_out="du_max", du_min_CFL_out="du_min",
           visc_rem_u="vr", visc_rem_max_in="vrm", **c)
    R.call("launch_set_zonal_BT_cont_kernel", u="u", h_in="h_in", visc_rem_u="vr",
           por_face_areaU="h_W", visc_rem_max_in="vrm", du_max_CFL_in="du_max",
           du_min_CFL_in="du_min", uh_tot_0_in="uh_tot_0", duhdu_tot_0_in="duhdu_tot_0", **c)
    R.call("launch_zonal_flux_adjust_kernel", du_out="du", visc_rem_u="vr",
           por_face_areaU="h_W", du_max_CFL_in="du_max", du_min_CFL_in="du_min",
           uh_tot_0_in="uh_tot_0", duhdu_tot_0_in="duhdu_tot_0", **c)
    R.call("launch_u_cor_kernel", u_cor="u_cor", u="u", du="du", visc_rem_u="vr", **c)
    R.call("launch_zonal_flux_thickness_kernel", h_u="h_u", u="u_cor", h="h_in",
           por_face_areaU="h_W", visc_rem_u="vr", marginal_flag=1, has_visc_rem_flag=1, **c)
    R.call("launch_zonal_convergence_kernel", hin="h_in", **c)
    ho, uho = o.continuity(st["u"], hin, dt)
    ih = (slice(o.is_ - 1, o.ie), slice(o.js - 1, o.je))
    iu = (slice(o.is_ - 2, o.ie), slice(o.js - 1, o.je))
    assert _relmax(ho[ih], R.get("h", (n1, n2, nk))[ih]) < 1e-13
    assert _relmax(uho[iu], R.get("uh", (n1, n2, nk))[iu]) < 1e-13
    assert _relmax(o.get("hu_bt")[iu], R.get("h_u", (n1, n2, nk))[iu]) < 1e-13
    assert _relmax(o.get("du_cor")[iu], R.get("du", (n1, n2))[iu]) < 1e-12
    for f in bt:
        tol = 1e-7 if low else (1e-8 if f.startswith("uBT") else 1e-12)
        assert _relmax(o.get(f)[iu], R.get(f, (n1, n2))[iu]) < tol, f
