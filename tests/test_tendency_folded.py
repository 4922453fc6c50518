"""The fast tendency's folded uniform metrics, restated in numpy and held to
the oracle's serial phases on CPU.

On a grid whose metrics are uniform, the fast FP64 tendency (tendency_tile with
FAST and uniform metrics) multiplies its stencils by products of the metrics
formed once on the host (TendFold, mom6b_api.cu detect_uniform) instead of
evaluating the serial expressions term by term: the relative vorticity as
kRv dv - kRu du, the potential vorticity as absv kQn / (S + kQe), the strain
stresses as (kSv dv + kSu du)(h00 + h10 + h01 + h11) and h (kXv dv - kXu du),
the kinetic energy as kKu (uc^2 + um^2) + kKv (vc^2 + vm^2), the transports as
kTu u (h + h+), and the Coriolis and viscous accelerations from those.  This
restatement evaluates the same products over the interior of a seeded state and
must agree with the oracle's compute_transports, CorAdCalc and hor_visc
(rk2_serial_driver.F90:544-561, mom6_coriolis_serial.F90:112-252,
mom6_hor_visc_serial.F90:464-1109) to rounding: 1e-13 relative per field.  The
GPU kernel itself is held to the exact form in test_gpu_fast.py.
"""
import numpy as np

from oracle.pyoracle import INIT_CFG, Oracle

HV_NEGLECT = 1.0e-3


def _fold(o, Kh):
    """The products of TendFold from the oracle's (uniform) metric arrays."""
    m = {n: float(o.array(n)[1, 1]) for n in (
        "IareaT", "areaT", "dxCu", "dyCu", "IdxCu", "IdyCu", "dxCv", "dyCv", "IdxCv", "IdyCv",
        "IareaBu", "IareaCu", "IareaCv", "mask2dT", "mask2dBu", "Area_q", "dx2h", "dy2h", "dx2q",
        "dy2q", "DX_dyT", "DY_dxT", "DX_dyBu", "DY_dxBu", "reduction_xx", "reduction_xy")}
    mB = m["mask2dBu"]
    return m, dict(
        kRv=mB * m["dyCv"] * m["IareaBu"], kRu=mB * m["dxCu"] * m["IareaBu"],
        kQn=2.0 * m["Area_q"] / m["areaT"], kQe=2.0e-20 / m["areaT"],
        kSv=-0.25 * Kh * mB * mB * m["reduction_xy"] * m["DY_dxBu"] * m["IdyCv"],
        kSu=-0.25 * Kh * mB * mB * m["reduction_xy"] * m["DX_dyBu"] * m["IdxCu"],
        kKu=0.25 * m["dyCu"] / m["areaT"], kKv=0.25 * m["dxCv"] / m["areaT"],
        kXu=Kh * m["reduction_xx"] * m["DY_dxT"] * m["IdyCu"],
        kXv=Kh * m["reduction_xx"] * m["DX_dyT"] * m["IdxCv"],
        kTu=0.5 * m["dyCu"], kTv=0.5 * m["dxCv"], kCu=0.25 * m["IdxCu"], kCv=0.25 * m["IdyCv"],
        kHm=0.5 * m["mask2dT"], kDq=m["IdxCu"] * m["dx2q"] * m["IareaCu"],
        kDh=m["IdyCu"] * m["dy2h"] * m["IareaCu"], kEq=m["IdyCv"] * m["dy2q"] * m["IareaCv"],
        kEh=m["IdxCv"] * m["dx2h"] * m["IareaCv"])


def test_folded_tendency_matches_the_oracle_phases():
    Kh = 1.0e3
    o = Oracle(30, 24, 5, 30, INIT_CFG, seed=13, Kh=Kh)
    u, v, h = (np.asfortranarray(o.get(n)) for n in ("u", "v", "h"))
    m, K = _fold(o, Kh)
    cor = o.array("CoriolisBu")
    # 0-based slices: X(a, di, dj) is a(i + di, j + dj) on the interior block
    # i in [I0, I1], j in [J0, J1] (1-based; away from every boundary quirk)
    I0, I1, J0, J1 = o.is_ + 1, o.ie - 2, o.js + 1, o.je - 2

    def X(a, di=0, dj=0):
        return a[I0 - 1 + di:I1 + di, J0 - 1 + dj:J1 + dj]

    def corner_q_sxy(di, dj):
        dv = X(v, 1 + di, dj) - X(v, di, dj)
        du = X(u, di, 1 + dj) - X(u, di, dj)
        h00, h10, h01, h11 = X(h, di, dj), X(h, 1 + di, dj), X(h, di, 1 + dj), X(h, 1 + di, 1 + dj)
        a, b = h00 + h10, h01 + h11
        absv = X(cor, di, dj)[..., None] + (K["kRv"] * dv - K["kRu"] * du)
        S = (a + b) + ((h00 + h01) + (h10 + h11))
        q = absv * K["kQn"] / (S + K["kQe"])
        sxy = (K["kSv"] * dv + K["kSu"] * du) * (a + b)
        return q, sxy

    def centre_ke_sxx(di, dj):
        uc, um = X(u, di, dj), X(u, di - 1, dj)
        vc, vm = X(v, di, dj), X(v, di, dj - 1)
        ke = K["kKu"] * (uc * uc + um * um) + K["kKv"] * (vc * vc + vm * vm)
        sxx = X(h, di, dj) * (K["kXv"] * (vc - vm) - K["kXu"] * (uc - um))
        return ke, sxx

    uh = lambda di, dj: K["kTu"] * X(u, di, dj) * (X(h, di, dj) + X(h, di + 1, dj))
    vh = lambda di, dj: K["kTv"] * X(v, di, dj) * (X(h, di, dj) + X(h, di, dj + 1))

    q00, sxy00 = corner_q_sxy(0, 0)
    q0m, sxy0m = corner_q_sxy(0, -1)
    qm0, sxym0 = corner_q_sxy(-1, 0)
    ke00, sxx00 = centre_ke_sxx(0, 0)
    kep0, sxxp0 = centre_ke_sxx(1, 0)
    ke0p, sxx0p = centre_ke_sxx(0, 1)
    CAu = (K["kCu"] * (q00 * (vh(1, 0) + vh(0, 0)) + q0m * (vh(0, -1) + vh(1, -1)))
           - m["IdxCu"] * (kep0 - ke00))
    CAv = -(K["kCv"] * (qm0 * (uh(-1, 0) + uh(-1, 1)) + q00 * (uh(0, 0) + uh(0, 1)))
            + m["IdyCv"] * (ke0p - ke00))
    diffu = ((K["kDq"] * (sxy0m - sxy00) + K["kDh"] * (sxx00 - sxxp0))
             / (K["kHm"] * (X(h) + X(h, 1, 0)) + HV_NEGLECT))
    diffv = ((K["kEq"] * (sxym0 - sxy00) - K["kEh"] * (sxx00 - sxx0p))
             / (K["kHm"] * (X(h) + X(h, 0, 1)) + HV_NEGLECT))

    ouh, ovh = o.transports(u, v, h)
    ocu, ocv = o.coriolis(u, v, h, ouh, ovh)
    odu, odv = o.hor_visc(u, v, h)

    def close(a, b, name):
        assert np.linalg.norm(a - b) <= 1e-13 * np.linalg.norm(b), name

    close(uh(0, 0), X(ouh), "uh")
    close(vh(0, 0), X(ovh), "vh")
    close(CAu, X(ocu), "CAu")
    close(CAv, X(ocv), "CAv")
    close(diffu, X(odu), "diffu")
    close(diffv, X(odv), "diffv")
