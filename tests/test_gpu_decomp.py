"""The decomposed FP64 step on one GPU equals the single-domain step bit for bit.

npes_x x npes_y subdomain models (mom6b_config's subdomain fields: global
sizes, offsets, cut sides) run on cuda:0, each from its own host thread, and
exchange halos through the library's in-process halo group (peer 3-D copies
between the models' buffers, two host barriers per exchange) at the points of
the decomposed driver (rk2_mpi_cuda_c_driver.F90:305-412): up, vp before the
predictor continuity, h after it, u, v before the corrector continuity, and
the barotropic eta, ubt, vbt before every substep (one launch per substep).
Each subdomain's compute domain is compared with the single-domain model's
at the same global points.  The same decomposition of the oracle is held to
the undecomposed oracle on gloo ranks in test_decomp_step.py.
"""
import threading

import numpy as np
import pytest

# prognostic state, the step's other outputs, and the continuity's BT_cont
FIELDS = ("u", "v", "h", "eta", "up", "vp", "uh", "ubt_av", "vbt_av", "eta_av",
          "taux_bot", "tauy_bot", "du_cor", "hu_bt", "FA_u_W0", "uBT_EE")


def _run(px, py, NI, NJ, mode, exact, nk=6, nbt=9, nsteps=2):
    from hackathon_mom6_miniapp_b200 import HaloGroup, Model, subdomain_config
    glob = Model(NI, NJ, nk, nbt, init_mode=mode, bc_fill=False, exact=exact)
    group = HaloGroup(px, py, timeout_s=120.0)
    locs = []
    for r in range(px * py):
        ni, nj, sub = subdomain_config(NI, NJ, px, py, r)
        m = Model(ni, nj, nk, nbt, init_mode=mode, bc_fill=False, exact=exact, subdomain=sub)
        group.join(m, r)
        locs.append((m, sub))
    errs = []

    def run(m):
        try:
            m.step(nsteps)
            m.synchronize()
        except Exception as e:   # reported below
            errs.append(e)

    threads = [threading.Thread(target=run, args=(m,)) for m, _ in locs]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=600)
    assert not errs, errs
    glob.step(nsteps)
    glob.synchronize()
    bad = {}
    for r, (m, sub) in enumerate(locs):
        io, jo = sub[2], sub[3]
        i0, i1, j0, j1 = m.is_ - 1, m.ie, m.js - 1, m.je
        for name in FIELDS:
            a = m.get(name)[i0:i1, j0:j1]
            g = glob.get(name)[i0 + io:i1 + io, j0 + jo:j1 + jo]
            n = int(np.count_nonzero(a != g))
            if n:
                bad[(r, name)] = n
    group.close()
    return bad


@pytest.mark.gpu
@pytest.mark.parametrize("px,py,NI,NJ,mode", [
    (2, 1, 44, 36, 1),    # an east-west cut, seeded state
    (1, 2, 40, 41, 0),    # a north-south cut, analytic state
    (2, 2, 45, 39, 1),    # four subdomains, uneven split, both cuts and the corner
])
def test_decomposed_step_is_bit_identical(px, py, NI, NJ, mode):
    bad = _run(px, py, NI, NJ, mode, exact=True)
    assert not bad, bad


@pytest.mark.gpu
def test_decomposed_fast_form_is_bit_identical():
    """The fast FP64 kernels evaluate every point independently of the
    decomposition, so the decomposed fast step is the single-domain fast step."""
    bad = _run(2, 2, 46, 40, 1, exact=False)
    assert not bad, bad


@pytest.mark.gpu
def test_cut_model_refuses_to_step_without_exchange():
    from hackathon_mom6_miniapp_b200 import Model, Mom6bError, subdomain_config
    ni, nj, sub = subdomain_config(40, 40, 2, 1, 0)
    m = Model(ni, nj, 4, 5, init_mode=1, bc_fill=False, exact=True, subdomain=sub)
    with pytest.raises(Mom6bError):
        m.step(1)


@pytest.mark.gpu
@pytest.mark.parametrize("batch", [False, True])
def test_python_exchange_hook_is_bit_identical(batch):
    """Model.set_exchange with decomp.LocalHaloExchange: the library calls back
    into Python with torch views of its device fields on the model's stream
    (the path a one-process-per-GPU run takes with decomp.HaloExchange over
    NCCL); the decomposed step equals the single-domain one."""
    from hackathon_mom6_miniapp_b200 import Model, subdomain_config
    from hackathon_mom6_miniapp_b200.decomp import Decomposition, LocalBoard, LocalHaloExchange
    px, py, NI, NJ, nk, nbt, nsteps = 2, 2, 40, 36, 5, 7, 2
    glob = Model(NI, NJ, nk, nbt, init_mode=1, bc_fill=False, exact=True)
    board = LocalBoard(px * py, timeout=120.0)
    locs, errs = [], []
    for r in range(px * py):
        ni, nj, sub = subdomain_config(NI, NJ, px, py, r)
        m = Model(ni, nj, nk, nbt, init_mode=1, bc_fill=False, exact=True, subdomain=sub)
        x = LocalHaloExchange(Decomposition(NI - 4, NJ - 4, px, py, r), board)
        if batch:   # one round per exchange point
            m.set_exchange(x.exchange_many, batch=True)
        else:       # one round per field
            m.set_exchange(lambda t, kind, x=x: x.exchange(t))
        locs.append((m, sub))

    def run(m):
        try:
            m.step(nsteps)
            m.synchronize()
        except Exception as e:
            errs.append((e, getattr(m, "exchange_error", None)))

    ts = [threading.Thread(target=run, args=(m,)) for m, _ in locs]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=600)
    assert not errs, errs
    glob.step(nsteps)
    for m, sub in locs:
        io, jo = sub[2], sub[3]
        i0, i1, j0, j1 = m.is_ - 1, m.ie, m.js - 1, m.je
        for name in ("u", "v", "h", "eta", "ubt_av", "vbt_av", "eta_av"):
            a = m.get(name)[i0:i1, j0:j1]
            g = glob.get(name)[i0 + io:i1 + io, j0 + jo:j1 + jo]
            assert np.array_equal(a, g), (sub, name, int(np.count_nonzero(a != g)))
        m.set_exchange(None)


@pytest.mark.gpu
def test_halo_group_reports_a_member_that_never_arrives():
    """Failure detection on the host: one member of a 2x1 group never steps.
    The other's first exchange waits out the group's timeout, the step returns
    an error instead of hanging, and the group stays failed (a later exchange
    fails at once).  No kernel waits on another: the wait is a host barrier."""
    import time
    from hackathon_mom6_miniapp_b200 import HaloGroup, Model, Mom6bError, subdomain_config
    group = HaloGroup(2, 1, timeout_s=2.0)
    ms = []
    for r in range(2):
        ni, nj, sub = subdomain_config(40, 36, 2, 1, r)
        m = Model(ni, nj, 4, 5, init_mode=1, bc_fill=False, exact=True, subdomain=sub)
        group.join(m, r)
        ms.append(m)
    t0 = time.perf_counter()
    with pytest.raises(Mom6bError):
        ms[0].step(1)
    waited = time.perf_counter() - t0
    assert 1.5 < waited < 60.0, waited
    t0 = time.perf_counter()
    with pytest.raises(Mom6bError):
        ms[0].step(1)
    assert time.perf_counter() - t0 < 1.5
    ms[0].synchronize()
    group.close()
