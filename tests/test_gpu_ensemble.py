"""The ensemble: many domains of uneven size in one launch per phase.

Every domain of an ensemble runs the same device code as a mixed-form model
of its own, so its fields must equal that model's bit for bit after the same
steps, under any launch shapes the autotuner may pick; the autotuner must
leave the state as it found it."""
import numpy as np
import pytest

from tests.util import rel_l2

FIELDS = ["h", "u", "v", "eta", "ubt_av", "vbt_av", "eta_av", "du_cor", "FA_u_W0",
          "taux_bot"]

# uneven sizes and depths, each with its own seed (the config-3 construction
# at small sizes)
DOMAINS = [dict(ni=40, nj=36, nk=12, bt_nsteps=30, seed=3),
           dict(ni=70, nj=50, nk=25, bt_nsteps=30, seed=7),
           dict(ni=36, nj=30, nk=8, bt_nsteps=30, seed=11),
           dict(ni=96, nj=90, nk=25, bt_nsteps=30, seed=2)]

OTHER_TUNING = dict(tend_tile=2, tend_kc=3, vv_nb=64, vv_ch=2, ppm_nb=256, faces_nb=64,
                    bt_tile=32)


def _singles(domains, nsteps):
    from hackathon_mom6_miniapp_b200 import INIT_CFG, MIXED, Model
    out = []
    for kw in domains:
        m = Model(kw["ni"], kw["nj"], kw["nk"], kw["bt_nsteps"], INIT_CFG, seed=kw["seed"],
                  precision=MIXED, exact=True)
        m.step(nsteps)
        out.append({f: m.get(f) for f in FIELDS})
        m.close()
    return out


def _ensemble(domains, nsteps, tuning=None, autotune=False):
    from hackathon_mom6_miniapp_b200 import Ensemble
    e = Ensemble(domains)
    if tuning:
        e.set_tuning(tuning)
    t = e.autotune(reps=1) if autotune else None
    e.step(nsteps)
    e.synchronize()
    out = [{f: e.get(d, f) for f in FIELDS} for d in range(len(domains))]
    info = {"tuning": e.tuning(), "launches": e.launch_count(), "times": t}
    e.close()
    return out, info


@pytest.mark.gpu
def test_ensemble_domains_equal_single_models():
    ref = _singles(DOMAINS, 3)
    got, info = _ensemble(DOMAINS, 3)
    for d in range(len(DOMAINS)):
        for f in FIELDS:
            assert np.array_equal(got[d][f], ref[d][f]), (d, f, rel_l2(got[d][f], ref[d][f]))


@pytest.mark.gpu
def test_ensemble_results_do_not_depend_on_launch_shapes():
    a, _ = _ensemble(DOMAINS, 2)
    b, info = _ensemble(DOMAINS, 2, tuning=OTHER_TUNING)
    assert info["tuning"] == OTHER_TUNING
    for d in range(len(DOMAINS)):
        for f in FIELDS:
            assert np.array_equal(a[d][f], b[d][f]), (d, f)


@pytest.mark.gpu
def test_autotune_restores_state_and_picks_supported_shapes():
    a, _ = _ensemble(DOMAINS, 2)
    b, info = _ensemble(DOMAINS, 2, autotune=True)
    t = info["tuning"]
    assert 0 <= t["tend_tile"] < 4 and 1 <= t["tend_kc"] <= 16
    assert t["vv_nb"] in (64, 128, 256) and t["vv_ch"] in (2, 4)
    assert t["ppm_nb"] in (128, 256) and t["faces_nb"] in (64, 128, 256)
    assert t["bt_tile"] in (32, 48, 64)
    assert all(v > 0 for v in info["times"].values()), info["times"]
    for d in range(len(DOMAINS)):
        for f in FIELDS:
            assert np.array_equal(a[d][f], b[d][f]), (d, f)


@pytest.mark.gpu
def test_one_launch_per_phase_whatever_the_domain_count():
    _, one = _ensemble(DOMAINS[:1], 2)
    _, four = _ensemble(DOMAINS, 2)
    assert one["launches"] == four["launches"] == 2 * 14


@pytest.mark.gpu
def test_ensemble_rejects_fp64_members():
    from hackathon_mom6_miniapp_b200 import FP64, INIT_CFG, Mom6bError, library
    from hackathon_mom6_miniapp_b200._lib import Config, make_config
    import ctypes
    arr = (Config * 1)()
    arr[0] = make_config(40, 36, 12, 30, INIT_CFG, precision=FP64)
    h = ctypes.c_void_p()
    rc = library().mom6b_ensemble_create(1, arr, ctypes.byref(h))
    assert rc != 0 and not h.value
    assert "mixed" in library().mom6b_last_error().decode()
