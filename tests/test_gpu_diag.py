"""The diagnostics module (mom6_diag.F90) on device fields, and field dumps.

The driver's diagnostics (rk2_serial_driver.F90 with diag_mode = 1: diffu_sum
and diffv_sum after every predictor, KE and mass after the last iteration)
are compared with the oracle bit for bit through the files the posts write;
the statistics lines with the same statistics formed in the serial loop's
order; the generic posts, the output frequency, the shared work array of
the product sums, the 100-field limit and the checkpoint dumps against the
model's own fields."""
import math

import numpy as np
import pytest

from hackathon_mom6_miniapp_b200.diag_format import dump_name, read_bin, stats_line

NONE, STATS, FILE, BOTH = 0, 1, 2, 3
ARGS = (40, 30, 6, 30)


def _model(**kw):
    from hackathon_mom6_miniapp_b200 import INIT_CFG, Model
    return Model(*ARGS, INIT_CFG, seed=kw.pop("seed", 2), **kw, exact=True)


def _comp(m, a):
    """The computational domain of a full (n1, n2[, nk]) array."""
    return a[m.is_ - 1:m.ie, m.js - 1:m.je, ...]


def _stats(a):
    """post_data's min/max/mean/rms, summed in the serial loop's order."""
    flat = np.asarray(a, dtype=np.float64).flatten(order="F").tolist()
    fmin, fmax, s, s2 = math.inf, -math.inf, 0.0, 0.0
    for x in flat:
        fmin = x if x < fmin else fmin
        fmax = x if x > fmax else fmax
        s = s + x
        s2 = s2 + x * x
    n = len(flat)
    return (fmin, fmax, s / n, math.sqrt(s2 / n))


def _lines(out):
    return [ln for ln in out.splitlines() if ln.startswith("  Diag: ")]


@pytest.mark.gpu
def test_driver_diagnostics_match_the_oracle(tmp_path, capfd):
    from oracle.pyoracle import INIT_CFG, Oracle
    m = _model()
    m.diag_init(tmp_path, 1)
    m.diag_driver(BOTH)
    capfd.readouterr()
    m.step(3)
    m.synchronize()
    lines = _lines(capfd.readouterr().out)
    names = ["diffu_sum", "diffv_sum"] * 3 + ["KE", "mass"]
    assert [ln.split()[1] for ln in lines] == names
    o = Oracle(*ARGS, INIT_CFG, seed=2)
    o.diag_enable()
    # the oracle keeps the last post of each field: compare after iterations 1 and 3
    checks = [(1, {1: "diffu_sum", 2: "diffv_sum"}),
              (2, {5: "diffu_sum", 6: "diffv_sum", 7: "KE", 8: "mass"})]
    for nsteps, posts in checks:
        o.step(nsteps)
        for count, name in posts.items():
            got = read_bin(dump_name(tmp_path, name, count))
            want = _comp(o, o.diag_get(name))
            assert got.shape == want.shape, name
            assert np.array_equal(got, want), (name, count, np.abs(got - want).max())
            st = _stats(want)
            assert lines[count - 1] == stats_line(name, st), (lines[count - 1], st)
    assert m.diag_stats(4) == _stats(_comp(o, o.diag_get("mass")))   # id 4 = mass
    assert m.diag_report() == {"registered": 4, "post_calls": 8, "call_count": 8}


@pytest.mark.gpu
def test_driver_diagnostics_leave_the_step_unchanged():
    a, b = _model(), _model()
    b.diag_init("./", 1)
    b.diag_driver(NONE)   # registers nothing active, but runs the diagnostic kernels
    b2 = _model()
    b2.diag_init("./", 1)
    b2.diag_driver(STATS)
    for m in (a, b, b2):
        m.step(2)
    for f in ("u", "v", "h", "eta", "ubt_av"):
        assert np.array_equal(a.get(f), b2.get(f)), f
        assert np.array_equal(a.get(f), b.get(f)), f


@pytest.mark.gpu
def test_posts_frequency_and_inactive_ids(tmp_path, capfd):
    import torch
    m = _model()
    m.diag_init(tmp_path, 2)
    assert m.diag_register("off", "x", "1", 2, "h", NONE) == -1
    i_u = m.diag_register("u3", "u", "m/s", 3, "u", FILE)
    i_e = m.diag_register("eta", "eta", "m", 2, "h", BOTH)
    assert (i_u, i_e) == (1, 2)
    m.diag_post(-1, "eta")                       # inactive: no call counted
    m.diag_post(i_u, "u")                        # call 1: not written (freq 2)
    m.diag_post(i_e, "eta")                      # call 2: written
    t = torch.tensor(np.asfortranarray(m.get("u")).flatten(order="F") * 2.0, device="cuda")
    m.diag_post(i_u, t)                          # call 3: not written
    m.diag_post(i_u, t)                          # call 4: written
    assert not (tmp_path / "u3000001.bin").exists()
    assert not (tmp_path / "u3000003.bin").exists()
    assert np.array_equal(read_bin(dump_name(tmp_path, "eta", 2)), _comp(m, m.get("eta")))
    assert np.array_equal(read_bin(dump_name(tmp_path, "u3", 4)), _comp(m, m.get("u") * 2.0))
    lines = _lines(capfd.readouterr().out)
    assert lines == [stats_line("eta", _stats(_comp(m, m.get("eta"))))]   # only eta has STATS
    assert m.diag_stats(i_u) == _stats(_comp(m, m.get("u") * 2.0))
    assert m.diag_report()["call_count"] == 4


@pytest.mark.gpu
def test_product_sums_share_one_work_array(tmp_path):
    """post_product_sum_u covers I in [is, ie-1], post_product_sum_v J in
    [js, je-1]; both post the whole computational domain of the one work
    array, so a u sum after a v sum carries the v sum's last column."""
    m = _model()
    m.diag_init(tmp_path, 1)
    iu = m.diag_register("us", "u sum", "1", 2, "u", FILE)
    iv = m.diag_register("vs", "v sum", "1", 2, "v", FILE)
    u, v, h = m.get("u"), m.get("v"), m.get("h")
    m.diag_post_product_sum(iv, "v", "h", "v")
    m.diag_post_product_sum(iu, "u", "h", "u")
    is_, ie, js, je = m.is_ - 1, m.ie, m.js - 1, m.je
    want_v = np.zeros(u.shape[:2])
    want_v[is_:ie, js:je - 1] = (v * h).sum(axis=2)[is_:ie, js:je - 1]
    got_v = read_bin(dump_name(tmp_path, "vs", 1))
    np.testing.assert_allclose(got_v, want_v[is_:ie, js:je], rtol=1e-13, atol=0)
    want_u = want_v.copy()
    want_u[is_:ie - 1, js:je] = (u * h).sum(axis=2)[is_:ie - 1, js:je]
    got_u = read_bin(dump_name(tmp_path, "us", 2))
    np.testing.assert_allclose(got_u, want_u[is_:ie, js:je], rtol=1e-13, atol=0)
    # the last column of the u post is the v sum's
    assert np.array_equal(got_u[-1, :], got_v[-1, :])


@pytest.mark.gpu
def test_field_limit(capfd):
    m = _model()
    m.diag_init("./", 1)
    ids = [m.diag_register(f"d{q}", "x", "1", 2, "h", STATS) for q in range(100)]
    assert ids == list(range(1, 101))
    assert m.diag_register("extra", "x", "1", 2, "h", STATS) == -1
    assert "WARNING: Maximum diagnostics reached:  100" in capfd.readouterr().out


@pytest.mark.gpu
def test_checkpoint_dump_and_restore(tmp_path):
    from hackathon_mom6_miniapp_b200 import Mom6bError
    m = _model()
    m.step(1)
    h, eta = m.get("h"), m.get("eta")
    m.write_field_bin("h", tmp_path / "h.bin")
    m.write_field_bin("eta", tmp_path / "eta.bin")
    assert np.array_equal(read_bin(tmp_path / "h.bin"), _comp(m, h))
    assert np.array_equal(read_bin(tmp_path / "eta.bin"), _comp(m, eta))
    m.set("h", np.zeros_like(h))
    m.set("eta", np.zeros_like(eta))
    m.read_field_bin("h", tmp_path / "h.bin")
    m.read_field_bin("eta", tmp_path / "eta.bin")
    h2, eta2 = m.get("h"), m.get("eta")
    assert np.array_equal(_comp(m, h2), _comp(m, h))
    assert np.array_equal(_comp(m, eta2), _comp(m, eta))
    with pytest.raises(Mom6bError):
        m.read_field_bin("h", tmp_path / "eta.bin")   # a 2-D dump into a 3-D field
