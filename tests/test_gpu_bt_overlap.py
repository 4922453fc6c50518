"""The barotropic chain on its own stream (Model.set_bt_overlap): the step is
unchanged bit for bit, eagerly and from the captured graph, both forms."""
import numpy as np
import pytest

from oracle.pyoracle import INIT_CFG, Oracle

FIELDS = ["u", "v", "h", "eta", "ubt_av", "vbt_av", "eta_av"]


@pytest.mark.gpu
@pytest.mark.parametrize("use_graph", [False, True])
def test_overlapped_steps_match_the_oracle(use_graph):
    from hackathon_mom6_miniapp_b200 import Model
    m = Model(48, 36, 6, 30, INIT_CFG, seed=3, use_graph=use_graph, exact=True)
    m.set_bt_overlap(True)
    o = Oracle(48, 36, 6, 30, INIT_CFG, seed=3)
    m.step(4)
    o.step(4)
    for f in FIELDS:
        assert np.array_equal(m.get(f), o.get(f)), f


@pytest.mark.gpu
def test_overlap_leaves_the_mixed_form_unchanged():
    from hackathon_mom6_miniapp_b200 import MIXED, Model
    a = Model(48, 36, 6, 30, INIT_CFG, seed=4, precision=MIXED, exact=True)
    b = Model(48, 36, 6, 30, INIT_CFG, seed=4, precision=MIXED, exact=True)
    b.set_bt_overlap(True)
    a.step(3)
    b.step(3)
    for f in FIELDS:
        assert np.array_equal(a.get(f), b.get(f)), f
