"""Host logic of the single-operator kernel autotuner, without a GPU: the choice rule and the cache
key (stable for the same inputs, different when the batch size, form or candidates change)."""
from __future__ import annotations

import numpy as np


def _op():
    from cf_b200 import geometry
    from cf_b200.operator import CollisionOperator

    class FakeOp:  # the attributes the key reads; no plan, no device
        pass

    geo = geometry.sort_for_contraction(geometry.generate_geometry(2))
    op = FakeOp()
    op.N_Q, op.K, op.n_g, op.n_l, op.device = geo.n_q, 4, geo.n_g, geo.n_l, 0
    op._host_operator = (geo.labels, geo.vals, geo.ic_map, np.zeros(4))
    op.content_digest = lambda: CollisionOperator.content_digest(op)
    return op


def test_choice_rule():
    from cf_b200 import operator

    assert operator.choose_fastest({"auto": 2.0, "gather": 3.0, "lblock": 1.5}) == "lblock"
    assert operator.choose_fastest({"auto": 1.0, "band": 1.0}) == "auto"


def test_cache_key():
    from cf_b200 import operator

    op = _op()
    k = operator._autotune_key(op, 300, "af_sym", operator.AUTOTUNE_PATHS)
    assert k == operator._autotune_key(op, 300, "af_sym", operator.AUTOTUNE_PATHS)
    assert k != operator._autotune_key(op, 301, "af_sym", operator.AUTOTUNE_PATHS)
    assert k != operator._autotune_key(op, 300, "af", operator.AUTOTUNE_PATHS)
    assert k != operator._autotune_key(op, 300, "af_sym", ("auto", "gather"))
