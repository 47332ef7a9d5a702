"""The three layers together: a batch of uneven instances with FP16 storage
and the learned regrid inside the step's graph, against the plain FP64 path
of the same batch with the reference's criterion (Refine_Derefine.f90:18-54,
327-351) every 10 steps. No reference counterpart."""
import numpy as np
import pytest

import amrlbm
from amrlbm import AmrLbm, Net

pytestmark = pytest.mark.gpu


def _run(insts, precision, every, net, steps):
    g = AmrLbm(amrlbm.batch_params(n=16, max_blks=60000, regrid_every=every), instances=insts)
    g.initialize_rising_bubble()
    if precision != "fp64":
        g.set_precision(precision)
    if net is not None:
        g.set_regrid_net(net, horizon=16.0, threshold=0.5)
    g.main_loop(steps)
    d = g.output_instances()
    st = g.regrid_stats()
    g.close()
    return d, st


def test_fp16_batch_with_learned_regrid_against_fp64():
    """16 seeded instances, 160 steps. The forecaster has seeded weights with
    the output bias set so that it forecasts some leaves and not others; the
    regrid statistics must add up, every instance must stay physical, and
    each instance's mass must stay within 1e-5 and its rise velocity within
    5 % of the FP64 run (different regrid intervals give different meshes,
    so the two runs are not the same discretisation)."""
    insts = amrlbm.batch_instances(16)
    steps = 160
    d64, s64 = _run(insts, "fp64", 10, None, steps)
    net = Net(seed=3, max_batch=64)
    p = net.params()
    p[-1] = -2.0
    net.set_params(p)
    d16, s16 = _run(insts, "fp16", 32, net, steps)
    net.close()
    assert s64["regrids"] == steps // 10 and s16["regrids"] == steps // 32
    assert s64["forecast"] == 0 and s64["missed"] == s64["flagged"]
    assert s16["missed"] <= s16["flagged"]
    assert s16["forecast"] - s16["extra"] == s16["flagged"] - s16["missed"]
    for i, (a, b) in enumerate(zip(d64, d16)):
        for x in (a, b):
            assert np.isfinite(x["mass"]) and x["u_max"] < 0.05 and x["rho_min"] > 0, i
        assert abs(b["mass"] - a["mass"]) <= 1e-5 * abs(a["mass"]), i
        assert abs(b["rise_velocity"] - a["rise_velocity"]) <= 0.05 * abs(a["rise_velocity"]) + 1e-7, i
