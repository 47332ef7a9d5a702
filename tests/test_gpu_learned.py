"""The learned regrid: the forecaster's samples taken from the solver, the
network trained on the reference criterion's flags 16 steps ahead, and the
regrid every 32 steps with the forecast and the criterion as its fallback,
against the criterion alone at the same interval. No reference counterpart:
the reference regrids every step from the current field
(Refine_Derefine.f90:18-54, 327-351)."""
import json
import os

import numpy as np
import pytest

import amrlbm
from amrlbm import AmrLbm, Net
from parity import assert_physical

pytestmark = pytest.mark.gpu
OUT = os.environ.get("AMRLBM_LEARNED_REPORT")


def _sim(seed, regrid_every=32, refin_tol=5e-2):
    """Six bubbles rising fast (density ratio 10, velocity scale sqrt(Gy D)
    ~ 0.03) against a narrow refined band (refine tolerance 5e-2: only the
    interface's core refines)."""
    p, bubbles = amrlbm.learned_workload(128, 256, 3, 6, seed=seed, rmin=16.0, rmax=32.0,
                                         regrid_every=regrid_every, rho_ratio=10.0,
                                         visc_ratio=10.0, eo=10.0, ar=amrlbm.archimedes(10.0, 1e-3),
                                         gy=2e-5, refin_tol=refin_tol, deref_tol=refin_tol / 2)
    g = AmrLbm(p)
    g.set_bubbles(bubbles)
    g.initialize_rising_bubble()
    return g


def test_features_are_the_fields():
    g = _sim(3)
    g.main_loop(32)
    ids = g.leaves()[:5]
    x = g.block_features(ids, 16.0)
    t = g.topology()
    for i, b in enumerate(ids):
        f = g.download_block(int(b))
        C = f["C"]  # (-1:18, -1:18)
        dx = float(t["dx"][b - 1])
        assert np.array_equal(x[i, 0], C[1:19, 1:19].T.astype(np.float32))
        gx = C[2:20, 1:19] - C[0:18, 1:19]
        gy = C[1:19, 2:20] - C[1:19, 0:18]
        e = np.log1p(np.sqrt(gx ** 2 + gy ** 2) / (2 * dx) / g.params.refin_tol)
        assert np.allclose(x[i, 1], e.T, rtol=1e-6, atol=1e-6)
        assert np.allclose(x[i, 2, 1:17, 1:17], (f["Ux"] * 16.0 / dx).T, rtol=1e-6, atol=1e-12)
        assert np.all(x[i, 3, 0] == 0) and np.all(x[i, 3, :, 17] == 0)
    g.close()


def test_learned_regrid_flags_fewer_escapes_than_the_criterion_alone():
    """Regrids 256 steps apart, forecast horizon 128: with 16x16 blocks the
    refined region holds the interface for tens of steps (at the default
    interval of 32 the criterion flags almost nothing), so the interval is
    long enough here for the interface to leave refined blocks between
    regrids. An escape is a leaf the criterion flags at a regrid: the
    interface has been on it at a coarse level since the last one. Trained on
    three seeded runs, evaluated on a fourth."""
    R, H = 256, 128
    xs, ys, seen, pos = [], [], 0, 0
    for seed in (11, 12, 13):
        g = _sim(seed, regrid_every=R)
        x, y, c = amrlbm.collect_samples(g, regrids=20, horizon=H)
        g.close()
        xs.append(x)
        ys.append(y)
        seen, pos = seen + c["samples"], pos + c["positives"]
    x, y = np.concatenate(xs), np.concatenate(ys)
    net = Net(seed=7, max_batch=512)
    losses = amrlbm.train_net(net, x, y, epochs=20, batch=128, lr=2e-3)
    z = net.forward(x.astype(np.float32))
    recall = float(((z > 0) & (y > 0)).sum() / max(y.sum(), 1))
    # the criterion alone, counted the same way: a forecaster that never fires
    never = Net(seed=7, max_batch=512)
    p = never.params()
    p[-1] = -1e4  # output bias: probability 0
    never.set_params(p)
    res = {}
    for name, n in (("criterion", never), ("learned", net)):
        s = _sim(23, regrid_every=R)
        s.set_regrid_net(n, horizon=float(H), threshold=0.5)
        s.main_loop(R * 16)
        res[name] = s.regrid_stats()
        res[name]["leaves"] = s.counts()["nleaf"]
        assert_physical(s.output(), 0.1, name)
        s.close()
    report = {"samples": seen, "positives": pos, "losses": losses, "train_recall": recall,
              "criterion_only": res["criterion"], "learned": res["learned"]}
    if OUT:
        with open(OUT, "w") as f:
            json.dump(report, f, indent=1)
    print(json.dumps(report))
    assert losses[-1] < losses[0] and recall > 0.5
    assert res["learned"]["regrids"] == res["criterion"]["regrids"] == 16
    assert res["criterion"]["flagged"] > 0
    assert res["learned"]["flagged"] < res["criterion"]["flagged"]
    assert res["learned"]["missed"] <= res["learned"]["flagged"]
    net.close()
    never.close()
