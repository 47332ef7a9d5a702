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


@pytest.mark.parametrize("precision", ["fp64", "fp16"])
def test_fused_forecast_equals_the_network(precision):
    """The learned regrid's fused kernel (features from the pool, three
    convolutions on the tensor cores, max pool, dense output in one launch)
    gives the unfused network's logits on the same samples: bit for bit in
    FP64 storage; with FP16 storage it reads the FP32 fields, so the samples
    (and logits) differ from the FP64 copy's by storage rounding only."""
    g = _sim(4)
    g.main_loop(40)
    net = Net(seed=5, max_batch=256)
    p = net.params()
    rng = np.random.default_rng(9)
    p[:] = p + 0.05 * rng.standard_normal(p.shape).astype(np.float32)
    net.set_params(p)
    g.set_regrid_net(net, horizon=16.0, threshold=0.5)
    if precision != "fp64":
        g.set_precision(precision)
        g.main_loop(4)
    ids = g.leaves()
    z_fused = g.forecast_blocks(ids)
    x = g.block_features(ids, 16.0)
    z_ref = net.forward(x)
    assert np.all(np.isfinite(z_fused)) and np.std(z_ref) > 0
    if precision == "fp64":
        assert np.array_equal(z_fused, z_ref)
    else:
        assert np.allclose(z_fused, z_ref, rtol=2e-2, atol=2e-2 * np.abs(z_ref).max())
    g.set_regrid_net(None)
    g.close()
    net.close()


def test_regrid_statistics_without_a_net():
    """The criterion alone counts its regrids and flagged leaves (every one
    of them an escape: nothing forecast it)."""
    g = _sim(6, regrid_every=64)
    assert g.regrid_stats() == {"regrids": 0, "forecast": 0, "flagged": 0, "missed": 0, "extra": 0}
    g.main_loop(64 * 4)
    st = g.regrid_stats()
    assert st["regrids"] == 4 and st["forecast"] == 0 and st["extra"] == 0
    assert st["missed"] == st["flagged"]
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
    res = {}
    for name, n in (("criterion", None), ("learned", net)):
        s = _sim(23, regrid_every=R)
        if n is not None:
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
