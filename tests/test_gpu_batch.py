"""Batched instances (amrlbm_create_batch): independent rising bubbles of
different sizes, depths and physics in one pool, advanced by the same
launches. Each instance must equal, bit for bit, the same problem run alone
(whose FP64 path is bit for bit with the CPU oracle): the same leaves (matched
by level and block position, since block ids are the pool's) and the same
fields. No reference counterpart: the reference runs one bubble per process."""
import numpy as np
import pytest

import amrlbm
from amrlbm import AmrLbm, Instance
from parity import assert_physical

pytestmark = pytest.mark.gpu

FIELDS = ("h", "g", "C", "P", "Ux", "Uy")


def _instances():
    mk = lambda **k: Instance(**k)
    return [
        # 64x128 base, 2 levels, density ratio 10 (the small workload's physics)
        mk(nbx=4, nby=8, dx0=4, max_levels=2, rho_l=0.1, rho_h=1.0, visc_ratio=10.0, bo=10.0,
           ar=amrlbm.archimedes(10.0, 1e-3), gy=5e-6, w=4.0, m0=0.02, radius=20.0, xc=128.0,
           yc=128.0, hydrostatic_start=1),
        # 32x64 base, 3 levels, density ratio 1000 (the large workload's physics)
        mk(nbx=2, nby=4, dx0=8, max_levels=3, rho_l=0.001, rho_h=1.0, visc_ratio=100.0, bo=10.0,
           ar=100.0, gy=2.5e-7, w=4.0, m0=0.02, radius=24.0, xc=128.0, yc=128.0,
           hydrostatic_start=1),
        # 64x64 base, 1 level, density ratio 100
        mk(nbx=4, nby=4, dx0=2, max_levels=1, rho_l=0.01, rho_h=1.0, visc_ratio=100.0, bo=5.0,
           ar=amrlbm.archimedes(5.0, 1e-4), gy=1e-6, w=4.0, m0=0.02, radius=16.0, xc=64.0,
           yc=40.0, hydrostatic_start=1),
        # the first again with a smaller bubble and the reference's start-up pressure
        mk(nbx=4, nby=8, dx0=4, max_levels=2, rho_l=0.1, rho_h=1.0, visc_ratio=10.0, bo=10.0,
           ar=amrlbm.archimedes(10.0, 1e-3), gy=5e-6, w=4.0, m0=0.02, radius=14.0, xc=100.0,
           yc=140.0, hydrostatic_start=0),
    ]


def _by_position(sim, inst=None, which=None):
    """{(level, I, J): fields} of the leaves (of instance `which` in a batch)."""
    ids = np.asarray(sim.leaves(), dtype=np.int32)
    t = sim.topology()
    if inst is not None:
        ids = ids[inst[ids - 1] == which]
    f = sim.download_fields(ids)
    out = {}
    for i, b in enumerate(ids):
        key = (int(t["level"][b - 1]), int(t["bi"][b - 1]), int(t["bj"][b - 1]))
        out[key] = [f[k][i] for k in FIELDS]
    return out


def _compare(batch, alone, which):
    inst = batch.block_instances()
    a = _by_position(batch, inst, which)
    b = _by_position(alone)
    assert sorted(a) == sorted(b), f"instance {which}: leaf sets differ"
    for key in b:
        for k, x, y in zip(FIELDS, a[key], b[key]):
            assert np.array_equal(x, y), f"instance {which} leaf {key} field {k}"


@pytest.mark.parametrize("regrid_every", [1, 5])
def test_batch_instances_equal_their_runs_alone(regrid_every):
    insts = _instances()
    bp = amrlbm.batch_params(n=16, max_blks=sum(amrlbm.tree_blocks(i.nbx, i.nby, i.max_levels)
                                                 for i in insts),
                             regrid_every=regrid_every)
    steps = 40
    with AmrLbm(bp, instances=insts) as batch:
        batch.initialize_rising_bubble()
        alone = []
        for i, ins in enumerate(insts):
            g = AmrLbm(ins.params(bp))
            g.initialize_rising_bubble()
            _compare(batch, g, i)
            alone.append(g)
        batch.main_loop(steps)
        diag = batch.output_instances()
        for i, g in enumerate(alone):
            g.main_loop(steps)
            _compare(batch, g, i)
            d = g.output()
            for k in d:
                assert abs(diag[i][k] - d[k]) <= 1e-12 * max(1.0, abs(d[k])), (i, k)
            assert_physical(d, 0.05, f"instance {i}")
            g.close()


def test_batch_in_mixed_precision():
    """The same batch in FP16 storage: every instance stays physical and close
    to its FP64 trajectory."""
    insts = _instances()
    bp = amrlbm.batch_params(n=16, max_blks=sum(amrlbm.tree_blocks(i.nbx, i.nby, i.max_levels)
                                                 for i in insts), regrid_every=5)
    with AmrLbm(bp, instances=insts) as a, AmrLbm(bp, instances=insts) as b:
        for g in (a, b):
            g.initialize_rising_bubble()
        b.set_precision("fp16")
        a.main_loop(200)
        b.main_loop(200)
        for i, (da, db) in enumerate(zip(a.output_instances(), b.output_instances())):
            assert_physical(db, 0.05, f"instance {i}")
            assert abs(db["mass"] - da["mass"]) <= 1e-6 * da["mass"], i
            assert abs(db["y_centroid"] - da["y_centroid"]) <= 0.05, i


def test_launch_shape_does_not_change_results():
    """The CTAs-per-SM cap the autotuner sweeps changes the schedule, not the
    bits: two FP16 batches, one capped at 1 CTA per SM, stay identical."""
    insts = _instances()
    bp = amrlbm.batch_params(n=16, max_blks=sum(amrlbm.tree_blocks(i.nbx, i.nby, i.max_levels)
                                                 for i in insts), regrid_every=5)
    with AmrLbm(bp, instances=insts) as a, AmrLbm(bp, instances=insts) as b:
        for g in (a, b):
            g.initialize_rising_bubble()
            g.set_precision("fp16")
        b.set_launch(1)
        a.main_loop(30)
        b.main_loop(30)
        ids = a.leaves()
        assert np.array_equal(ids, b.leaves())
        fa, fb = a.download_fields(ids), b.download_fields(ids)
        for k in FIELDS:
            assert np.array_equal(fa[k], fb[k]), k


def test_autotune_reports_every_candidate():
    insts = _instances()[:2]
    best, table = amrlbm.autotune(insts, "fp16", block_sizes=(16, 8), ctas=(0, 1), warmup=1,
                                  intervals=1, regrid_every=5)
    assert len(table) == 4 and all(r["mlups"] > 0 for r in table)
    assert best == max(table, key=lambda r: r["mlups"])
