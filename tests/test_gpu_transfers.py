"""Field transfers through the C ABI: amrlbm_upload_fields / amrlbm_download_fields
(batched, the caller's arrays in the reference's layouts, h, g(9, 0:nx+1,
0:ny+1), C(-1:nx+2, -1:ny+2), P, Ux, Uy(nx, ny)) and amrlbm_upload_block /
amrlbm_download_block (one block). These replace the reference's direct reads
and writes of Blk(n)%h, %g, %C, %P, %Ux, %Uy (Parameters.f90:23-39).

Round trips are bit for bit on ragged requests (none, one block, a reversed
subset with gaps, every leaf); the batched and per-block entry points agree;
fields left out of an upload keep their values; ids outside the pool are
rejected with an error and change nothing; a non-finite value uploaded into
a leaf is reported by the diagnostics."""
import numpy as np
import pytest

import amrlbm
from amrlbm import AmrLbm, AmrLbmError

pytestmark = pytest.mark.gpu

FIELDS = ("h", "g", "C", "P", "Ux", "Uy")


def _started(steps=0):
    sim = AmrLbm(amrlbm.workload_small())
    sim.initialize_rising_bubble()
    if steps:
        sim.main_loop(steps)
    sim.sync()
    return sim


def _subset(ids, pick):
    return {"none": ids[:0],
            "one": ids[len(ids) // 2:len(ids) // 2 + 1],
            "reversed_with_gaps": ids[1::3][::-1],
            "all": ids}[pick]


def test_batched_and_per_block_downloads_agree():
    with _started(steps=3) as sim:
        sel = sim.leaves()[::-1][:7]
        f = sim.download_fields(sel)
        for r, bid in enumerate(sel):
            b = sim.download_block(int(bid))
            for k in FIELDS:
                assert np.array_equal(f[k][r], b[k].ravel(order="F")), (k, int(bid))


@pytest.mark.parametrize("pick", ["none", "one", "reversed_with_gaps", "all"])
def test_upload_download_round_trip(pick):
    with _started() as sim:
        ids = sim.leaves()
        sel = _subset(ids, pick)
        before = sim.download_fields(ids)
        rng = np.random.default_rng(20261203)
        new = {k: rng.standard_normal((len(sel), v.shape[1])) for k, v in before.items()}
        sim.upload_fields(sel, new)
        after = sim.download_fields(ids)
        row = {int(b): i for i, b in enumerate(ids)}
        chosen = {int(b) for b in sel}
        for k in FIELDS:
            for r, bid in enumerate(sel):
                assert np.array_equal(after[k][row[int(bid)]], new[k][r]), (k, int(bid))
            for bid in ids:
                if int(bid) not in chosen:
                    assert np.array_equal(after[k][row[int(bid)]], before[k][row[int(bid)]])


def test_upload_of_some_fields_keeps_the_others():
    with _started(steps=2) as sim:
        ids = sim.leaves()
        sel = ids[::2]
        before = sim.download_fields(ids)
        rng = np.random.default_rng(7)
        newC = rng.standard_normal((len(sel), before["C"].shape[1]))
        newUy = rng.standard_normal((len(sel), before["Uy"].shape[1]))
        sim.upload_fields(sel, {"C": newC, "Uy": newUy})
        after = sim.download_fields(ids)
        row = {int(b): i for i, b in enumerate(ids)}
        for r, bid in enumerate(sel):
            i = row[int(bid)]
            assert np.array_equal(after["C"][i], newC[r])
            assert np.array_equal(after["Uy"][i], newUy[r])
            for k in ("h", "g", "P", "Ux"):
                assert np.array_equal(after[k][i], before[k][i]), (k, int(bid))


def test_per_block_upload_round_trip():
    with _started(steps=1) as sim:
        bid = int(sim.leaves()[-1])
        b = sim.download_block(bid)
        rng = np.random.default_rng(11)
        new = {k: rng.standard_normal(v.shape) for k, v in b.items()}
        sim.upload_block(bid, **new)
        got = sim.download_block(bid)
        for k in FIELDS:
            assert np.array_equal(got[k], new[k]), k


def test_ids_outside_the_pool_are_rejected():
    with _started() as sim:
        ids = sim.leaves()
        before = sim.download_fields(ids)
        csize = before["C"].shape[1]
        for bad in (0, -1, sim.params.max_blks + 1):
            with pytest.raises(AmrLbmError):
                sim.download_fields(np.array([int(ids[0]), bad], dtype=np.int32))
            with pytest.raises(AmrLbmError):
                sim.upload_fields(np.array([int(ids[0]), bad], dtype=np.int32),
                                  {"C": np.ones((2, csize))})
        after = sim.download_fields(ids)
        for k in FIELDS:
            assert np.array_equal(after[k], before[k]), k


def test_non_finite_field_is_reported_by_the_diagnostics():
    """Output (AMR_Rising_2D_OMP.f90:456-489) on a state with a NaN in C or
    an infinite Uy in one leaf interior: AMRLBM_ERR_NAN instead of numbers;
    a finite state again reports normally."""
    with _started(steps=1) as sim:
        sim.output()
        bid = int(sim.leaves()[3])
        b = sim.download_block(bid)
        for field, bad in (("C", np.nan), ("Uy", np.inf)):
            a = b[field].copy()
            a[2, 2] = bad
            sim.upload_block(bid, **{field: a})
            with pytest.raises(AmrLbmError) as e:
                sim.output()
            assert e.value.status == amrlbm.ERR_NAN
            sim.upload_block(bid, **{field: b[field]})
            sim.output()
