"""amrlbm_download_fields_noalloc (the download that stages through a fixed
per-device scratch area instead of buffers it allocates) against
amrlbm_download_fields, through the C ABI. Kept in its own file, collected
last, so that it runs both alone and after every other GPU test."""
import ctypes as ct

import numpy as np
import pytest

import amrlbm
from amrlbm import AmrLbm

pytestmark = pytest.mark.gpu

FIELDS = ("h", "g", "C", "P", "Ux", "Uy")
ERR_CAPACITY = 9
STAGE_DOUBLES = 524288
MAX_BLOCKS = 16384


def _bind(lib):
    f = lib.amrlbm_download_fields_noalloc
    f.restype = ct.c_int
    f.argtypes = [ct.c_void_p, ct.c_int32, ct.POINTER(ct.c_int32)] + [ct.POINTER(ct.c_double)] * 6
    return f


def _ptr(a, t):
    return None if a is None else a.ctypes.data_as(ct.POINTER(t))


def _noalloc(sim, ids, fields=FIELDS):
    ids = np.ascontiguousarray(ids, dtype=np.int32)
    n = len(ids)
    size = dict(h=int(np.prod(sim.hshape)), g=int(np.prod(sim.hshape)), C=int(np.prod(sim.cshape)),
                P=int(np.prod(sim.pshape)), Ux=int(np.prod(sim.pshape)), Uy=int(np.prod(sim.pshape)))
    out = {k: (np.full((n, size[k]), np.nan) if k in fields else None) for k in FIELDS}
    rc = _bind(sim.lib)(sim.ctx, n, _ptr(ids, ct.c_int32), *[_ptr(out[k], ct.c_double) for k in FIELDS])
    return rc, out


def _same(a, b):
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


def test_noalloc_download_matches_download_fields():
    p = amrlbm.workload_small()
    with AmrLbm(p) as sim:
        sim.initialize_rising_bubble()
        sim.main_loop(3)
        leaves = np.asarray(sim.leaves(), dtype=np.int32)
        # two calls in a row, on different blocks and after further steps
        for ids in (leaves[:7], None):
            if ids is None:
                sim.main_loop(2)
                leaves = np.asarray(sim.leaves(), dtype=np.int32)
                ids = leaves[::-1][:11]
            ref = sim.download_fields(ids)
            rc, out = _noalloc(sim, ids)
            assert rc == 0, sim.lib.amrlbm_last_error(sim.ctx)
            for k in FIELDS:
                assert _same(out[k], ref[k]), k
        # some fields only (NULL pointers for the rest)
        ref = sim.download_fields(leaves[:3])
        rc, out = _noalloc(sim, leaves[:3], fields=("g", "Uy"))
        assert rc == 0
        assert _same(out["g"], ref["g"]) and _same(out["Uy"], ref["Uy"])


def test_noalloc_download_rejects_oversize_requests():
    p = amrlbm.workload_small()
    with AmrLbm(p) as sim:
        sim.initialize_rising_bubble()
        leaf = int(sim.leaves()[0])
        per_block = 2 * int(np.prod(sim.hshape)) + int(np.prod(sim.cshape)) + 3 * int(np.prod(sim.pshape))
        n = STAGE_DOUBLES // per_block + 1
        rc, out = _noalloc(sim, np.full(n, leaf, dtype=np.int32))
        assert rc == ERR_CAPACITY
        assert all(np.isnan(out[k]).all() for k in FIELDS)  # nothing ran
        # the largest request that fits still works
        n = STAGE_DOUBLES // per_block
        ids = np.full(n, leaf, dtype=np.int32)
        rc, out = _noalloc(sim, ids)
        assert rc == 0
        ref = sim.download_fields(ids[:1])
        for k in FIELDS:
            assert _same(out[k][-1:], ref[k]), k


def test_noalloc_download_rejects_too_many_blocks():
    """The block-count limit on its own: with 4x4 blocks, MAX_BLOCKS + 1 blocks
    of one 16-double field fit in the stage, so only the block limit refuses
    the request."""
    p = amrlbm.bubble_params(32, 64, 1, radius=8.0, xc=16.0, yc=24.0, rho_ratio=10.0,
                             visc_ratio=10.0, eo=10.0, mo=1e-3, n=4)
    with AmrLbm(p) as sim:
        sim.initialize_rising_bubble()
        leaf = int(sim.leaves()[0])
        assert (MAX_BLOCKS + 1) * int(np.prod(sim.pshape)) <= STAGE_DOUBLES
        rc, out = _noalloc(sim, np.full(MAX_BLOCKS + 1, leaf, dtype=np.int32), fields=("Uy",))
        assert rc == ERR_CAPACITY
        assert np.isnan(out["Uy"]).all()  # nothing ran
        rc, out = _noalloc(sim, np.full(MAX_BLOCKS, leaf, dtype=np.int32), fields=("Uy",))
        assert rc == 0
        ref = sim.download_fields(np.array([leaf], dtype=np.int32))
        assert _same(out["Uy"][-1:], ref["Uy"]) and _same(out["Uy"][:1], ref["Uy"])


def test_noalloc_download_reports_a_device_error_once():
    """A pending device error status is returned by the next call and then
    cleared, as amrlbm_download_fields does. amrlbm_step does not synchronise,
    so a level jump planted in the neighbour table (a finest leaf whose left
    neighbour pointer names a leaf two levels coarser) leaves its status on
    the device for the download to find."""
    p = amrlbm.bubble_params(16, 32, 3, radius=10.0, xc=64.0, yc=80.0, rho_ratio=1000.0,
                             visc_ratio=100.0, eo=10.0, mo=1e-5, n=8, regrid_every=1000)
    with AmrLbm(p) as sim:
        sim.initialize_rising_bubble()
        t = sim.topology()
        lv = t["level"]
        leaves = np.asarray(sim.leaves())
        deep = [int(b) for b in leaves if lv[b - 1] == lv.max()]
        coarse = [int(b) for b in leaves if lv[b - 1] <= lv.max() - 2]
        assert deep and coarse
        t["nbr_owner"][deep[0] - 1, 0] = coarse[0]
        t["nbr_slot"][deep[0] - 1, 0] = 0
        sim.set_topology(t, sim.counts()["kk"])
        assert sim.lib.amrlbm_step(sim.ctx, 1) == 0
        ids = np.array([deep[0]], dtype=np.int32)
        rc1, _ = _noalloc(sim, ids, fields=("P",))
        rc2, out = _noalloc(sim, ids, fields=("P",))
        assert rc1 == amrlbm.ERR_LEVEL_JUMP
        assert rc2 == 0
        assert _same(out["P"], sim.download_fields(ids)["P"])
