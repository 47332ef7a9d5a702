"""Parity of the B200 path with the CPU oracle, through the C ABI.

Every test runs the same inputs through libamrlbm.so (amrlbm.AmrLbm) and the
oracle and requires identical integer state and identical FP64 fields
(tolerance 0: the FP64 path's stated bound is 1e-12 relative; the device path
meets it exactly because it keeps the reference's operation order without
FMA).
"""
import numpy as np
import pytest

import amrlbm
from amrlbm import AmrLbm, AmrLbmError
from oracle_lib import Oracle
from parity import (compare_counts, compare_fields, compare_state, compare_topology,
                    copy_state_to_gpu, randomize_leaves)

pytestmark = pytest.mark.gpu


def tiny_params(**kw):
    """Small rising bubble with 8x8 blocks: 2x4 base blocks, 3 levels."""
    p = amrlbm.bubble_params(16, 32, 3, radius=10.0, xc=64.0, yc=80.0, rho_ratio=1000.0,
                             visc_ratio=100.0, eo=10.0, mo=1e-5, n=8, regrid_every=1)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


CASES = {
    "reference_default": amrlbm.reference_params,
    "tiny_minlevels0": tiny_params,
    "small_16x16": amrlbm.workload_small,
}


@pytest.mark.parametrize("case", list(CASES))
def test_init_parity(case):
    p = CASES[case]()
    orc = Oracle(p)
    orc.initialize_rising_bubble()
    with AmrLbm(p) as gpu:
        gpu.initialize_rising_bubble()
        compare_state(gpu, orc)


@pytest.mark.parametrize("case", list(CASES))
def test_phase_by_phase(case):
    """Main_Loop call sites one by one (AMR_Rising_2D_OMP.f90:304-360)."""
    p = CASES[case]()
    orc = Oracle(p)
    orc.initialize_rising_bubble()
    with AmrLbm(p) as gpu:
        gpu.initialize_rising_bubble()
        for step in range(3):
            assert gpu.determine_min_max_levels() == orc.determine_min_max_levels()
            orc.fill_ghost_cells_c2()
            gpu.fill_ghost_cells_c2()
            compare_fields(gpu, orc, fields=("C",))
            orc.phase_field_lbm_h_g()
            gpu.phase_field_lbm_h_g()
            compare_fields(gpu, orc, fields=("h", "g"))
            orc.macroscopic_values_h()
            gpu.macroscopic_values_h()
            compare_fields(gpu, orc, fields=("C",))
            orc.fill_ghost_cells_c()
            gpu.fill_ghost_cells_c()
            compare_fields(gpu, orc, fields=("C",))
            orc.macroscopic_values_g()
            gpu.macroscopic_values_g()
            compare_fields(gpu, orc, fields=("P", "Ux", "Uy"))
            errs = gpu.block_errors()
            for bid in orc.leaves():
                assert errs[bid - 1] == orc.block_error(int(bid))
            orc.refine_derefine_mesh()
            gpu.refine_derefine_mesh()
            compare_state(gpu, orc)


@pytest.mark.parametrize("case,regrid_every,nsteps", [
    ("reference_default", 1, 12),
    ("tiny_minlevels0", 1, 15),
    ("tiny_minlevels0", 4, 13),
    ("small_16x16", 3, 10),
])
def test_main_loop_parity(case, regrid_every, nsteps):
    """amrlbm_step (fused, graph-captured) against the oracle's Main_Loop body."""
    p = CASES[case]()
    p.regrid_every = regrid_every
    orc = Oracle(p)
    orc.initialize_rising_bubble()
    with AmrLbm(p) as gpu:
        gpu.initialize_rising_bubble()
        orc.main_loop(nsteps)
        gpu.main_loop(nsteps)
        gpu.sync()
        compare_state(gpu, orc)
        # a second call continues the same trajectory
        orc.main_loop(5)
        gpu.main_loop(5)
        gpu.sync()
        compare_state(gpu, orc)


def test_random_fields_all_branches():
    """Random C outside [0,1] (both tau clamps), random P, U, h, g on a
    3-level mesh; every phase and the regrid must agree."""
    p = tiny_params()
    orc = Oracle(p)
    orc.initialize_rising_bubble()
    randomize_leaves(orc, seed=20261203)
    with AmrLbm(p) as gpu:
        copy_state_to_gpu(orc, gpu)
        compare_state(gpu, orc)
        orc.fill_ghost_cells_c2()
        gpu.fill_ghost_cells_c2()
        compare_fields(gpu, orc, fields=("C",))
        orc.phase_field_lbm_h_g()
        gpu.phase_field_lbm_h_g()
        compare_fields(gpu, orc, fields=("h", "g"))
        for f in ("macroscopic_values_h", "fill_ghost_cells_c", "macroscopic_values_g"):
            getattr(orc, f)()
            getattr(gpu, f)()
        compare_fields(gpu, orc)
        orc.refine_derefine_mesh()
        gpu.refine_derefine_mesh()
        compare_state(gpu, orc)


def test_diagnostics_match():
    p = tiny_params()
    orc = Oracle(p)
    orc.initialize_rising_bubble()
    with AmrLbm(p) as gpu:
        gpu.initialize_rising_bubble()
        orc.main_loop(7)
        gpu.main_loop(7)
        a, b = gpu.output(), orc.output()
        for k in a:
            assert a[k] == b[k], (k, a[k], b[k])


def test_pool_full_is_reported():
    """Add_Child_Blocks STOP (AMR_Rising_2D_OMP.f90:527-531) -> status code."""
    p = tiny_params(max_blks=20)
    orc = Oracle(p)
    with pytest.raises(AssertionError):
        orc.initialize_rising_bubble()
    assert orc.error() == amrlbm.ERR_POOL_FULL
    with AmrLbm(p) as gpu:
        with pytest.raises(AmrLbmError) as ei:
            gpu.initialize_rising_bubble()
        assert ei.value.status == amrlbm.ERR_POOL_FULL


def test_level_jump_is_reported():
    """A leaf whose neighbour is two levels coarser: the reference prints
    "Error in SUB_Fill_*" and leaves the ghost cells; the device reports
    AMRLBM_ERR_LEVEL_JUMP and leaves them too."""
    p = tiny_params()
    orc = Oracle(p)
    orc.initialize_rising_bubble()
    t = orc.topology()
    lv = t["level"]
    leaves = orc.leaves()
    deep = [b for b in leaves if lv[b - 1] == lv.max()]
    coarse = [b for b in leaves if lv[b - 1] <= lv.max() - 2]
    assert deep and coarse
    b = deep[0]
    t["nbr_owner"][b - 1, 0] = coarse[0]   # left neighbour pointer -> constant coarse id
    t["nbr_slot"][b - 1, 0] = 0
    orc.set_topology(t, orc.counts()["kk"])
    with AmrLbm(p) as gpu:
        copy_state_to_gpu(orc, gpu)
        orc.fill_ghost_cells_c2()
        assert orc.level_jumps() > 0
        with pytest.raises(AmrLbmError) as ei:
            gpu.fill_ghost_cells_c2()
        assert ei.value.status == amrlbm.ERR_LEVEL_JUMP
        compare_fields(gpu, orc, fields=("C",))


def test_large_workload_topology_and_fields():
    """The 256x512-base, 3-level, R=128 workload at full size: start-up and
    20 steps with a regrid every 10."""
    p = amrlbm.workload_large()
    orc = Oracle(p)
    orc.initialize_rising_bubble()
    with AmrLbm(p) as gpu:
        gpu.initialize_rising_bubble()
        compare_state(gpu, orc)
        orc.main_loop(20)
        gpu.main_loop(20)
        gpu.sync()
        compare_counts(gpu, orc)
        compare_topology(gpu, orc)
        compare_fields(gpu, orc)


@pytest.mark.parametrize("name", ["reference_default", "small_16x16"])
def test_device_matches_golden_fixtures(name):
    """The device path against the committed fixtures of tests/golden/
    (start-up state and the state after a few time steps, bit for bit)."""
    import json
    import os
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(here, "golden"))
    from make_golden import CASES, snapshot
    with open(os.path.join(here, "golden", f"oracle_{name}.json")) as f:
        want = json.load(f)
    factory, steps = CASES[name]
    p = factory()
    with AmrLbm(p) as gpu:
        gpu.initialize_rising_bubble()
        assert snapshot(gpu, p) == want["init"]
        gpu.main_loop(steps)
        assert snapshot(gpu, p) == want["after_steps"]


@pytest.mark.parametrize("case", ["reference_default", "small_16x16"])
@pytest.mark.parametrize("narrow", ["finest_out", "coarsest_out"])
def test_level_range_narrower_than_the_leaves(case, narrow):
    """Fills over a level range that leaves some leaves out (the reference's
    DO L = LevelMin, LevelMax with a narrower range): those leaves keep their
    ghost cells and the rest read them as they are. This takes the
    level-ordered path of the fill kernels."""
    p = CASES[case]()
    orc = Oracle(p)
    orc.initialize_rising_bubble()
    with AmrLbm(p) as gpu:
        gpu.initialize_rising_bubble()
        for step in range(2):
            lo, hi = orc.determine_min_max_levels()
            assert gpu.determine_min_max_levels() == (lo, hi)
            if hi == lo:
                pytest.skip("a single leaf level")
            a, b = (lo, hi - 1) if narrow == "finest_out" else (lo + 1, hi)
            orc.set_level_range(a, b)
            gpu.set_level_range(a, b)
            orc.fill_ghost_cells_c2()
            gpu.fill_ghost_cells_c2()
            compare_fields(gpu, orc, fields=("C",))
            orc.phase_field_lbm_h_g()
            gpu.phase_field_lbm_h_g()
            compare_fields(gpu, orc, fields=("h", "g"))
            orc.macroscopic_values_h()
            gpu.macroscopic_values_h()
            orc.fill_ghost_cells_c()
            gpu.fill_ghost_cells_c()
            orc.macroscopic_values_g()
            gpu.macroscopic_values_g()
            compare_state(gpu, orc)


@pytest.mark.parametrize("case", ["reference_default", "tiny_minlevels0", "small_16x16"])
@pytest.mark.parametrize("narrow", ["finest_out", "coarsest_out"])
def test_regrid_with_a_narrower_level_range(case, narrow):
    """Refine_Derefine_Mesh with LevelMin..LevelMax narrower than the leaves:
    flags outside the range refine nothing (Refine.f90's DO L = LevelMin,
    LevelMax), so a regrid whose only flags lie outside it changes nothing
    and keeps the fill plans; then the fused loop goes on from there."""
    p = CASES[case]()
    orc = Oracle(p)
    orc.initialize_rising_bubble()
    with AmrLbm(p) as gpu:
        gpu.initialize_rising_bubble()
        for step in range(3):
            lo, hi = orc.determine_min_max_levels()
            assert gpu.determine_min_max_levels() == (lo, hi)
            if hi > lo:
                a, b = (lo, hi - 1) if narrow == "finest_out" else (lo + 1, hi)
                orc.set_level_range(a, b)
                gpu.set_level_range(a, b)
            orc.macroscopic_values_g()
            gpu.macroscopic_values_g()
            orc.refine_derefine_mesh()
            gpu.refine_derefine_mesh()
            compare_state(gpu, orc)
        orc.main_loop(4)
        gpu.main_loop(4)
        gpu.sync()
        compare_state(gpu, orc)


@pytest.mark.parametrize("case,regrid_every,nsteps", [
    ("tiny_minlevels0", 1, 8),
    ("small_16x16", 3, 7),
])
def test_bgk_collision_option(case, regrid_every, nsteps):
    """BGK_Collision_AMR (LBM_Subroutines.f90:337-344), which the reference
    keeps commented out at :180, in place of MRT_Collision_AMR: phase by phase
    and in the fused loop, bit for bit with the oracle under the same option;
    switching the model between calls drops the captured intervals."""
    p = CASES[case]()
    p.regrid_every = regrid_every
    orc = Oracle(p)
    orc.set_g_collision(amrlbm.G_BGK)
    orc.initialize_rising_bubble()
    with AmrLbm(p) as gpu:
        gpu.set_g_collision(amrlbm.G_BGK)
        gpu.initialize_rising_bubble()
        orc.fill_ghost_cells_c2()
        gpu.fill_ghost_cells_c2()
        orc.phase_field_lbm_h_g()
        gpu.phase_field_lbm_h_g()
        compare_fields(gpu, orc, fields=("h", "g"))
        orc.macroscopic_values_h()
        gpu.macroscopic_values_h()
        orc.fill_ghost_cells_c()
        gpu.fill_ghost_cells_c()
        orc.macroscopic_values_g()
        gpu.macroscopic_values_g()
        orc.main_loop(nsteps)
        gpu.main_loop(nsteps)
        gpu.sync()
        compare_state(gpu, orc)
        for model in (amrlbm.G_MRT, amrlbm.G_BGK):
            orc.set_g_collision(model)
            gpu.set_g_collision(model)
            orc.main_loop(3)
            gpu.main_loop(3)
            gpu.sync()
            compare_state(gpu, orc)


def test_physics_replaced_between_calls():
    """amrlbm_set_physics (a driver with its own Set_Rising_Bubble_Parameters,
    AMR_Rising_2D_OMP.f90:235-263) between fused calls: the captured
    intervals are rebuilt with the new constants, bit for bit with the oracle."""
    p = tiny_params()
    p.regrid_every = 2
    orc = Oracle(p)
    orc.initialize_rising_bubble()
    with AmrLbm(p) as gpu:
        gpu.initialize_rising_bubble()
        orc.main_loop(3)
        gpu.main_loop(3)
        ph = orc.physics()
        ph.tau_h = ph.tau_h * 1.5
        ph.sigma = ph.sigma * 0.8
        ph.beta = ph.beta * 0.8
        ph.kappa = ph.kappa * 0.8
        ph.gy = ph.gy * 2.0
        orc.set_physics(ph)
        gpu.set_physics(ph)
        orc.main_loop(4)
        gpu.main_loop(4)
        gpu.sync()
        compare_state(gpu, orc)
