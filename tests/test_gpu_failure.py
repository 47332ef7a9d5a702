"""Failure detection without a GPU fault: a bounded device wait that runs out
reports AMRLBM_ERR_TIMEOUT to the host and the context stays usable.

The level-ordered fills (a level range narrower than the leaves, the
reference's DO L = LevelMin, LevelMax over a subset of the levels) order their
items by per-block flags. amrlbm_set_wait_test shortens every flag wait and
keeps one block's flag from ever being raised, so the items that wait for it
run out of their bound, record the timeout and return."""
import pytest

import amrlbm
from amrlbm import AmrLbm, AmrLbmError
from oracle_lib import Oracle
from parity import compare_state, copy_state_to_gpu

pytestmark = pytest.mark.gpu


def test_flag_wait_runs_out_and_the_context_recovers():
    p = amrlbm.workload_small()
    orc = Oracle(p)
    orc.initialize_rising_bubble()
    with AmrLbm(p) as gpu:
        gpu.initialize_rising_bubble()
        lo, hi = gpu.determine_min_max_levels()
        assert hi > lo
        gpu.set_level_range(lo + 1, hi)  # narrower than the leaves: level order
        lv = gpu.topology()["level"]
        held = next(int(b) for b in gpu.leaves() if lv[b - 1] == lo + 1)
        gpu.set_wait_test(spin_limit=2000, hold_block=held)
        status = 0
        try:
            gpu.fill_ghost_cells_c2()
            gpu.phase_field_lbm_h_g()
        except AmrLbmError as e:
            status = e.status
        assert status == amrlbm.ERR_TIMEOUT
        assert "wait ran out" in gpu.lib.amrlbm_last_error(gpu.ctx).decode()
        # the status was reported once; normal operation resumes
        gpu.set_wait_test(0, 0)
        gpu.sync()
        copy_state_to_gpu(orc, gpu)
        orc.main_loop(3)
        gpu.main_loop(3)
        gpu.sync()
        compare_state(gpu, orc)


def test_wait_test_rejects_bad_arguments():
    p = amrlbm.workload_small()
    with AmrLbm(p) as gpu:
        lib = gpu.lib
        assert lib.amrlbm_set_wait_test(gpu.ctx, -1, 0) == amrlbm.ERR_ARG
        assert lib.amrlbm_set_wait_test(gpu.ctx, 0, p.max_blks + 1) == amrlbm.ERR_ARG
        assert lib.amrlbm_set_wait_test(gpu.ctx, 0, 0) == 0
