"""The device path over the full lengths of the plain FP64 workloads, bit for
bit with the CPU oracle, on trajectories checked to be physical (finite,
velocities far below the lattice sound speed, density positive, the bubble
rising): the states the bench times."""
import numpy as np
import pytest

import amrlbm
from amrlbm import AmrLbm
from oracle_lib import Oracle
from parity import assert_physical, compare_counts, compare_fields, compare_state, compare_topology

pytestmark = pytest.mark.gpu


def _lockstep(p, chunks, u_bound, full_compare_every=1):
    """Runs the device and the oracle side by side in `chunks` (steps per
    call); after each call the diagnostics must be equal and physical, and
    every `full_compare_every`-th call the complete state is compared."""
    orc = Oracle(p)
    orc.initialize_rising_bubble()
    gpu = AmrLbm(p)
    gpu.initialize_rising_bubble()
    compare_state(gpu, orc)
    start = gpu.leaves().copy()
    done = 0
    for i, n in enumerate(chunks):
        orc.main_loop(n)
        gpu.main_loop(n)
        gpu.sync()
        done += n
        a, b = gpu.output(), orc.output()
        for k in a:
            assert a[k] == b[k], (done, k, a[k], b[k])
        assert_physical(b, u_bound, f"step {done}")
        if (i + 1) % full_compare_every == 0 or i == len(chunks) - 1:
            compare_counts(gpu, orc)
            compare_topology(gpu, orc)
            compare_fields(gpu, orc)
    return gpu, orc, start


def test_small_workload_2000_steps():
    """64x128 base, density ratio 10, a regrid after every step: 2000 steps."""
    p = amrlbm.workload_small()
    gpu, orc, _ = _lockstep(p, [500] * 4, 0.05)
    gpu.close()


def test_large_workload_5000_steps():
    """256x512 base, 3 levels, R=128, density ratio 1000, regrid every 10
    steps: 5000 steps, the full length of the configuration."""
    p = amrlbm.workload_large()
    gpu, orc, _ = _lockstep(p, [250, 750] + [1000] * 4, 0.01, full_compare_every=2)
    gpu.close()


def test_large_workload_mesh_growth():
    """The same geometry with Gy = 1e-6 and M0 = 0.1, whose mesh grows from 788
    leaves as the bubble rises: 800 steps with refining and derefining
    regrids, bit for bit."""
    p = amrlbm.workload_large()
    p.gy = 1e-6
    p.m0 = 0.1
    gpu, orc, start = _lockstep(p, [200] * 4, 0.01)
    assert not np.array_equal(gpu.leaves(), start)
    assert gpu.counts()["nleaf"] > len(start)
    gpu.close()
