"""The two plain FP64 rising-bubble workloads run on the CPU oracle for their
full lengths (2000 steps of the 64x128-base, density-ratio-10 bubble; 5000
steps of the 256x512-base, density-ratio-1000 R=128 bubble with a regrid every
10 steps), checked for a physical trajectory: finite fields, velocities far
below the lattice sound speed, a rising centroid, and the mass drift. These are
the trajectories the device path is compared with bit for bit
(tests/test_gpu_long.py) and the bench times.

Also pins the hydrostatic start-up pressure against its formula."""
import numpy as np
import pytest

import amrlbm
from oracle_lib import Oracle
from parity import assert_physical

pytestmark = pytest.mark.slow


def _run(p, total, every):
    orc = Oracle(p)
    orc.initialize_rising_bubble()
    d0 = orc.output()
    rows = [(0, d0)]
    for s in range(every, total + 1, every):
        orc.main_loop(every)
        rows.append((s, orc.output()))
    return orc, rows


def test_small_workload_2000_steps():
    p = amrlbm.workload_small()
    orc, rows = _run(p, 2000, 500)
    m0 = rows[0][1]["mass"]
    for s, d in rows[1:]:
        assert_physical(d, 0.05, f"step {s}")
        assert abs(d["mass"] - m0) / m0 < 1e-5, (s, d["mass"], m0)
    yc = [d["y_centroid"] for _, d in rows]
    assert all(b > a for a, b in zip(yc[1:], yc[2:])), yc  # the bubble rises
    assert rows[-1][1]["rise_velocity"] > rows[1][1]["rise_velocity"]


def test_large_workload_5000_steps():
    """BASELINE-size bubble (R=128, density ratio 1000, Eo 10, Mo 1e-5): 5000
    steps stay finite with |Uy| < 0.01 and a relative mass drift below 1e-6."""
    p = amrlbm.workload_large()
    orc, rows = _run(p, 5000, 1000)
    m0 = rows[0][1]["mass"]
    for s, d in rows[1:]:
        assert_physical(d, 0.01, f"step {s}")
        assert abs(d["mass"] - m0) / m0 < 1e-6, (s, d["mass"], m0)
    yc = [d["y_centroid"] for _, d in rows]
    assert all(b > a for a, b in zip(yc[1:], yc[2:])), yc
    assert rows[-1][1]["rise_velocity"] > rows[1][1]["rise_velocity"]
    c = orc.counts()
    assert c["level_max"] == p.max_levels and c["nleaf"] >= 788


@pytest.mark.parametrize("hydro", [0, 1])
def test_hydrostatic_start_pressure(hydro):
    """P after Initialize_AMR_Rising_Bubble: the reference's -Sigma/R*C
    (AMR_Rising_2D_OMP.f90:193), plus Gy*(Rhoh-Rhol)*(1-C)*(y-yc) with
    hydrostatic_start = 1."""
    p = amrlbm.workload_small()
    p.hydrostatic_start = hydro
    orc = Oracle(p)
    orc.initialize_rising_bubble()
    ph = orc.physics()
    t = orc.topology()
    nx = p.nx
    for b in orc.leaves()[:40]:
        blk = orc.download_block(int(b))
        dx = int(t["dx"][b - 1])
        C = blk["C"][2:nx + 2, 2:nx + 2]
        y = float(t["bj"][b - 1] * dx * nx) + dx * (np.arange(1, nx + 1) - 0.5)
        want = -ph.sigma / p.radius * C
        if hydro:
            want = want + ph.gy * (ph.rho_h - ph.rho_l) * (1.0 - C) * (y[None, :] - p.yc)
        assert np.array_equal(blk["P"], want)
