"""Known-answer and invariant tests of the CPU oracle (no GPU).

The reference ships no tests, fixtures or golden vectors and cannot be
compiled here (Fortran 90, no Fortran compiler on this machine or on the GPU
machines), so the oracle's parity with it is unpinned. These tests pin the
restatement to answers that follow from the reference's formulas:

* MRT_Collision_AMR (LBM_Subroutines.f90:348-401): with s9 = 1 the moment
  space relaxation returns geq; with g = geq it leaves g unchanged.
* Equilibrium_h_g_AMR (:2-21): sum of Gamma = 1, sum of heq = C.
* Biquadratic_from_Fine / _Coarse (Interpolations.f90:2-138) are exact on
  quadratic fields, Bilinear_from_Fine (:142-194) on bilinear fields, and the
  restriction of a constant is that constant.
* Perfect_Shift_AMR (:41-62) moves every population by its lattice vector;
  Streaming_LaxWendroff_AMR (:66-90) is exact on linear fields.
* Collision at C = 1, U = 0, h = Gamma, g = P Wa is a fixed point.
* Uniform mesh: sum of C conserved, mirror symmetry of a centred bubble.
* Topology after start-up and regrids: leaves tile the domain once, no level
  jump, leaves point to themselves as children, same-level neighbours are
  mutual.
* The regression fixtures of tests/golden/ (written by make_golden.py).
"""
import ctypes as ct
import json
import os

import numpy as np
import pytest

import amrlbm
from oracle_lib import Oracle, P

HERE = os.path.dirname(os.path.abspath(__file__))
EX = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1])
EY = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1])
WA = np.array([16, 4, 4, 4, 4, 1, 1, 1, 1]) / 36.0


@pytest.fixture(scope="module")
def orc():
    o = Oracle(amrlbm.reference_params(), 1)
    yield o
    o.close()


def test_mrt_relaxes_to_equilibrium(orc):
    rng = np.random.default_rng(1)
    geq = rng.uniform(0.0, 0.5, 9)
    g = geq + rng.normal(0.0, 1e-3, 9)
    out = g.copy()
    orc.L.orc_mrt(1.0, P(geq), P(out))
    np.testing.assert_allclose(out, geq, rtol=0, atol=1e-15)
    same = geq.copy()
    orc.L.orc_mrt(0.7, P(geq), P(same))
    assert np.array_equal(same, geq)


def test_equilibrium_moments(orc):
    rng = np.random.default_rng(2)
    for _ in range(50):
        C, U, V = rng.uniform(0, 1), rng.uniform(-0.1, 0.1), rng.uniform(-0.1, 0.1)
        a = rng.uniform(0, 2 * np.pi)
        gam, heq = np.zeros(9), np.zeros(9)
        orc.L.orc_equilibrium(orc.s, C, U, V, np.cos(a), np.sin(a), P(gam), P(heq))
        assert abs(gam.sum() - 1.0) < 1e-15
        assert abs(heq.sum() - C) < 1e-15
        # first moment of Gamma is the velocity, as the reference's Gamma
        # is the second-order expansion of the Maxwellian
        assert abs((EX * gam).sum() - U) < 1e-16 and abs((EY * gam).sum() - V) < 1e-16


def _quad(u, v):
    return 0.3 + 0.7 * u - 0.2 * v + 0.05 * u * u - 0.03 * u * v + 0.011 * v * v


def test_biquadratic_from_fine_exact_on_quadratics(orc):
    i2 = j2 = 7
    X2 = Y2 = 3
    u, v = np.meshgrid(np.arange(1, i2 + 1), np.arange(1, j2 + 1), indexing="ij")
    cin = np.asfortranarray(_quad(u, v))
    cout = np.zeros((X2, Y2), order="F")
    orc.L.orc_biquadratic_from_fine(i2, j2, X2, Y2, P(cin), P(cout))
    U, V = np.meshgrid(2 * np.arange(1, X2 + 1) - 0.5, 2 * np.arange(1, Y2 + 1) - 0.5, indexing="ij")
    np.testing.assert_allclose(cout, _quad(U, V), rtol=0, atol=1e-13)


def test_biquadratic_from_coarse_exact_on_quadratics(orc):
    I2 = J2 = 5
    x2 = y2 = 6
    u, v = np.meshgrid(np.arange(1, I2 + 1), np.arange(1, J2 + 1), indexing="ij")
    cin = np.asfortranarray(_quad(u, v))
    cout = np.zeros((x2, y2), order="F")
    orc.L.orc_biquadratic_from_coarse(I2, J2, x2, y2, P(cin), P(cout))
    pos = 1.25 + 0.5 * np.arange(1, x2 + 1)
    U, V = np.meshgrid(pos, pos, indexing="ij")
    np.testing.assert_allclose(cout, _quad(U, V), rtol=0, atol=1e-13)


def test_bilinear_from_fine_exact_on_bilinear_and_constants(orc):
    i2 = j2 = 8
    X2 = Y2 = 4
    u, v = np.meshgrid(np.arange(1, i2 + 1), np.arange(1, j2 + 1), indexing="ij")
    lin = lambda a, b: 0.25 + 0.5 * a - 0.125 * b + 0.0625 * a * b
    cin = np.asfortranarray(lin(u, v))
    cout = np.zeros((X2, Y2), order="F")
    orc.L.orc_bilinear_from_fine(i2, j2, X2, Y2, P(cin), P(cout))
    U, V = np.meshgrid(2 * np.arange(1, X2 + 1) - 0.5, 2 * np.arange(1, Y2 + 1) - 0.5, indexing="ij")
    np.testing.assert_allclose(cout, lin(U, V), rtol=0, atol=1e-13)
    const = np.full((i2, j2), 0.1234567890123, order="F")
    orc.L.orc_bilinear_from_fine(i2, j2, X2, Y2, P(const), P(cout))
    assert np.all(cout == 0.1234567890123)


def test_perfect_shift_moves_every_population(orc):
    nx = ny = orc.params.nx
    rng = np.random.default_rng(3)
    f = np.asfortranarray(rng.uniform(size=(9, nx + 2, ny + 2)))
    out = f.copy(order="F")
    orc.L.orc_stream_block(orc.s, 1, P(out))
    for k in range(9):
        for x in range(1, nx + 1):
            for y in range(1, ny + 1):
                assert out[k, x, y] == f[k, x - EX[k], y - EY[k]]


def test_lax_wendroff_exact_on_linear_fields(orc):
    nx = ny = orc.params.nx
    dx = 2
    c = 1.0 / dx
    x, y = np.meshgrid(np.arange(nx + 2), np.arange(ny + 2), indexing="ij")
    f = np.zeros((9, nx + 2, ny + 2), order="F")
    for k in range(9):
        f[k] = 0.1 + 0.01 * (k + 1) + 0.003 * x - 0.002 * y
    out = f.copy(order="F")
    orc.L.orc_stream_block(orc.s, dx, P(out))
    for k in range(9):
        want = 0.1 + 0.01 * (k + 1) + 0.003 * (x - c * EX[k]) - 0.002 * (y - c * EY[k])
        np.testing.assert_allclose(out[k, 1:nx + 1, 1:ny + 1], want[1:nx + 1, 1:ny + 1],
                                   rtol=0, atol=1e-15)


def test_collision_fixed_point_in_the_heavy_phase(orc):
    nx = ny = orc.params.nx
    C = np.ones((nx + 4, ny + 4), order="F")
    Pp = np.full((nx, ny), 0.0123, order="F")
    Ux = np.zeros((nx, ny), order="F")
    Uy = np.zeros((nx, ny), order="F")
    h = np.asfortranarray(np.broadcast_to(WA[:, None, None], (9, nx + 2, ny + 2)).copy())
    g = np.asfortranarray(h * 0.0123)
    h0, g0 = h.copy(), g.copy()
    orc.L.orc_collision_block(orc.s, 1, *[P(a) for a in (C, Pp, Ux, Uy, h, g)])
    np.testing.assert_allclose(h[:, 1:nx + 1, 1:ny + 1], h0[:, 1:nx + 1, 1:ny + 1], rtol=0, atol=1e-16)
    np.testing.assert_allclose(g[:, 1:nx + 1, 1:ny + 1], g0[:, 1:nx + 1, 1:ny + 1], rtol=0, atol=1e-16)


def _uniform_params():
    # one level of 16x16 blocks, 4x4 of them, dx = 1 (exact shift streaming)
    return amrlbm.bubble_params(64, 64, 0, 12.0, 32.0, 32.0, 10.0, 10.0, 10.0, 1e-3,
                                regrid_every=1)


def test_uniform_mesh_conserves_phase_and_mirror_symmetry():
    p = _uniform_params()
    o = Oracle(p, 2)
    try:
        o.initialize_rising_bubble()
        v0 = o.output()["phase_volume"]
        o.main_loop(30)
        d = o.output()
        assert d["status"] == 0
        assert abs(d["phase_volume"] - v0) <= 1e-12 * v0
        topo = o.topology()
        nx = p.nx
        blocks = {}
        for b in o.leaves():
            blocks[(int(topo["bi"][b - 1]), int(topo["bj"][b - 1]))] = o.download_block(int(b))
        nbx = p.nbx
        for (bi, bj), f in blocks.items():
            m = blocks[(nbx - 1 - bi, bj)]
            C = f["C"][2:nx + 2, 2:nx + 2]
            Cm = m["C"][2:nx + 2, 2:nx + 2][::-1, :]
            assert np.max(np.abs(C - Cm)) < 1e-12
            assert np.max(np.abs(f["Ux"] + m["Ux"][::-1, :])) < 1e-12
            assert np.max(np.abs(f["Uy"] - m["Uy"][::-1, :])) < 1e-12
    finally:
        o.close()


def _tiling_and_links(o, p):
    topo = o.topology()
    leaves = [int(b) for b in o.leaves()]
    nb = o.neighbours()
    finest = p.dx0 >> p.max_levels
    W = p.nbx * p.nx * p.dx0 // finest
    H = p.nby * p.ny * p.dx0 // finest
    cover = np.zeros((W, H), dtype=np.int32)
    lv = topo["level"]
    for b in leaves:
        dx = int(topo["dx"][b - 1]) // finest
        bi, bj = int(topo["bi"][b - 1]), int(topo["bj"][b - 1])
        cover[bi * p.nx * dx:(bi + 1) * p.nx * dx, bj * p.ny * dx:(bj + 1) * p.ny * dx] += 1
        assert all(int(c) == b for c in topo["child"][b - 1])  # child(:) = self
        assert int(topo["dx"][b - 1]) == p.dx0 >> int(lv[b - 1])
    assert np.all(cover == 1)
    opposite = {1: 2, 2: 1, 3: 4, 4: 3, 5: 8, 8: 5, 6: 7, 7: 6}
    leafset = set(leaves)
    for b in leaves:
        for d in range(1, 9):
            n = int(nb[b - 1][d - 1])
            if n <= 0:
                continue
            assert abs(int(lv[n - 1]) - int(lv[b - 1])) <= 1 or n not in leafset
            if n in leafset and lv[n - 1] == lv[b - 1]:
                assert int(nb[n - 1][opposite[d] - 1]) == b, (b, d, n)


def test_topology_invariants_after_start_up_and_regrids():
    p = amrlbm.reference_params()
    o = Oracle(p, 2)
    try:
        o.initialize_rising_bubble()
        _tiling_and_links(o, p)
        for _ in range(3):
            o.main_loop(2)
            _tiling_and_links(o, p)
        assert o.error() == 0 and o.level_jumps() == 0
    finally:
        o.close()


@pytest.mark.parametrize("name", ["reference_default", "small_16x16"])
def test_oracle_matches_golden_fixtures(name):
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_golden import CASES, snapshot
    with open(os.path.join(HERE, "golden", f"oracle_{name}.json")) as f:
        want = json.load(f)
    factory, steps = CASES[name]
    p = factory()
    o = Oracle(p, 2)
    try:
        o.initialize_rising_bubble()
        assert snapshot(o, p) == want["init"]
        o.main_loop(steps)
        assert snapshot(o, p) == want["after_steps"]
    finally:
        o.close()


def test_bgk_option_changes_g_only_through_the_collision():
    """The oracle's BGK_Collision_AMR switch (LBM_Subroutines.f90:180): one
    collide-fill-stream pass from the same start-up state leaves h equal
    (the collision of h does not depend on the model of g) and changes g."""
    import numpy as np
    import amrlbm
    from oracle_lib import Oracle
    p = amrlbm.reference_params()
    runs = []
    for model in (amrlbm.G_MRT, amrlbm.G_BGK):
        o = Oracle(p)
        o.set_g_collision(model)
        o.initialize_rising_bubble()
        o.fill_ghost_cells_c2()
        o.phase_field_lbm_h_g()
        runs.append({int(b): o.download_block(int(b)) for b in o.leaves()})
    same_h = all(np.array_equal(runs[0][b]["h"], runs[1][b]["h"]) for b in runs[0])
    diff_g = any(not np.array_equal(runs[0][b]["g"], runs[1][b]["g"]) for b in runs[0])
    assert same_h and diff_g


def test_phase_timers_follow_main_loop():
    """The oracle's per-phase timers (the CPU baseline's breakdown, as
    Main_Loop's timers, AMR_Rising_2D_OMP.f90:366-375) all advance over steps
    with a regrid every step."""
    p = amrlbm.workload_small()
    o = Oracle(p, 2)
    o.initialize_rising_bubble()
    t0 = o.phase_times()
    o.main_loop(3)
    t1 = o.phase_times()
    o.close()
    assert list(t1) == list(Oracle.PHASES)
    for k in Oracle.PHASES:
        assert t1[k] > t0[k] >= 0.0, k
