"""The seeded generator of the batched-instances workload (amrlbm.batch_instances)."""
import numpy as np

import amrlbm


def test_seeded_and_in_range():
    a = amrlbm.batch_instances(64, seed=7)
    b = amrlbm.batch_instances(64, seed=7)
    assert [x.as_dict() for x in a] == [x.as_dict() for x in b]
    assert [x.as_dict() for x in a] != [x.as_dict() for x in amrlbm.batch_instances(64, seed=8)]
    for i in a:
        n = 16
        assert (i.nbx * n, i.nby * n) in {(64, 128), (128, 256), (256, 512)}
        assert i.max_levels in (2, 3) and i.dx0 == 2 ** i.max_levels
        assert 16.0 <= i.radius <= 96.0
        assert 10.0 <= i.rho_h / i.rho_l <= 1000.0 + 1e-9
        assert 1.0 <= i.bo <= 50.0
        mo = i.bo ** 3 / i.ar ** 4
        assert 1e-6 * (1 - 1e-9) <= mo <= 1e-2 * (1 + 1e-9)
        D = 2 * i.radius
        assert abs((i.gy * D) ** 0.5 - amrlbm.U_SCALE) < 1e-12
        muh = (i.gy * i.rho_h * (i.rho_h - i.rho_l) * D ** 3) ** 0.5 / i.ar
        for tau in (3 * muh / i.rho_h, 3 * (muh / i.visc_ratio) / i.rho_l):
            assert amrlbm.TAU_RANGE[0] <= tau <= amrlbm.TAU_RANGE[1]


def test_instance_params_round_trip():
    p = amrlbm.workload_small()
    i = amrlbm.Instance.from_params(p)
    q = i.params(amrlbm.batch_params(n=16))
    for k in ("nbx", "nby", "dx0", "max_levels", "rho_l", "rho_h", "visc_ratio", "bo", "ar", "gy",
              "w", "m0", "radius", "xc", "yc", "hydrostatic_start"):
        assert getattr(q, k) == getattr(p, k), k
