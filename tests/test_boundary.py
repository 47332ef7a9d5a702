"""The C ABI without a GPU: the library loads, exports every entry point that
include/amrlbm.h declares, and its host-only functions agree with the
oracle and the Python mirror."""
import ctypes as ct

import numpy as np

import amrlbm
from oracle_lib import Oracle


def test_library_exports_every_declared_symbol():
    lib = amrlbm.load_library()
    names = amrlbm.exported_symbols()
    assert len(names) >= 30, names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_default_params_match_reference_mirror():
    lib = amrlbm.load_library()
    p = amrlbm.Params()
    lib.amrlbm_default_params(ct.byref(p))
    assert p.as_dict() == amrlbm.reference_params().as_dict()


def test_derived_physics_bit_equal_to_oracle():
    lib = amrlbm.load_library()
    for p in (amrlbm.reference_params(), amrlbm.workload_small(), amrlbm.workload_large()):
        ph = amrlbm.Physics()
        assert lib.amrlbm_derive_physics(ct.byref(p), ct.byref(ph)) == 0
        o = Oracle(p).physics()
        for k, _ in amrlbm.Physics._fields_:
            assert getattr(ph, k) == getattr(o, k), k


def test_create_without_device_fails_loudly():
    """No CPU fallback: without a B200 the context cannot be created."""
    import torch
    if torch.cuda.is_available():
        return
    lib = amrlbm.load_library()
    ctx = ct.c_void_p()
    p = amrlbm.reference_params()
    assert lib.amrlbm_create(ct.byref(p), ct.byref(ctx)) == amrlbm.ERR_CUDA
    try:
        amrlbm.AmrLbm(p)
    except amrlbm.AmrLbmError as e:
        assert e.status == amrlbm.ERR_CUDA
    else:
        raise AssertionError("AmrLbm() succeeded without a device")


def test_workload_parameters():
    s, l = amrlbm.workload_small(), amrlbm.workload_large()
    assert (s.nbx * s.nx, s.nby * s.ny, s.dx0) == (64, 128, 4)
    assert (l.nbx * l.nx, l.nby * l.ny, l.dx0) == (256, 512, 8)
    assert abs(s.ar - (10.0 ** 3 / 1e-3) ** 0.25) < 1e-12 and abs(l.ar - 100.0) < 1e-9
    assert s.rho_h / s.rho_l == 10.0 and abs(l.rho_h / l.rho_l - 1000.0) < 1e-9
    assert amrlbm.tree_blocks(16, 32, 3) == 512 * 85
