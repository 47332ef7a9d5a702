"""The mixed-precision time step (amrlbm_set_precision: FP16 or BF16
population storage, FP32 collision and interpolation, FP64 restriction sums
and diagnostics) against the FP64 path on the same inputs. No reference
counterpart: its oracle is the FP64 path, which is bit for bit with the CPU
restatement of the reference."""
import numpy as np
import pytest

import amrlbm
from amrlbm import AmrLbm, AmrLbmError
from parity import assert_physical

pytestmark = pytest.mark.gpu


def _run(p, prec, checkpoints):
    gpu = AmrLbm(p)
    gpu.initialize_rising_bubble()
    gpu.set_precision(prec)
    out, done = {}, 0
    for c in checkpoints:
        gpu.main_loop(c - done)
        done = c
        out[c] = gpu.output()
    gpu.close()
    return out


@pytest.mark.parametrize("prec", ["fp16", "bf16"])
def test_three_steps_close_to_fp64(prec):
    """Three steps (three regrids) in 16-bit storage stay within the storage's
    rounding of the FP64 result, field by field, on the same mesh."""
    p = amrlbm.workload_small()
    a, b = AmrLbm(p), AmrLbm(p)
    for g in (a, b):
        g.initialize_rising_bubble()
    b.set_precision(prec)
    a.main_loop(3)
    b.main_loop(3)
    ids = a.leaves()
    assert np.array_equal(ids, b.leaves())
    fa, fb = a.download_fields(ids), b.download_fields(ids)
    tol = {"fp16": 1e-4, "bf16": 1e-3}[prec]
    u_scale = (p.gy * 2.0 * p.radius) ** 0.5  # sqrt(Gy D)
    assert np.abs(fa["C"] - fb["C"]).max() <= tol
    assert np.abs(fa["P"] - fb["P"]).max() <= 10 * tol * np.abs(fa["P"]).max()
    for k in ("Ux", "Uy"):
        assert np.abs(fa[k] - fb[k]).max() <= tol * u_scale, k
    a.close()
    b.close()


def test_precision_switches_back_to_fp64():
    """FP16 steps, then FP64 steps on the converted state: the FP64 path goes
    on from the mixed-precision state, and the state stays physical."""
    p = amrlbm.workload_small()
    with AmrLbm(p) as g:
        g.initialize_rising_bubble()
        g.set_precision("fp16")
        g.main_loop(50)
        d16 = g.output()
        g.set_precision("fp64")
        g.main_loop(50)
        assert_physical(g.output(), 0.05)
        assert_physical(d16, 0.05)
    q = amrlbm.bubble_params(48, 96, 2, 20.0, 96.0, 96.0, 10.0, 10.0, 10.0, 1e-3, n=12)
    with AmrLbm(q) as g:
        with pytest.raises(AmrLbmError):
            g.set_precision("fp16")  # 12x12 blocks: not supported
