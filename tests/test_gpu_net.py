"""The refine-flag forecaster's tensor-core kernels against NumPy: the BF16
product alone, the forward pass, and the gradient of every parameter
(tests/net_ref.py restates the network with the same BF16 roundings)."""
import ctypes as ct

import numpy as np
import pytest

import amrlbm
import net_ref

pytestmark = pytest.mark.gpu


def test_tensor_core_product():
    lib = amrlbm.load_library()
    rng = np.random.default_rng(3)
    for M, N, K in ((100, 40, 70), (64, 32, 16), (1, 300, 5), (333, 32, 288)):
        A = net_ref.bf16(rng.standard_normal((M, K))).astype(np.float32)
        B = net_ref.bf16(rng.standard_normal((K, N))).astype(np.float32)
        Ab = (A.view(np.uint32) >> 16).astype(np.uint16)
        Bb = (B.view(np.uint32) >> 16).astype(np.uint16)
        C = np.zeros((M, N), dtype=np.float32)
        assert lib.amrlbm_net_selftest_gemm(M, N, K, Ab.ctypes.data_as(ct.POINTER(ct.c_uint16)),
                                            Bb.ctypes.data_as(ct.POINTER(ct.c_uint16)),
                                            C.ctypes.data_as(ct.POINTER(ct.c_float))) == 0
        ref = A.astype(np.float64) @ B.astype(np.float64)
        assert np.abs(C - ref).max() <= 1e-5 * np.abs(ref).max() * np.sqrt(K), (M, N, K)


def test_forward_and_gradient_against_numpy():
    rng = np.random.default_rng(11)
    n = 12
    x = rng.standard_normal((n, 4, 18, 18)).astype(np.float32)
    y = (rng.random(n) < 0.4).astype(np.float32)
    net = amrlbm.Net(seed=5, max_batch=16)
    p = net.params()
    loss, g = net.gradient(x, y, pos_weight=3.0)
    rl, rg, rz = net_ref.loss_and_grad(p, x, y, pos_weight=3.0)
    z = net.forward(x)
    assert np.allclose(z, rz, rtol=1e-4, atol=1e-4)
    assert abs(loss - rl) <= 1e-4 * max(1.0, abs(rl))
    blocks = {"W1": (net_ref.O_W1, net_ref.O_B1), "b1": (net_ref.O_B1, net_ref.O_W2),
              "W2": (net_ref.O_W2, net_ref.O_B2), "b2": (net_ref.O_B2, net_ref.O_W3),
              "W3": (net_ref.O_W3, net_ref.O_B3), "b3": (net_ref.O_B3, net_ref.O_WD),
              "wd": (net_ref.O_WD, net_ref.O_BD), "bd": (net_ref.O_BD, net_ref.NPARAM)}
    for name, (a, b) in blocks.items():
        err = np.linalg.norm(g[a:b] - rg[a:b]) / max(np.linalg.norm(rg[a:b]), 1e-12)
        assert err < 1e-3, (name, err)
    net.close()


def test_training_reduces_the_loss():
    """Adam steps on a separable toy set (the label is whether channel 1 has
    a cell above a threshold, as a flag from |grad C| would be)."""
    rng = np.random.default_rng(2)
    x = rng.random((256, 4, 18, 18)).astype(np.float32) * 0.5
    y = (rng.random(256) < 0.5).astype(np.float32)
    x[y > 0.5, 1, 9, 9] = 3.0
    net = amrlbm.Net(seed=1, max_batch=256)
    first = net.train_step(x, y, lr=3e-3)
    for _ in range(60):
        last = net.train_step(x, y, lr=3e-3)
    assert last < 0.5 * first
    acc = ((net.forward(x) > 0) == (y > 0.5)).mean()
    assert acc > 0.95
    net.close()
