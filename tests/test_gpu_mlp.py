"""GPU forward/backward/Adam kernels of the refinement-proposer MLP against the numpy oracle."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from wanniernlqg_b200 import build, _lib
    build.build()
    return _lib


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def test_forward_and_gradient_match_oracle(lib):
    from oracle import mlp_oracle as M
    L = lib.load()
    assert L.wnlqg_b200_mlp_param_count() == M.COUNT
    m = ctypes.c_void_p()
    lib.check(L.wnlqg_b200_mlp_create(0, 7, ctypes.byref(m)))
    try:
        p = np.zeros(M.COUNT, dtype=np.float32)
        lib.check(L.wnlqg_b200_mlp_get_params(m, _fp(p)))
        rng = np.random.default_rng(1)
        n = 1000
        x = rng.normal(size=(n, M.F)).astype(np.float32)
        t = rng.normal(size=n).astype(np.float32)
        y = np.zeros(n, dtype=np.float32)
        lib.check(L.wnlqg_b200_mlp_forward(m, _fp(x), n, _fp(y)))
        yo, _ = M.forward(p, x)
        np.testing.assert_allclose(y, yo, rtol=1e-5, atol=1e-5)
        loss = ctypes.c_float()
        g = np.zeros(M.COUNT, dtype=np.float32)
        lib.check(L.wnlqg_b200_mlp_loss_grad(m, _fp(x), _fp(t), n, ctypes.byref(loss), _fp(g)))
        lo, go = M.loss_grad(p, x, t)
        assert abs(loss.value - lo) < 1e-5 * max(1.0, lo)
        assert np.max(np.abs(g - go)) < 1e-4 * np.max(np.abs(go))
    finally:
        L.wnlqg_b200_mlp_destroy(m)


def test_training_reduces_loss_and_is_deterministic(lib):
    L = lib.load()
    rng = np.random.default_rng(2)
    n = 4096
    x = rng.uniform(-1, 1, size=(n, 8)).astype(np.float32)
    t = (np.sin(2 * x[:, 0]) + x[:, 1] * x[:, 2] - 0.5 * x[:, 3] ** 2).astype(np.float32)
    losses = []
    params = []
    for _ in range(2):
        m = ctypes.c_void_p()
        lib.check(L.wnlqg_b200_mlp_create(0, 11, ctypes.byref(m)))
        try:
            l0 = ctypes.c_float()
            lib.check(L.wnlqg_b200_mlp_loss_grad(m, _fp(x), _fp(t), n, ctypes.byref(l0), None))
            l1 = ctypes.c_float()
            lib.check(L.wnlqg_b200_mlp_train(m, _fp(x), _fp(t), n, 300, 3e-3, ctypes.byref(l1)))
            p = np.zeros(L.wnlqg_b200_mlp_param_count(), dtype=np.float32)
            lib.check(L.wnlqg_b200_mlp_get_params(m, _fp(p)))
        finally:
            L.wnlqg_b200_mlp_destroy(m)
        losses.append((l0.value, l1.value))
        params.append(p)
    assert losses[0][1] < 0.2 * losses[0][0]
    assert np.array_equal(params[0], params[1])
