"""The tcgen05 BF16 MLP kernels of the learned warm start against the CPU
oracle (oracle/mlp_oracle.py): forward values, loss and every parameter
gradient, that a gradient is the same bits on every run, and that Adam
training on the GPU reduces the loss."""
import ctypes as C

import numpy as np
import pytest

import mlp_oracle as mo
from pigfem_assignment_b200 import _lib

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def flat(p):
    return np.concatenate([p[k].ravel() for k in ("W1", "b1", "W2", "b2", "W3", "b3")]).astype(np.float32)


def unflat(v):
    shapes = [("W1", (64, 16)), ("b1", (64,)), ("W2", (64, 64)), ("b2", (64,)), ("W3", (16, 64)), ("b3", (16,))]
    out, o = {}, 0
    for k, sh in shapes:
        n = int(np.prod(sh))
        out[k] = v[o:o + n].reshape(sh).copy()
        o += n
    return out


@pytest.fixture()
def mlp():
    h = C.c_void_p()
    _lib.check(_lib.lib.pg_mlp_create(0, 7, C.byref(h)))
    yield h
    _lib.lib.pg_mlp_destroy(h)


def set_params(h, p):
    v = flat(p)
    _lib.check(_lib.lib.pg_mlp_params(h, v.ctypes.data_as(C.POINTER(C.c_float)), 1))


def test_param_count():
    assert _lib.lib.pg_mlp_param_count() == 64 * 16 + 64 + 64 * 64 + 64 + 16 * 64 + 16


@pytest.mark.parametrize("n", [128, 1000, 20000])
def test_forward_matches_oracle(mlp, n):
    rng = np.random.default_rng(n)
    p = mo.init_params(1)
    p["W3"] = (rng.standard_normal((16, 64)) * 0.2).astype(np.float32)
    p["b1"] = (0.1 * rng.standard_normal(64)).astype(np.float32)
    p["b2"] = (0.1 * rng.standard_normal(64)).astype(np.float32)
    p["b3"] = (0.1 * rng.standard_normal(16)).astype(np.float32)
    set_params(mlp, p)
    x = rng.standard_normal((n, 16)).astype(np.float32)
    X = torch.from_numpy(x).cuda()
    Y = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    _lib.check(_lib.lib.pg_mlp_forward(mlp, C.c_void_p(X.data_ptr()), n, C.c_void_p(Y.data_ptr()), None))
    y = Y.cpu().numpy()
    yo, _ = mo.forward(p, x)
    scale = np.abs(yo[:, :2]).max()
    assert np.abs(y - yo[:, :2]).max() <= 2e-2 * scale


@pytest.mark.parametrize("n", [256, 3000])
def test_gradients_match_oracle(mlp, n):
    rng = np.random.default_rng(10 + n)
    p = mo.init_params(2)
    p["W3"] = (rng.standard_normal((16, 64)) * 0.2).astype(np.float32)
    p["b1"] = (0.1 * rng.standard_normal(64)).astype(np.float32)
    p["b2"] = (0.1 * rng.standard_normal(64)).astype(np.float32)
    set_params(mlp, p)
    x = rng.standard_normal((n, 16)).astype(np.float32)
    t = rng.standard_normal((n, 2)).astype(np.float32)
    X = torch.from_numpy(x).cuda()
    T = torch.from_numpy(t).cuda()
    loss = C.c_double()
    _lib.check(_lib.lib.pg_mlp_gradient(mlp, C.c_void_p(X.data_ptr()), C.c_void_p(T.data_ptr()), n, C.byref(loss)))
    g = np.zeros(_lib.lib.pg_mlp_param_count(), np.float32)
    _lib.check(_lib.lib.pg_mlp_grads(mlp, g.ctypes.data_as(C.POINTER(C.c_float))))
    gg = unflat(g)
    lo, go = mo.loss_and_grads(p, x, np.pad(t, ((0, 0), (0, 14))))
    assert abs(loss.value - lo) <= 1e-2 * lo
    for k in ("W1", "b1", "W2", "b2"):
        ref = go[k]
        assert np.linalg.norm(gg[k] - ref) <= 3e-2 * np.linalg.norm(ref) + 1e-7, k
    for k in ("W3", "b3"):
        ref = go[k][:2]
        assert np.linalg.norm(gg[k][:2] - ref) <= 3e-2 * np.linalg.norm(ref) + 1e-7, k
        assert np.abs(gg[k][2:]).max() == 0.0


def test_gradient_is_bit_reproducible(mlp):
    """Each CTA's part of the gradient is summed in a fixed order and the
    parts are added in CTA order: two gradients of the same rows agree bit
    for bit, and so do two trainings from the same start."""
    rng = np.random.default_rng(3)
    n = 50000  # more tiles than CTAs: every CTA sums several tiles
    X = torch.from_numpy(rng.standard_normal((n, 16)).astype(np.float32)).cuda()
    T = torch.from_numpy(rng.standard_normal((n, 2)).astype(np.float32)).cuda()
    out = []
    for _ in range(2):
        set_params(mlp, mo.init_params(4))
        loss = C.c_double()
        _lib.check(_lib.lib.pg_mlp_gradient(mlp, C.c_void_p(X.data_ptr()), C.c_void_p(T.data_ptr()), n,
                                            C.byref(loss)))
        g = np.zeros(_lib.lib.pg_mlp_param_count(), np.float32)
        _lib.check(_lib.lib.pg_mlp_grads(mlp, g.ctypes.data_as(C.POINTER(C.c_float))))
        hist = np.zeros(3)
        _lib.check(_lib.lib.pg_mlp_train(mlp, C.c_void_p(X.data_ptr()), C.c_void_p(T.data_ptr()), n, 3, 4096,
                                         C.c_float(1e-3), hist.ctypes.data_as(C.POINTER(C.c_double))))
        w = np.zeros(_lib.lib.pg_mlp_param_count(), np.float32)
        _lib.check(_lib.lib.pg_mlp_params(mlp, w.ctypes.data_as(C.POINTER(C.c_float)), 0))
        out.append((loss.value, g, hist, w))
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2])
    assert np.array_equal(out[0][3], out[1][3])


def test_training_reduces_loss(mlp):
    rng = np.random.default_rng(5)
    n = 16384
    x = rng.standard_normal((n, 16)).astype(np.float32)
    w = rng.standard_normal((16, 2)).astype(np.float32)
    t = np.tanh(x @ w).astype(np.float32)
    X = torch.from_numpy(x).cuda()
    T = torch.from_numpy(t).cuda()
    hist = np.zeros(20)
    _lib.check(_lib.lib.pg_mlp_train(mlp, C.c_void_p(X.data_ptr()), C.c_void_p(T.data_ptr()), n, 20, 1024, 3e-3,
                                     hist.ctypes.data_as(C.POINTER(C.c_double))))
    assert hist[-1] < 0.25 * hist[0], hist
