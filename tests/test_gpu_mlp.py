"""The MLP kernels of the learned stop predictor against the CPU oracle
(oracle/mlp.py): forward, loss gradient and Adam step bit for bit, and a
short GPU training run that lowers the loss."""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import mlp as M
from parex_b200 import _lib, learn

pytestmark = pytest.mark.gpu


def _case(seed=0, n=1000):
    rng = np.random.default_rng(seed)
    master = learn.init_master(seed)
    master[M.OFF_B1:M.OFF_W2] = rng.normal(0, 0.1, 32)
    master[M.OFF_B2:M.OFF_W3] = rng.normal(0, 0.1, 32)
    master[M.OFF_B3] = 0.5
    X = rng.normal(0, 1, (n, 16)).astype(np.float32)
    norm = np.concatenate([rng.normal(0, 0.1, 16), rng.uniform(0.5, 1.5, 16)]).astype(np.float32)
    T = rng.uniform(0, 4, n).astype(np.float32)
    return master.astype(np.float32), learn.to_bf16_bits(master), norm, X, T


def _d(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a if dtype is None else a.view(dtype))).cuda()
    return t


def _p(t):
    return C.c_void_p(t.data_ptr())


def test_forward_bit_exact():
    L = _lib.load()
    master, bits, norm, X, T = _case(1, 3001)
    out = torch.zeros(X.shape[0], dtype=torch.float32, device="cuda")
    dX, dw, dn = _d(X), _d(bits, np.int16), _d(norm)     # keep the device arrays alive across the call
    assert L.pxr_mlp_forward(_p(dX), X.shape[0], _p(dw), _p(dn), _p(out), None) == 0
    torch.cuda.synchronize()
    y, _ = M.forward(bits, norm, X)
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), y.view(np.uint32))


@pytest.mark.parametrize("n", [1, 64, 1000, 4099])
def test_gradient_bit_exact(n):
    L = _lib.load()
    master, bits, norm, X, T = _case(2, n)
    grad = torch.zeros(M.PARAMS, dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    scratch = torch.zeros(int(L.pxr_mlp_scratch_floats(n)), dtype=torch.float32, device="cuda")
    spec = _lib.MlpLoss(1.0, 4.0)
    dX, dT, dw, dn = _d(X), _d(T), _d(bits, np.int16), _d(norm)
    st = L.pxr_mlp_gradient(_p(dX), _p(dT), n, _p(dw), _p(dn), C.byref(spec), _p(scratch), _p(grad), _p(loss), None)
    assert st == 0
    torch.cuda.synchronize()
    g_ref, l_ref = M.gradient(bits, norm, X, T, 1.0, 4.0)
    np.testing.assert_array_equal(grad.cpu().numpy().view(np.uint32), g_ref.view(np.uint32))
    assert loss.cpu().numpy()[0].view(np.uint32) == np.float32(l_ref).view(np.uint32)
    # and it is the gradient: close to the float64 network without bf16 rounding
    l64, g64 = M.gradient_f64(M.from_bits(bits).astype(np.float64), norm, X, T, 1.0, 4.0)
    assert np.linalg.norm(grad.cpu().numpy() - g64) <= 0.05 * np.linalg.norm(g64) + 1e-6


def test_adam_step_bit_exact():
    L = _lib.load()
    master, bits, norm, X, T = _case(3, 10)
    rng = np.random.default_rng(4)
    g = rng.normal(0, 1e-2, M.PARAMS).astype(np.float32)
    m = rng.normal(0, 1e-3, M.PARAMS).astype(np.float32)
    v = np.abs(rng.normal(0, 1e-4, M.PARAMS)).astype(np.float32)
    dm, dv, dmaster = _d(m.copy()), _d(v.copy()), _d(master.copy())
    w = torch.zeros(M.PARAMS, dtype=torch.int16, device="cuda")
    opt = _lib.MlpAdam(3e-3, 0.9, 0.999, 1e-8)
    dg = _d(g)
    assert L.pxr_mlp_adam_step(_p(dmaster), _p(dm), _p(dv), _p(dg), _p(w), 7, C.byref(opt), None) == 0
    torch.cuda.synchronize()
    x_ref, m_ref, v_ref, w_ref = M.adam_step(master, m, v, g, 7, 3e-3, 0.9, 0.999, 1e-8)
    np.testing.assert_array_equal(dmaster.cpu().numpy().view(np.uint32), x_ref.view(np.uint32))
    np.testing.assert_array_equal(dm.cpu().numpy().view(np.uint32), m_ref.view(np.uint32))
    np.testing.assert_array_equal(dv.cpu().numpy().view(np.uint32), v_ref.view(np.uint32))
    np.testing.assert_array_equal(w.cpu().numpy().view(np.uint16), w_ref)


def test_training_lowers_loss():
    rng = np.random.default_rng(7)
    X = rng.normal(0, 1, (20000, 16)).astype(np.float32)
    T = np.maximum(0, 1.5 * X[:, 0] - X[:, 3] + 0.5 * X[:, 5] * X[:, 6] + 1).astype(np.float32)
    model = learn.train(X, T, epochs=8, batch=2048, lr=3e-3)
    y = learn.predict(model, X)
    y0 = np.full_like(T, T.mean())
    assert np.mean((y - T) ** 2) < 0.35 * np.mean((y0 - T) ** 2)
    # the model's forward on the GPU is the oracle's, bit for bit
    y_ref, _ = M.forward(model.weights, model.norm, X)
    np.testing.assert_array_equal(y.view(np.uint32), y_ref.view(np.uint32))
