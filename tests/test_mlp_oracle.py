"""CPU checks of the learned stop predictor's oracle and host logic.

The numpy restatement (oracle/mlp.py) is what the GPU kernels are checked
against bit for bit; here its backward formulas are checked against finite
differences of the float64 network, its bf16 rounding against known values,
and the trace-target logic of parex_b200.learn on a hand-built trace.
"""
import numpy as np

from oracle import mlp as M
from parex_b200 import _lib
from parex_b200 import learn


def _net(seed=0, n=200):
    rng = np.random.default_rng(seed)
    w = learn.init_master(seed).astype(np.float64)
    w[M.OFF_B1:M.OFF_W2] = rng.normal(0, 0.1, 32)
    w[M.OFF_B2:M.OFF_W3] = rng.normal(0, 0.1, 32)
    X = rng.normal(0, 1, (n, 16))
    norm = np.concatenate([rng.normal(0, 0.1, 16), rng.uniform(0.5, 1.5, 16)])
    T = rng.uniform(0, 4, n)
    return w, norm, X, T


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 0.0, 1.0 + 2 ** -7, 3.0e38], dtype=np.float32)
    y = M.bf16(x)
    assert y[0] == 1.0
    assert y[1] == 1.0                      # tie goes to the even mantissa
    assert y[2] == np.float32(1.0 + 2 ** -7)
    assert y[3] == -2.5 and y[4] == 0.0 and y[5] == np.float32(1.0 + 2 ** -7)
    np.testing.assert_array_equal(learn.to_bf16_bits(x), M.bf16_bits(x))


def test_backward_matches_finite_differences():
    w, norm, X, T = _net()
    loss, g = M.gradient_f64(w, norm, X, T, delta=1.0, over=4.0)
    rng = np.random.default_rng(1)
    idx = rng.choice(M.PARAMS, 60, replace=False)
    eps = 1e-6
    for p in idx:
        wp, wm = w.copy(), w.copy()
        wp[p] += eps
        wm[p] -= eps
        num = (M.gradient_f64(wp, norm, X, T, 1.0, 4.0)[0] - M.gradient_f64(wm, norm, X, T, 1.0, 4.0)[0]) / (2 * eps)
        assert abs(num - g[p]) <= 1e-5 + 1e-4 * abs(g[p]), (p, num, g[p])


def test_bf16_gradient_close_to_float64():
    w, norm, X, T = _net(seed=3, n=256)
    bits = M.bf16_bits(w.astype(np.float32))
    wq = M.from_bits(bits).astype(np.float64)
    g32, loss32 = M.gradient(bits, norm.astype(np.float32), X.astype(np.float32), T.astype(np.float32), 1.0, 4.0)
    loss64, g64 = M.gradient_f64(wq, norm, X, T, 1.0, 4.0)
    assert abs(loss32 - loss64) <= 0.05 * abs(loss64) + 1e-3
    rel = np.linalg.norm(g32 - g64) / np.linalg.norm(g64)
    assert rel < 0.05, rel


def test_forward_is_deterministic_and_layout():
    w, norm, X, T = _net(seed=5, n=37)
    bits = M.bf16_bits(w.astype(np.float32))
    y1, _ = M.forward(bits, norm, X)
    y2, _ = M.forward(bits, norm, X[::-1].copy())
    np.testing.assert_array_equal(y1, y2[::-1])
    assert M.PARAMS == _lib.MLP_PARAMS == 1633


def _rec(rows):
    rec = np.zeros(len(rows), dtype=_lib.RECORD_DTYPE)
    for i, (rnd, root, size, origin) in enumerate(rows):
        rec[i]["round"], rec[i]["root"], rec[i]["size"], rec[i]["origin"] = rnd, root, size, origin
    return rec


def test_trace_targets():
    S, C = learn.ORIGIN_SWEPT, learn.ORIGIN_CHILD
    rec = _rec([
        (0, 0, 100, C),                        # the start cluster splits: children
        (1, 0, 60, S), (1, 60, 40, S),
        (2, 0, 60, S), (2, 60, 40, S),
        (3, 0, 60, S), (3, 60, 30, C), (3, 90, 10, C),   # cluster 60 cut at round 3
        (4, 0, 60, S), (4, 60, 30, S),
        (5, 60, 30, S),                        # cluster 0 certified at round 5
    ])
    t = learn.trace_targets(rec)
    np.testing.assert_array_equal(t, [-1, 3, 1, 2, 0, 1, -1, -1, 0, 1, 0])
