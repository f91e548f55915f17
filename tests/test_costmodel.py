"""The learned cost model: host forward vs numpy (CPU), CUDA forward/backward vs a numpy gradient
(GPU), training, and what the trained model gains over the planner without it (GPU)."""
import ctypes as C

import numpy as np
import pytest

from rustatevec_b200 import _lib as L
from rustatevec_b200 import tuning

F = tuning.NUM_FEATURES


def n_params(H):
    return H * F + H + H * H + H + H + 1


def unpack(P, H):
    o = 0
    W1 = P[o:o + H * F].reshape(H, F); o += H * F
    b1 = P[o:o + H]; o += H
    W2 = P[o:o + H * H].reshape(H, H); o += H * H
    b2 = P[o:o + H]; o += H
    w3 = P[o:o + H]; o += H
    b3 = P[o]
    return W1, b1, W2, b2, w3, b3


def np_forward(P, H, X):
    W1, b1, W2, b2, w3, b3 = unpack(P.astype(np.float64), H)
    z1 = X @ W1.T + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0)
    return h2 @ w3 + b3, (z1, h1, z2, h2)


def np_loss_grad(P, H, X, T):
    X = X.astype(np.float64)
    y, (z1, h1, z2, h2) = np_forward(P, H, X)
    W1, b1, W2, b2, w3, b3 = unpack(P.astype(np.float64), H)
    n = len(T)
    r = y - T
    loss = np.sum(r * r) / n
    dy = 2 * r / n
    gw3 = h2.T @ dy
    gb3 = dy.sum()
    d2 = np.outer(dy, w3) * (z2 > 0)
    gW2 = d2.T @ h1
    gb2 = d2.sum(0)
    d1 = (d2 @ W2) * (z1 > 0)
    gW1 = d1.T @ X
    gb1 = d1.sum(0)
    return loss, np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gw3, [gb3]])


def random_image(H, rng):
    P = rng.normal(scale=0.3, size=n_params(H)).astype(np.float32)
    mean = rng.normal(size=F).astype(np.float32)
    scale = rng.uniform(0.5, 2.0, size=F).astype(np.float32)
    return np.concatenate([[H], mean, scale, [1.5, 2.0], P]).astype(np.float32), P, mean, scale


def test_host_forward_matches_numpy(built):
    rng = np.random.default_rng(0)
    H = 16
    img, P, mean, scale = random_image(H, rng)
    tuning.install(img)
    try:
        X = rng.normal(size=(50, F)).astype(np.float32)
        got = tuning.predict(X)
        want, _ = np_forward(P, H, (X - mean) * scale)
        assert np.max(np.abs(got - (want * 2.0 + 1.5))) < 1e-4
        assert np.array_equal(tuning.model_image(), img)
    finally:
        tuning.install(None)
    with pytest.raises(L.QsvbError):
        tuning.predict(np.zeros((1, F), np.float32))


def test_rejects_malformed_images(built):
    bad = np.zeros(10, np.float32)
    bad[0] = 16
    assert L.lib().qsvb_costmodel_set(bad.ctypes.data, len(bad)) == L.QSVB_E_INVALID


@pytest.mark.gpu
def test_cuda_gradients_match_numpy(be32):
    rng = np.random.default_rng(1)
    for H, n in ((8, 5), (32, 64), (64, 300)):
        P = rng.normal(scale=0.4, size=n_params(H)).astype(np.float32)
        X = rng.normal(size=(n, F)).astype(np.float32)
        T = rng.normal(size=n).astype(np.float32)
        loss = C.c_float()
        grad = np.zeros(n_params(H), np.float32)
        L.check(L.lib().qsvb_costmodel_forward_backward(be32.ctx, P.ctypes.data, H, X.ctypes.data, T.ctypes.data,
                                                        n, C.byref(loss), grad.ctypes.data))
        wl, wg = np_loss_grad(P, H, X, T.astype(np.float64))
        assert abs(loss.value - wl) <= 1e-4 * max(1.0, abs(wl))
        assert np.max(np.abs(grad - wg)) <= 1e-4 * max(1.0, np.max(np.abs(wg))), H


@pytest.mark.gpu
def test_training_fits_a_known_function(be32):
    rng = np.random.default_rng(2)
    X = rng.normal(size=(400, F)).astype(np.float32)
    y = (np.sin(X[:, 0]) + 0.5 * X[:, 1] * X[:, 2] - 0.3 * np.abs(X[:, 3])).astype(np.float32)
    secs = np.exp2(y)
    loss = tuning.train(be32, {"features": X, "seconds": secs}, hidden=32, epochs=1500, lr=3e-3)
    try:
        pred = tuning.predict(X)
        assert loss < 0.1
        assert np.corrcoef(pred, y)[0, 1] > 0.95
    finally:
        tuning.install(None)


@pytest.mark.gpu
def test_learned_planner_gains_over_the_untrained_method(be32):
    """Autotune at 24 qubits, train, and compare measured circuit times: the learned plan against
    the same planner on its roofline model and against qsv's greedy fuse at every width."""
    import torch
    from rustatevec_b200 import Plan, PLAN_GREEDY, PLAN_LEARNED, ENGINE_AUTO
    from rustatevec_b200.circuits import brickwork, random_circuit
    a = tuning.autotune(be32, 24, reps=3, seed=24)
    b = tuning.plan_records(be32, 24, reps=2, seed=24)
    rec = {k: np.concatenate([a[k], b[k]]) if k != "precision" else a[k] + b[k] for k in a}
    loss = tuning.train(be32, rec, hidden=64, epochs=3000)
    pred = tuning.predict(rec["features"])
    truth = np.log2(rec["seconds"])
    rank_corr = np.corrcoef(np.argsort(np.argsort(pred)), np.argsort(np.argsort(truth)))[0, 1]
    assert rank_corr > 0.8, rank_corr
    img = tuning.model_image()
    stream = torch.cuda.ExternalStream(be32.stream())

    def measure(circ, opts, reps=5):
        st = be32.alloc(circ.n_qubits())
        p = Plan(be32, circ, opts)
        be32.init_basis(st, 0)
        p.run(st)
        be32.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            p.run(st)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    try:
        report = {}
        for name, circ in (("brickwork24", brickwork(24, 20, 1)), ("random24", random_circuit(24, 400, 7))):
            tuning.install(img)
            t_learned = measure(circ, L.make_opts(PLAN_LEARNED, 6, ENGINE_AUTO))
            tuning.install(None)
            t_roofline = measure(circ, L.make_opts(PLAN_LEARNED, 6, ENGINE_AUTO))
            t_greedy = min(measure(circ, L.make_opts(PLAN_GREEDY, k, ENGINE_AUTO)) for k in (2, 3, 4, 5, 6))
            report[name] = (t_learned, t_roofline, t_greedy)
            assert t_learned <= 1.10 * t_greedy, report
            assert t_learned <= 1.10 * t_roofline, report
        print("learned vs roofline-model vs best greedy (ms):", report, "train loss", loss)
    finally:
        tuning.install(None)
