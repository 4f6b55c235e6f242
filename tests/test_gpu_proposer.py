"""Band proposer on the GPU: the device feature kernel against the NumPy
model, the training kernels (the loss falls), and the planned batch run
(identical consensus with and without the plan; fallback accounting)."""
import os

import numpy as np
import pytest

import poa_b200
from poa_b200 import synth
from tests import proposer_model as pm

pytestmark = pytest.mark.gpu


def _feature_windows():
    ws = synth.windows(31, 5, (300, 2500), (2, 12), 0.15, chimeric=0.1)
    reads, offs = [], [0]
    for w in range(ws.n_windows):
        rs = ws.window_reads(w)
        reads.extend(rs)
        offs.append(offs[-1] + len(rs))
    # edge window: a read shorter than a k-mer window, one with N, an empty one
    t = reads[0][:600]
    edge = [t, t[:10], t[:200] + b"N" * 30 + t[230:], b"", t.lower()]
    reads.extend(edge)
    offs.append(offs[-1] + len(edge))
    reads.append(t)  # single-read window
    offs.append(offs[-1] + 1)
    return synth.pack_windows_from_reads(reads, offs)


def test_device_features_match_model():
    ws = _feature_windows()
    prop = poa_b200.Proposer()
    with poa_b200.Context(poa_b200.Params.from_cli(["-B"])) as ctx:
        ctx.batch_upload(ws)
        X = ctx.batch_features(prop)
    for w in range(ws.n_windows):
        a, b = int(ws.win_off[w]), int(ws.win_off[w + 1])
        ref = pm.window_features(ws.window_reads(w))
        np.testing.assert_allclose(X[a:b], ref, rtol=1e-6, atol=1e-7, err_msg=f"window {w}")


def test_training_reduces_loss():
    rng = np.random.default_rng(5)
    n = 2048
    X = rng.random((n, 32, 8), dtype=np.float32)
    # smooth functions of bin averages (what convolutions + mean pooling express)
    Y = np.stack([X[:, :, 0].mean(1), X[:, :, 1].mean(1) * 2, X[:, :, 2].mean(1) ** 2,
                  (X[:, :, 0] * X[:, :, 3]).mean(1)], 1)
    prop = poa_b200.Proposer()
    losses = prop.train(X, Y, epochs=15, batch=128, lr=2e-3, seed=3)
    assert np.isfinite(losses).all()
    assert losses[-1] < 0.5 * losses[0]
    P = prop.predict(X)
    assert P.shape == (n, 4) and np.isfinite(P).all()
    r2 = 1 - ((P - Y) ** 2).mean(0) / Y.var(0)
    assert (r2 > 0.8).all(), r2
    # weights round-trip
    w = prop.get_weights()
    prop2 = poa_b200.Proposer()
    prop2.set_weights(w)
    np.testing.assert_array_equal(prop2.predict(X[:64]), prop.predict(X[:64]))


def _lb_windows():
    # config-5-like windows, fewer and with fewer reads (seconds, not minutes)
    return synth.windows(77, 24, (2000, 2000), (10, 30), 0.15, chimeric=0.02)


def test_planned_run_is_exact_and_smaller():
    ws = _lb_windows()
    prop = poa_b200.Proposer(weights=poa_b200.PROP_WEIGHTS)
    with poa_b200.Context(poa_b200.Params.from_cli(["-B"])) as ctx:
        ctx.batch_upload(ws)
        ctx.batch_run()
        cons0, st0 = ctx.batch_download()
        s0 = ctx.batch_stats()
        ctx.batch_use_proposer(prop)
        ctx.batch_run()
        cons1, st1 = ctx.batch_download()
        s1 = ctx.batch_stats()
        # the per-window plan the run used, against each window's real need
        p_nodes, p_tb, p_sp = ctx.batch_plan_get()
        rs = ctx.batch_read_stats()
        # the same through the host-buffer entry point
        cons2, st2 = ctx.batch_consensus(ws)
    assert st0 == [0] * ws.n_windows
    assert cons1 == cons0 and st1 == st0
    assert cons2 == cons0 and st2 == st0
    assert s1["cells"] == s0["cells"]
    assert s1["plan_us"] > 0 and s1["run_us"] >= s1["kernel_us"]
    assert s1["fallback"] <= 1
    assert s1["slot_bytes"] < s0["slot_bytes"]
    assert p_nodes.shape == (ws.n_windows,) and (p_nodes > 2).all() and (p_tb > 0).all()
    over = 0
    for w in range(ws.n_windows):
        a, b = int(ws.win_off[w]), int(ws.win_off[w + 1])
        over += int(rs[b - 1, 3] > p_nodes[w] or rs[a:b, 4].max() > p_tb[w])
    assert over <= max(2, ws.n_windows // 4)  # each window's own prediction mostly covers it


def test_undersized_plan_falls_back_exactly():
    ws = _lb_windows()
    prop = poa_b200.Proposer(weights=poa_b200.PROP_WEIGHTS)
    w = prop.get_weights()
    base = w.shape[0] - 12
    w[base + 8] = 0.2   # node margin far too small
    w[base + 9] = 0.05  # record-byte margin far too small
    prop.set_weights(w)
    with poa_b200.Context(poa_b200.Params.from_cli(["-B"])) as ctx:
        ctx.batch_upload(ws)
        ctx.batch_run()
        cons0, st0 = ctx.batch_download()
        ctx.batch_use_proposer(prop)
        ctx.batch_run()
        cons1, st1 = ctx.batch_download()
        s1 = ctx.batch_stats()
    assert cons1 == cons0 and st1 == st0
    assert s1["fallback"] == ws.n_windows


# ---- the network against its NumPy restatement (tests/proposer_net.py) ----
from tests import proposer_net as net  # noqa: E402


def _check_forward(prop, w, X):
    got = prop.predict(X)
    want = net.predict(w, X, use_bf16=True)
    scale = np.std(want, axis=0) + 1e-3
    # same BF16 rounding points, float32 accumulation in a different order: a
    # few activations may round to the neighbouring BF16 value
    assert np.all(np.abs(got - want) <= 2e-2 * scale[None, :]), np.max(np.abs(got - want) / scale[None, :])
    assert np.median(np.abs(got - want) / scale[None, :]) < 2e-3


def test_forward_pass_matches_numpy_committed_weights():
    prop = poa_b200.Proposer(weights=poa_b200.PROP_WEIGHTS)
    w = prop.get_weights().astype(np.float64)
    ws = _feature_windows()
    with poa_b200.Context(poa_b200.Params.from_cli(["-B"])) as ctx:
        ctx.batch_upload(ws)
        X = ctx.batch_features(prop)
    _check_forward(prop, w, X)


def test_forward_pass_matches_numpy_random_weights():
    w, X, _ = net.random_problem(7, 300)
    prop = poa_b200.Proposer()
    prop.set_weights(w.astype(np.float32))
    _check_forward(prop, prop.get_weights().astype(np.float64), X.astype(np.float32))


@pytest.mark.parametrize("n", [1, 64, 300])
def test_backward_kernels_match_numpy_gradient(n):
    w, X, Y = net.random_problem(11 + n, n)
    prop = poa_b200.Proposer()
    prop.set_weights(w.astype(np.float32))
    w32 = prop.get_weights().astype(np.float64)
    loss, g = prop.gradient(X.astype(np.float32), Y.astype(np.float32))
    want_loss, want = net.loss_and_gradient(w32, X.astype(np.float32), Y.astype(np.float32), use_bf16=True)
    assert abs(loss - want_loss) <= 1e-3 * abs(want_loss) + 1e-6
    o = 0
    for name, shape in net.SHAPES:
        k = int(np.prod(shape))
        a, b = g[o:o + k].astype(np.float64), want[o:o + k]
        o += k
        err = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-12)
        assert err < 2e-2, (name, err)
