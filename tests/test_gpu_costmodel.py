"""GPU: the learned cost model (ultraprecise_costmodel.h).

* Its forward kernel and its backward pass (the training kernel run without
  the update) against the float64 restatement oracle/costmodel_ref.py.
* Training by the library's kernels fits a known smooth function.
* Ablation on measured kernel times: trained on launches of the training
  shapes, the model chooses threads per value for held-out shapes (other
  precisions and expressions), and its choices run no slower in total than
  the width rule's (cooperative from 96 limbs for division-free expressions),
  the method without the model; with the model set as the default,
  up_module_compile follows its choice.
"""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import costmodel_ref as ref
from ultraprecise_b200 import codec, costmodel, runtime, workloads

pytestmark = pytest.mark.gpu


def _identity_norm():
    return np.concatenate([np.zeros(16), np.ones(16), [0.0, 1.0]]).astype(np.float32)


def test_forward_matches_reference():
    rng = np.random.default_rng(1)
    m = costmodel.CostModel(seed=5)
    p = rng.normal(0, 0.25, costmodel.PARAMS).astype(np.float32)
    m.set_params(p, _identity_norm())
    X = rng.normal(0, 1, (300, 16)).astype(np.float32)
    got = m.predict(X)
    exp, _ = ref.forward(p, X)
    np.testing.assert_allclose(got, exp, rtol=1e-4, atol=1e-4 * float(np.max(np.abs(exp))))


@pytest.mark.parametrize("n", [1, 37, 128])
def test_gradients_match_reference(n):
    rng = np.random.default_rng(n)
    m = costmodel.CostModel(seed=n)
    p = rng.normal(0, 0.25, costmodel.PARAMS).astype(np.float32)
    m.set_params(p, _identity_norm())
    X = rng.normal(0, 1, (n, 16)).astype(np.float32)
    y = rng.normal(0, 1, n).astype(np.float32)
    g, loss = m.gradients(X, y)
    eloss, eg = ref.loss_and_grads(p, X, y)
    assert abs(loss - eloss) <= 1e-4 * max(1.0, eloss)
    scale = float(np.max(np.abs(eg)))
    np.testing.assert_allclose(g, eg, rtol=1e-3, atol=2e-4 * scale)


def test_training_fits_a_smooth_function():
    rng = np.random.default_rng(11)
    # 12 of the 16 inputs are noise: enough samples that a fit generalises
    X = rng.uniform(-1, 1, (2048, 16)).astype(np.float32)
    y = (np.sin(2 * X[:, 0]) + 0.5 * X[:, 1] * X[:, 2] + 0.3 * X[:, 3] ** 2).astype(np.float32)
    m = costmodel.CostModel(seed=2)
    loss = m.train(X, y, epochs=120, batch=64, lr=3e-3, seed=4)
    assert loss < 0.02, loss
    Xt = rng.uniform(-1, 1, (200, 16)).astype(np.float32)
    yt = np.sin(2 * Xt[:, 0]) + 0.5 * Xt[:, 1] * Xt[:, 2] + 0.3 * Xt[:, 3] ** 2
    assert float(np.mean((m.predict(Xt) - yt) ** 2)) < 0.05 * float(np.var(yt)) + 1e-3


def _eval_times(shape, rows):
    """Measured ms of every threads-per-value choice of a held-out shape."""
    name, e, cols = shape
    p = cols[0].precision
    data = [runtime.DeviceColumn(runtime.gen_digits(rows, p, 900 + k, nonzero=True), p, cols[k].scale)
            for k in range(len(cols))]
    out = {}
    for t in costmodel.TPV_CHOICES:
        mod = runtime.compile_expr(e, cols, threads_per_value=t)
        out[t] = costmodel.time_launch(mod, data, rows, reps=5)
    return out


def test_model_beats_or_matches_the_width_rule_on_held_out_shapes():
    X, y, recs, secs = costmodel.collect_samples(workloads.costmodel_train_shapes(), (1 << 18, 1 << 20))
    assert len(y) >= 200
    nets = []
    for k in range(5):  # an ensemble: single networks disagree where the data is thin
        net = costmodel.CostModel(seed=3 + k)
        loss = net.train(X, y, epochs=400, batch=64, lr=3e-3, seed=5 + k)
        assert loss < 0.2, loss
        nets.append(net)
    m = nets[0]
    for net in nets[1:]:
        m.add_member(net)
    rows = 1 << 20
    tot = {"model": 0.0, "rule": 0.0, "best": 0.0}
    for shape in workloads.costmodel_eval_shapes():
        name, e, cols = shape
        times = _eval_times(shape, rows)
        costmodel.CostModel.clear_default()
        rule_t = runtime.compile_expr(e, cols).threads_per_value
        model_t, _ = m.choose_tpv(e, cols, rows)
        tot["model"] += times[model_t]
        tot["rule"] += times[rule_t]
        tot["best"] += min(times.values())
    print("held-out totals (ms):", {k: round(v, 3) for k, v in tot.items()})
    assert tot["model"] <= 1.05 * tot["rule"], tot
    # as the default model, up_module_compile follows its choice
    e, cols = workloads.costmodel_eval_shapes()[-1][1:]
    want, _ = m.choose_tpv(e, cols, 1 << 20)
    m.set_default()
    try:
        assert runtime.compile_expr(e, cols).threads_per_value == want
    finally:
        costmodel.CostModel.clear_default()


def test_ensemble_averages_members_and_guard_keeps_the_rule():
    rng = np.random.default_rng(5)
    X = rng.uniform(-1, 1, (64, 16)).astype(np.float32)
    a, b = costmodel.CostModel(seed=11), costmodel.CostModel(seed=12)
    ens = costmodel.CostModel(seed=13)
    ens.set_params(*a.params())
    ens.add_member(b)
    np.testing.assert_allclose(ens.predict(X), (a.predict(X) + b.predict(X)) / 2, rtol=1e-5, atol=1e-5)
    # a guard of 99.9999 %: the width rule's choice unless a 10^6-fold saving is predicted
    for name, e, cols in workloads.costmodel_eval_shapes():
        ens.set_guard(0.999999)
        t, _ = ens.choose_tpv(e, cols, 1 << 20)
        assert t == costmodel.rule_tpv(e, cols), name
    ens.set_guard(0.0)
