"""CPU: the cost model's host side — features of expression launches and the
float64 restatement of its network (oracle/costmodel_ref.py) that the GPU
tests check the kernels against; the restatement's own gradients are checked
here by central finite differences."""
import numpy as np

from oracle import costmodel_ref as ref
from ultraprecise_b200 import abi, costmodel, workloads
from ultraprecise_b200 import expr as E


def test_parameter_count_matches_the_header():
    assert costmodel.PARAMS == 16 * 64 + 64 + 64 * 64 + 64 + 64 + 1 == 5313


def test_features_follow_the_launch():
    a, b, c = E.col(0), E.col(1), E.col(2)
    cols = [E.ColType(300, 75)] * 3
    f1, ok = costmodel.features(a * b + c, cols, 1, 1 << 20)
    f8, _ = costmodel.features(a * b + c, cols, 8, 1 << 20)
    f1s, _ = costmodel.features(a * b + c, cols, 1, 1 << 16)
    assert ok
    assert f1[1] == 0.0 and f8[1] == 3.0                  # log2 threads per value
    assert f8[13] < f1[13]                                # work per thread shrinks with the group
    assert f1s[0] == 16.0 and f1[0] == 20.0               # log2 rows
    assert f1[4] > 0 and f1[7] == 0                       # multiply work, no division
    fd, _ = costmodel.features(a / b, cols[:2], 1, 1 << 20)
    assert fd[11] == 1.0 and fd[5] > 0 and fd[7] == 1     # division work


def test_nullable_expressions_have_no_cooperative_form():
    a, b = E.col(0), E.col(1)
    _, ok = costmodel.features(a * b, [E.ColType(300, 75, nullable=True), E.ColType(300, 75)], 1, 1000)
    assert not ok


def test_every_cost_model_shape_has_features():
    for name, e, cols in workloads.costmodel_train_shapes() + workloads.costmodel_eval_shapes():
        for t in costmodel.TPV_CHOICES:
            f, ok = costmodel.features(e, cols, t, 1 << 18)
            assert ok and np.all(np.isfinite(f)), name


def test_bad_threads_per_value_is_rejected():
    lib = abi.load()
    b = E.build([E.col(0) * E.col(1)], [E.ColType(38, 9)] * 2)
    E.derive_types(b)
    out = np.zeros(16, dtype=np.float32)
    st = lib.up_costmodel_expr_features(b.nodes, b.n_nodes, b.roots[0], b.col_types, b.n_cols, 3, 100,
                                        out.ctypes.data_as(abi.C.c_void_p), None)
    assert st == abi.UP_ERR_INVALID_ARG


def test_reference_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    p = rng.normal(0, 0.3, costmodel.PARAMS)
    X = rng.normal(0, 1, (24, 16))
    y = rng.normal(0, 1, 24)
    _, g = ref.loss_and_grads(p, X, y)
    h = 1e-6
    for i in list(range(0, costmodel.PARAMS, 97)) + [costmodel.PARAMS - 1]:
        e = np.zeros_like(p)
        e[i] = h
        num = (ref.loss_and_grads(p + e, X, y)[0] - ref.loss_and_grads(p - e, X, y)[0]) / (2 * h)
        assert abs(num - g[i]) <= 1e-6 + 1e-5 * abs(num), i


def test_width_rule_and_batch_candidates():
    """The automatic threads per value without a model (the width rule) and
    the group sizes the measured batch policy times."""
    from ultraprecise_b200 import batch, workloads
    e, cols = workloads.sweep_expr(600, "mad")
    assert costmodel.rule_tpv(e, cols) == 16          # 127 limbs: 16 threads of 8 limbs
    e, cols = workloads.sweep_expr(150, "mad")
    assert costmodel.rule_tpv(e, cols) == 1           # below the cooperative width
    e, cols = workloads.sweep_expr(600, "div")
    assert costmodel.rule_tpv(e, cols) == 1           # divisions: one thread per value
    a, b = E.col(0), E.col(1)
    assert costmodel.rule_tpv(a * b, [E.ColType(600, 150, nullable=True), E.ColType(600, 150)]) == 1
    e, cols = workloads.sweep_expr(600, "mad")
    cand = batch.tpv_candidates(batch.TaskSpec(e, cols, -1))
    assert cand[0] == 1 and set(cand[1:]) <= {2, 4, 8, 16, 32} and 16 in cand
    assert batch.tpv_candidates(batch.TaskSpec(e, cols, 1)) == [1]   # aggregates: one thread
    e, cols = workloads.sweep_expr(38, "mad")
    assert batch.tpv_candidates(batch.TaskSpec(e, cols, -1)) == [1]  # narrow: one thread
