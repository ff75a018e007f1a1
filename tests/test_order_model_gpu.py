"""Order model on the GPU: CUDA gradients against the numpy restatement, BF16
inference against FP32, training, and exactness of learned orders."""
import os

import numpy as np
import pytest

import matrixgraph_b200 as mg
from matrixgraph_b200 import order_model as OM
from oracle import mpnn_ref as R

pytestmark = pytest.mark.gpu

MODEL_DIR = os.path.join(os.path.dirname(mg.__file__), "data", "order_model") + "/"


@pytest.fixture(scope="module")
def setup():
    g = mg.chung_lu(3000, avg_deg=8, n_labels=6)
    dg = mg.DeviceGraph(g)
    qs = [mg.query_random(g, 3 + i % 5, 0.3, seed=70 + i) for i in range(6)]
    yield g, dg, qs
    dg.free()


def _samples(qs, rng):
    sq, sm, st = [], [], []
    for qi, q in enumerate(qs):
        order = OM.random_connected_order(q, rng)
        mask = 0
        for v in order:
            mask |= 1 << v
            sq.append(qi)
            sm.append(mask)
            st.append(float(rng.random() * 8))
    return np.array(sq), np.array(sm), np.array(st, dtype=np.float32)


def test_cuda_gradient_matches_numpy(setup):
    g, dg, qs = setup
    rng = np.random.default_rng(1)
    model = OM.OrderModel.create(seed=3)
    sq, sm, st = _samples(qs, rng)
    grad, loss, pred = model.grad(dg, qs, sq, sm, st)
    feats = [OM.features(dg, q) for q in qs]
    p = model.params().astype(np.float64)
    samples = list(zip(sq.tolist(), sm.tolist(), st.tolist()))
    want_loss, want_grad = R.loss_and_grad(p, samples, feats)
    assert abs(loss - want_loss) <= 1e-4 * max(1.0, abs(want_loss))
    scale = np.abs(want_grad).max()
    assert np.allclose(grad, want_grad, rtol=2e-3, atol=2e-5 * scale)
    Pd = R.unpack(p)
    for i, (q, m, _) in enumerate(samples):
        assert abs(pred[i] - R.forward(Pd, *feats[q], m)) <= 1e-3 * max(1.0, abs(pred[i]))
    model.free()


def test_bf16_inference_close_to_fp32(setup):
    g, dg, qs = setup
    rng = np.random.default_rng(2)
    model = OM.OrderModel.create(seed=4)
    sq, sm, st = _samples(qs, rng)
    _, _, fp32 = model.grad(dg, qs, sq, sm, st)
    bf16 = model.predict(dg, qs, sq, sm)
    assert np.allclose(bf16, fp32, rtol=5e-2, atol=5e-2 * np.abs(fp32).max())
    model.free()


def test_training_lowers_loss_and_orders_stay_exact(setup, tmp_path):
    g, dg, qs = setup
    train_q = [mg.query_random(g, 4 + i % 4, 0.3, seed=500 + i) for i in range(24)]
    (sq, sm, st), records = OM.record_prefix_counts(dg, train_q, n_random=4, budget=1 << 24,
                                                    seed=9)
    assert len(sq) > 100
    model = OM.OrderModel.create(seed=5)
    _, before, _ = model.grad(dg, train_q, sq, sm, st)
    model.train(dg, train_q, sq, sm, st, epochs=20, batch=256, lr=3e-3)
    _, final, _ = model.grad(dg, train_q, sq, sm, st)
    assert final < 0.5 * before, (before, final)
    # recorded prefix counts are the enumerator's own: P_k is the count
    for qi, od, c, rows in records:
        if c != 2 ** 64 - 1:
            assert rows[len(od)] == c
    # learned orders: valid permutations, exact counts, single == batch
    for q in qs + train_q[:10]:
        assert sorted(mg.plan_order(q, order="learned", graph=dg, model=model)) == list(range(q.n))
        assert dg.count(q, order="learned", model=model) == dg.count(q)
    batch = dg.batch_count(qs + train_q[:10], order="learned", model=model)
    assert batch.tolist() == [dg.count(q) for q in qs + train_q[:10]]
    model.save(str(tmp_path) + "/")
    again = OM.OrderModel.load(str(tmp_path) + "/")
    assert np.array_equal(again.params(), model.params())
    model.free()
    again.free()


def test_committed_model_loads_and_keeps_counts_exact(setup):
    g, dg, qs = setup
    if not os.path.exists(MODEL_DIR + "embedding.bin"):
        pytest.skip("no trained model committed")
    model = OM.OrderModel.load(MODEL_DIR)
    for q in qs:
        assert dg.count(q, order="learned", model=model) == dg.count(q)
    model.free()
