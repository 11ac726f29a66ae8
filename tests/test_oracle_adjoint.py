"""The FP64 adjoint reference (oracle/dg_oracle_adjoint.c) against central finite
differences and a direct numpy evaluation of the loss (CPU)."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def problem():
    rng = np.random.default_rng(7)
    vocab, d, n_pairs, batch, neg = 300, 16, 2000, 21, 5
    zipf = 1.0 / np.arange(1, vocab + 1)
    zipf /= zipf.sum()
    inputs = rng.choice(vocab, size=n_pairs, p=zipf).astype(np.uint32)
    outputs = rng.choice(vocab, size=n_pairs, p=zipf).astype(np.uint32)
    n_batches = (n_pairs + batch - 1) // batch
    negatives = rng.choice(vocab, size=n_batches * neg, p=zipf).astype(np.uint32)
    v = rng.normal(size=(vocab, d)) * 0.3
    u = rng.normal(size=(vocab, d)) * 0.3
    return v, u, inputs, outputs, negatives, batch, neg


def _numpy_loss(v, u, inputs, outputs, negatives, batch, neg):
    sp = lambda x: np.logaddexp(0.0, x)  # noqa: E731  softplus
    s = np.einsum("ij,ij->i", v[inputs], u[outputs])
    total = sp(-s).sum()
    b = np.arange(inputs.size) // batch
    for k in range(neg):
        w = negatives[b * neg + k]
        total += sp(np.einsum("ij,ij->i", v[inputs], u[w])).sum()
    return total


def test_loss_matches_numpy(oracle, problem):
    v, u, inputs, outputs, negatives, batch, neg = problem
    loss, _, _ = oracle.sgns_loss_grad(v, u, inputs, outputs, negatives, batch, neg, grad=False)
    assert loss == pytest.approx(_numpy_loss(v, u, inputs, outputs, negatives, batch, neg), rel=1e-12)


def test_gradient_matches_central_differences(oracle, problem):
    v, u, inputs, outputs, negatives, batch, neg = problem
    _, gi, go = oracle.sgns_loss_grad(v, u, inputs, outputs, negatives, batch, neg)
    h = 1e-3
    rng = np.random.default_rng(0)
    for table, rows, grad in [(0, v, gi), (1, u, go)]:
        used = np.unique(inputs if table == 0 else np.concatenate([outputs, negatives]))
        for row in list(used[:3]) + list(rng.choice(used, 5)):
            c = int(rng.integers(rows.shape[1]))
            plus, minus = rows.copy(), rows.copy()
            plus[row, c] += h
            minus[row, c] -= h
            args = (inputs, outputs, negatives, batch, neg)
            if table == 0:
                lp, _, _ = oracle.sgns_loss_grad(plus, u, *args, grad=False, only=(0, int(row)))
                lm, _, _ = oracle.sgns_loss_grad(minus, u, *args, grad=False, only=(0, int(row)))
            else:
                lp, _, _ = oracle.sgns_loss_grad(v, plus, *args, grad=False, only=(1, int(row)))
                lm, _, _ = oracle.sgns_loss_grad(v, minus, *args, grad=False, only=(1, int(row)))
            fd = (lp - lm) / (2 * h)
            assert fd == pytest.approx(grad[row, c], rel=1e-5, abs=1e-7)


def test_restricted_sum_gives_the_same_differences(oracle, problem):
    v, u, inputs, outputs, negatives, batch, neg = problem
    row, c, h = int(outputs[0]), 3, 1e-3
    plus, minus = u.copy(), u.copy()
    plus[row, c] += h
    minus[row, c] -= h
    args = (inputs, outputs, negatives, batch, neg)
    full = (oracle.sgns_loss_grad(v, plus, *args, grad=False)[0] -
            oracle.sgns_loss_grad(v, minus, *args, grad=False)[0]) / (2 * h)
    part = (oracle.sgns_loss_grad(v, plus, *args, grad=False, only=(1, row))[0] -
            oracle.sgns_loss_grad(v, minus, *args, grad=False, only=(1, row))[0]) / (2 * h)
    assert part == pytest.approx(full, rel=1e-6, abs=1e-8)


def test_pairs_from_walks_window_rule():
    from distger.adjoint import pairs_from_walks
    verts = np.arange(12, dtype=np.uint32)
    offsets = np.array([0, 12], dtype=np.uint64)
    v2w = np.arange(12, dtype=np.int32)
    table = np.arange(12, dtype=np.int32)
    inputs, outputs, negs = pairs_from_walks(offsets, verts, v2w, table, window=3, batch=4, negative=2,
                                             n_pairs=10_000, seed=3)
    assert inputs.size == outputs.size and inputs.size > 0
    dist = np.abs(inputs.astype(int) - outputs.astype(int))
    assert dist.min() >= 1 and dist.max() <= 3
    assert negs.size == ((inputs.size + 3) // 4) * 2
