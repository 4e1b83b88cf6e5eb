"""The surrogate ΔASPL ranker (gg_surrogate_*).

CPU: the numpy restatement of its forward/backward (oracle/surrogate_ref.py) is
checked against finite differences, and its bf16 rounding against torch.
GPU: the CUDA forward and gradients are checked against that restatement
(same bf16 rounding of every product operand).  Tolerances: predictions within
1e-2 of the largest |prediction| (plus 1e-4); gradients with cosine similarity
> 0.999 and relative L2 error < 2e-2 -- the GPU accumulates in fp32 (in a
different order, with atomics), the restatement in float64.  Training on exact
ΔASPL labels must cut the loss and rank held-out swaps (Spearman > 0.3)."""
import numpy as np
import pytest

import graphgolf as G
import instances as I
import surrogate_ref as R

F = 5


def small_case(seed=0, n=40, d=4, P=24):
    adj = G.random_regular(n, d, seed + 3)
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, F)).astype(np.float32)
    sw = G.gen_swaps(adj, 0, P, seed + 7)
    t = rng.normal(size=P).astype(np.float32)
    return adj, X, sw, t


def init_params(seed=0):
    _, k = R.layout(F)
    rng = np.random.default_rng(seed)
    return (rng.normal(size=k) * 0.3).astype(np.float32)


def test_bf16_rounding_matches_torch():
    import torch
    x = np.random.default_rng(0).normal(size=10000).astype(np.float32) * 10
    want = torch.from_numpy(x).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(R.to_bf16(x), want)


def test_reference_backward_matches_finite_differences():
    adj, X, sw, t = small_case(1, n=16, d=3, P=6)
    net = R.Net(adj, X, bf16=False)
    p = init_params(1).astype(np.float64)
    loss, g, _ = net.loss_grad(p, sw, t)
    rng = np.random.default_rng(2)
    for i in rng.choice(len(p), 60, replace=False):
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        num = (net.loss_grad(pp, sw, t)[0] - net.loss_grad(pm, sw, t)[0]) / (2 * h)
        assert abs(num - g[i]) <= 1e-5 * max(1.0, abs(num)), (i, num, g[i])


@pytest.mark.gpu
def test_gpu_forward_and_gradient_match_reference():
    adj, X, sw, t = small_case(0, n=300, d=6, P=200)
    s = G.Surrogate(300, 6, F, seed=1)
    p = init_params(0)
    s.set_params(p)
    s.set_graph(adj, X)
    y = s.predict(sw)
    net = R.Net(adj, X, bf16=True)
    y_ref, _ = net.forward(p.astype(np.float64), sw)
    assert np.all(np.abs(y - y_ref) <= 1e-2 * np.abs(y_ref).max() + 1e-4)
    mask = (np.arange(len(sw)) % 5 != 0).astype(np.int32)
    g, loss = s.grad(sw, t, mask)
    loss_ref, g_ref, _ = net.loss_grad(p.astype(np.float64), sw, t, mask)
    assert abs(loss - loss_ref) <= 1e-2 * abs(loss_ref)
    o, _ = R.layout(F)
    for name, (off, shape) in o.items():
        a = g[off:off + int(np.prod(shape))].astype(np.float64)
        b = g_ref[off:off + int(np.prod(shape))]
        nb = np.linalg.norm(b)
        if nb < 1e-12:
            assert np.linalg.norm(a) < 1e-6
            continue
        cos = float(a @ b) / (np.linalg.norm(a) * nb)
        assert cos > 0.999 and np.linalg.norm(a - b) / nb < 2e-2, (name, cos)


def hist_features(batch, bid, K=4):
    h = batch.vertex_hist(bid, K).astype(np.float64)
    h = (h - h.mean(0)) / (h.std(0) + 1e-6)
    return np.concatenate([h, np.ones((len(h), 1))], axis=1).astype(np.float32)


@pytest.mark.gpu
def test_vertex_hist_is_distance_histogram():
    import oracle as O
    adj = G.random_regular(200, 4, 9)
    b = G.Batch(0)
    bid = b.add_base(adj)
    h = b.vertex_hist(bid, 5)
    for v in (0, 17, 123):
        r = O.bfs_pull(adj, np.array([v]))
        assert h[v].tolist() == [int(x) for x in r.level_counts[1:6]]


@pytest.mark.gpu
def test_training_on_exact_labels_learns_to_rank():
    n, d = 1024, 6
    adj = G.random_regular(n, d, 5)
    b = G.Batch(0)
    bid = b.add_base(adj)
    base_total = int(b.eval(np.array([(bid, -1, -1, -1, -1, 0)], dtype=G.SWAP_DTYPE))[0]["total"])
    sw = G.gen_swaps(adj, bid, 3000, 6)
    res = b.eval(sw)
    delta = (res["total"].astype(np.float64) - base_total) / (n * (n - 1))
    ok = res["connected"] == 1
    mu, sd = delta[ok].mean(), delta[ok].std()
    target = ((delta - mu) / sd).astype(np.float32)
    train, test = np.arange(2000), np.arange(2000, 3000)
    s = G.Surrogate(n, d, 5, seed=3)
    s.set_graph(adj, hist_features(b, bid))
    first = None
    for it in range(300):
        idx = train[(it * 256 + np.arange(256)) % len(train)]
        loss = s.train(sw[idx], target[idx], lr=2e-3, mask=ok[idx].astype(np.int32))
        first = loss if first is None else first
    assert loss < 0.5 * first
    pred = s.predict(sw[test])
    from scipy.stats import spearmanr
    rho = spearmanr(pred[ok[test]], target[test][ok[test]]).correlation
    assert rho > 0.3, rho
