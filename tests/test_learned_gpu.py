"""The learned bucket assigners: GPU forward/backward kernels checked against a
float64 CPU restatement (analytic and finite differences), and what training
gains over the sampled-pivot method."""
import numpy as np
import pytest

import ggms_b200 as G
import ggms_oracle as orc
from ggms_b200 import datagen as D
from conftest import to_device

pytestmark = pytest.mark.gpu


def softplus(v):
    return np.logaddexp(0.0, v)


def sigmoid(v):
    return 1.0 / (1.0 + np.exp(-v))


# ---------------------------------------------------------------- PL-CDF
def pl_loss_cpu(keys, knots, theta):
    """Brute force over every sample (float64), same u as the device (float32 division)."""
    S = len(keys)
    M = len(knots) - 1
    d = softplus(theta.astype(np.float64))
    P = np.concatenate([[0.0], np.cumsum(d)])[:-1]
    D_ = d.sum()
    j = np.searchsorted(knots, keys, side="right") - 1
    j = np.clip(j, 0, M - 1)
    num = (keys - knots[j]).astype(np.float32)
    den = (knots[j + 1] - knots[j]).astype(np.float32)
    u = np.minimum(num / den, np.float32(1.0)).astype(np.float64)
    F = (P[j] + u * d[j]) / D_
    y = (np.arange(S) + 0.5) / S
    return np.mean((F - y) ** 2)


def pl_grad_cpu(keys, knots, theta):
    S = len(keys)
    M = len(knots) - 1
    th = theta.astype(np.float64)
    d = softplus(th)
    P = np.concatenate([[0.0], np.cumsum(d)])[:-1]
    D_ = d.sum()
    j = np.clip(np.searchsorted(knots, keys, side="right") - 1, 0, M - 1)
    u = np.minimum((keys - knots[j]).astype(np.float32) / (knots[j + 1] - knots[j]).astype(np.float32),
                   np.float32(1.0)).astype(np.float64)
    F = (P[j] + u * d[j]) / D_
    r = F - (np.arange(S) + 0.5) / S
    # dF_i/d delta_t = (1{t<j_i} + u_i 1{t=j_i} - F_i) / D
    R = np.bincount(j, weights=r, minlength=M)
    U = np.bincount(j, weights=r * u, minlength=M)
    after = np.concatenate([np.cumsum(R[::-1])[::-1][1:], [0.0]])
    Q = np.sum(r * F)
    gd = 2.0 / (S * D_) * (after + U - Q)
    return gd * sigmoid(th)


@pytest.mark.parametrize("gen", ["normal_f32", "mixture8_f32", "lognormal_f32", "distinct256_f32"])
def test_pl_gradient_matches_cpu(gen):
    v = D.VALUE_GENERATORS[gen](1 << 16, 5)
    keys = np.sort(orc.keys(v))
    g = np.random.default_rng(1)
    theta = (0.5413 + 0.3 * g.standard_normal(G.PL_KNOTS)).astype(np.float32)
    loss, grad, knots = G.diag_pl_gradient(keys, theta)
    M = len(grad)
    assert 16 <= M <= G.PL_KNOTS
    th = theta[:M]
    ref_loss = pl_loss_cpu(keys, knots, th)
    ref_grad = pl_grad_cpu(keys, knots, th)
    np.testing.assert_allclose(loss, ref_loss, rtol=2e-3, atol=1e-9)
    tol = 1e-3 * np.max(np.abs(ref_grad))
    np.testing.assert_allclose(grad, ref_grad, rtol=5e-3, atol=tol)
    # finite differences of the brute-force loss on a few coordinates
    for t in g.choice(M, size=6, replace=False):
        h = 1e-3
        e = np.zeros(M)
        e[t] = h
        fd = (pl_loss_cpu(keys, knots, th + e) - pl_loss_cpu(keys, knots, th - e)) / (2 * h)
        assert abs(fd - ref_grad[t]) <= 2e-2 * abs(ref_grad[t]) + 1e-3 * np.max(np.abs(ref_grad))


# ---------------------------------------------------------------- MLP-CDF
P_V1, P_C1, P_V2, P_C2, P_V3, P_C3 = 0, 32, 64, 1088, 1120, 1152


def mlp_forward_backward_cpu(x, t, p):
    x = x.astype(np.float64)
    t = t.astype(np.float64)
    p = p.astype(np.float64)
    V1, c1 = p[P_V1:P_C1], p[P_C1:P_V2]
    V2, c2 = p[P_V2:P_C2].reshape(32, 32), p[P_C2:P_V3]
    V3, c3 = p[P_V3:P_C3], p[P_C3]
    w1, W2, w3 = softplus(V1), softplus(V2), softplus(V3)
    h1 = np.tanh(np.outer(x, w1) + c1)            # Q x 32
    h2 = np.tanh(h1 @ W2.T + c2)                  # Q x 32
    z = h2 @ w3 + c3
    # the loss is taken on the sigmoid's argument: targets in logit units
    tl = np.log(t) - np.log1p(-t)
    Q = len(x)
    loss = np.mean((z - tl) ** 2)
    dz = 2 * (z - tl) / Q
    gw3 = h2.T @ dz
    gc3 = dz.sum()
    da2 = np.outer(dz, w3) * (1 - h2 ** 2)
    gW2 = da2.T @ h1
    gc2 = da2.sum(0)
    da1 = (da2 @ W2) * (1 - h1 ** 2)
    gw1 = da1.T @ x
    gc1 = da1.sum(0)
    g = np.concatenate([gw1 * sigmoid(V1), gc1, (gW2 * sigmoid(V2)).ravel(), gc2,
                        gw3 * sigmoid(V3), [gc3]])
    return loss, g


def test_mlp_gradient_matches_cpu():
    g = np.random.default_rng(3)
    x = np.sort(g.random(1024)).astype(np.float32)
    t = np.clip((np.arange(1024) + 0.5) / 1024 + 0.05 * np.sin(7 * x), 1e-3, 1 - 1e-3).astype(np.float32)
    p = (0.3 * g.standard_normal(1153)).astype(np.float32)
    p[P_V2:P_C2] -= 3.0
    loss, grad = G.diag_mlp_gradient(x, t, p)
    ref_loss, ref_grad = mlp_forward_backward_cpu(x, t, p)
    np.testing.assert_allclose(loss, ref_loss, rtol=1e-4)
    tol = 2e-4 * np.max(np.abs(ref_grad))
    np.testing.assert_allclose(grad, ref_grad, rtol=2e-3, atol=tol)
    for i in g.choice(1153, size=8, replace=False):
        h = 1e-4
        e = np.zeros(1153)
        e[i] = h
        fd = (mlp_forward_backward_cpu(x, t, p + e)[0] - mlp_forward_backward_cpu(x, t, p - e)[0]) / (2 * h)
        assert abs(fd - ref_grad[i]) <= 1e-3 * abs(ref_grad[i]) + 1e-6 * np.max(np.abs(ref_grad)) + 1e-9


# ---------------------------------------------------------------- what training gains
@pytest.mark.parametrize("gen", ["mixture8_f32", "lognormal_f32"])
@pytest.mark.parametrize("kind", [G.ASSIGNER_LEARNED_PL, G.ASSIGNER_LEARNED_MLP])
def test_training_improves_balance(gen, kind):
    v = D.VALUE_GENERATORS[gen](1 << 16, 7)
    keys = np.sort(orc.keys(v))
    r = G.diag_fit(keys, kind)
    if kind == G.ASSIGNER_LEARNED_PL:
        # training never ends worse than its quantile init (keep-best), and the
        # learned model's buckets are more even than the 17 sampled pivots'
        assert r["loss_after"] <= r["loss_before"]
        assert r["imbalance_model"] < r["imbalance_sampled"], r
    else:
        # the MLP reaches a small error (mean squared, logit units), and its
        # buckets, measured on the same sample, are more even than the 17
        # sampled pivots'
        assert r["loss_after"] < 1e-2, r
        assert r["imbalance_model"] < r["imbalance_sampled"], r


@pytest.mark.parametrize("gen,seed", [("mixture8_f32", 31), ("lognormal_f32", 32)])
def test_learned_needs_less_refinement(ctx, gen, seed):
    n = 1 << 26
    v = D.VALUE_GENERATORS[gen](n, seed)
    ks = D.ks_uniform(n, 1 << 12, 33)
    exp = orc.cpu_multiselect(v, ks)
    d = to_device(v)
    res = {}
    for a in (G.ASSIGNER_SAMPLED, G.ASSIGNER_LEARNED_PL, G.ASSIGNER_LEARNED_MLP):
        out, st = G.select(ctx, d.data_ptr(), n, ks, np.float32, assigner=a, stats=True)
        np.testing.assert_array_equal(out.view(np.uint32), exp.view(np.uint32))
        res[a] = st
    samp, pl, mlp = res[G.ASSIGNER_SAMPLED], res[G.ASSIGNER_LEARNED_PL], res[G.ASSIGNER_LEARNED_MLP]
    assert pl["assigner_used"] == "learned_pl"
    assert pl["bucket_max_over_mean"] < samp["bucket_max_over_mean"]
    assert pl["candidates"] <= samp["candidates"]
    # the MLP, when its fit is accepted, also beats the sampled pivots on the
    # whole input: more even level-0 buckets and no more candidates
    if mlp["assigner_used"] == "learned_mlp":
        assert mlp["bucket_max_over_mean"] < samp["bucket_max_over_mean"], (mlp, samp)
        assert mlp["candidates"] <= samp["candidates"], (mlp, samp)
