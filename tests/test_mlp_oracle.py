"""The closure network's CPU oracle: its analytic gradient against central
finite differences (float64; tolerance 1e-6 relative)."""
import numpy as np

from oracle import mlp_oracle


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    nin, nhid, nout, n = 4, 6, 3, 7
    npar = nhid * nin + nhid + nhid * nhid + nhid + nout * nhid + nout
    # parameters exactly representable in bfloat16 so the rounding is the identity
    p = mlp_oracle.bf16_round(rng.standard_normal(npar).astype(np.float32) * 0.5).astype(np.float32)
    x = rng.standard_normal((n, nin))
    t = rng.standard_normal((n, nout))
    loss, g = mlp_oracle.loss_grad(p, x, t, nin, nhid, nout)
    # perturb only the biases (float32, not rounded) and compare
    o = 0
    idx = []
    for size, is_bias in ((nhid * nin, False), (nhid, True), (nhid * nhid, False), (nhid, True),
                          (nout * nhid, False), (nout, True)):
        if is_bias:
            idx += list(range(o, o + size))
        o += size
    for i in idx:
        h = 1e-3
        pp, pm = p.astype(np.float64).copy(), p.astype(np.float64).copy()
        pp[i] += h
        pm[i] -= h
        lp, _ = mlp_oracle.loss_grad(pp.astype(np.float32), x, t, nin, nhid, nout)
        lm, _ = mlp_oracle.loss_grad(pm.astype(np.float32), x, t, nin, nhid, nout)
        num = (lp - lm) / (np.float32(p[i] + h) - np.float32(p[i] - h))
        assert abs(num - g[i]) <= 1e-6 * max(1.0, abs(g[i])) + 1e-6, (i, num, g[i])


def test_bf16_round_is_nearest_even():
    a = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 65504.0], np.float32)
    r = mlp_oracle.bf16_round(a)
    assert r[0] == 1.0
    assert r[1] == 1.0                     # tie (1 + 2^-8) rounds to even
    assert r[2] == 1.0078125               # above the tie rounds up
    assert abs(r[3] - (-3.140625)) < 1e-12
    assert r[4] == 65536.0
