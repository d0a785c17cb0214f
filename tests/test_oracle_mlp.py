"""The warm-start network's CPU oracle checked against finite differences
(FP64, without BF16 rounding), so that it can serve as the reference for
the GPU gradients."""
import numpy as np

from oracle import mlp


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    nsites = 6
    p = (rng.standard_normal(mlp.n_params(nsites)) * 0.2).astype(np.float32).astype(np.float64)
    states = rng.integers(0, 1 << nsites, 9).astype(np.uint64)
    j2 = rng.uniform(0, 1, 9)
    tg = np.stack([rng.standard_normal(9), rng.choice([-1.0, 1.0], 9), rng.uniform(0.5, 1.5, 9)], 1)

    def f(q):
        # FP64 parameters, no rounding: evaluate the loss directly
        X = mlp.inputs(states, j2, nsites)
        W1, W2, W3, b1, b2, b3 = mlp.split(q, nsites)
        O = mlp.gelu(mlp.gelu(X @ W1.T + b1) @ W2.T + b2) @ W3.T + b3
        e = O[:, 0] - tg[:, 0]
        m = -tg[:, 1] * O[:, 1]
        return np.mean(tg[:, 2] * (e * e + 0.7 * np.log1p(np.exp(m))))

    def grad(q):
        X = mlp.inputs(states, j2, nsites)
        W1, W2, W3, b1, b2, b3 = mlp.split(q, nsites)
        Z1 = X @ W1.T + b1; H1 = mlp.gelu(Z1); Z2 = H1 @ W2.T + b2; H2 = mlp.gelu(Z2); O = H2 @ W3.T + b3
        n = len(states)
        e = O[:, 0] - tg[:, 0]
        m = -tg[:, 1] * O[:, 1]
        dO = np.stack([tg[:, 2] * 2 * e / n, tg[:, 2] * 0.7 / (1 + np.exp(-m)) * (-tg[:, 1]) / n], 1)
        dZ2 = (dO @ W3) * mlp.gelu_d(Z2)
        dZ1 = (dZ2 @ W2) * mlp.gelu_d(Z1)
        return np.concatenate([(dZ1.T @ X).ravel(), (dZ2.T @ H1).ravel(), (dO.T @ H2).ravel(),
                               dZ1.sum(0), dZ2.sum(0), dO.sum(0)])

    g = grad(p)
    # the oracle's own loss_grad (with rounding off) is the same function
    l2, g2 = mlp.loss_grad(p.astype(np.float32), states, j2, tg, nsites, 0.7, round_bf16=False)
    assert abs(l2 - f(p.astype(np.float32).astype(np.float64))) < 1e-12
    assert np.allclose(g2, grad(p.astype(np.float32).astype(np.float64)), rtol=1e-10, atol=1e-12)
    for k in rng.choice(p.size, 40, replace=False):
        h = 1e-6
        q1, q2 = p.copy(), p.copy()
        q1[k] += h
        q2[k] -= h
        fd = (f(q1) - f(q2)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k])), k


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 65504.0], np.float32)
    r = mlp.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0             # exactly halfway: rounds to the even neighbour
    assert r[2] == 1.0078125
    assert abs(r[3] + 3.140625) < 1e-12


def test_tanh_gelu_stays_close_to_the_gaussian_one():
    # Hendrycks & Gimpel's tanh form: max |error| about 4.7e-4 (near |z| = 2.7)
    z = np.linspace(-12.0, 12.0, 480001)
    assert np.abs(mlp.gelu(z) - mlp.gelu_exact(z)).max() < 5e-4
    h = 1e-6
    d = (mlp.gelu(z + h) - mlp.gelu(z - h)) / (2 * h)
    assert np.abs(d - mlp.gelu_d(z)).max() < 1e-7
