"""The surrogate's CPU oracle: its backward pass against finite differences.

With bf16 rounding switched off the oracle is plain fp64 arithmetic, so its
analytic gradients must match central differences of its loss (tolerance:
1e-4 relative, limited by the ReLU kinks and the step size)."""
import importlib

import numpy as np
import pytest

import surrogate_ref


def random_params(rng):
    p = {}

    def lin(name, K, N, bias=True):
        p[name + ".W"] = rng.standard_normal((K, N)) / np.sqrt(K)
        if bias:
            p[name + ".b"] = rng.standard_normal(N) * 0.1

    def mlp(name, K, N):
        lin(name + ".0", K, 128)
        lin(name + ".1", 128, 128)
        lin(name + ".2", 128, N)

    mlp("enc", 8, 128)
    for l in (1, 2):
        lin(f"hop{l}.edge.a", 128, 128, False)
        lin(f"hop{l}.edge.b", 128, 128, False)
        lin(f"hop{l}.edge.0", 16, 128)
        lin(f"hop{l}.edge.1", 128, 128)
        lin(f"hop{l}.edge.2", 128, 128)
        mlp(f"hop{l}.node", 256, 128)
    mlp("dec", 128, 4)
    return p


def random_graph(rng, n=12, E=40):
    f = rng.standard_normal((n, 8))
    xe = rng.standard_normal((E, 16))
    dst = np.sort(rng.integers(0, n, E))
    src = rng.integers(0, n, E)
    fluid = rng.random(n) < 0.7
    t = rng.standard_normal((n, 4))
    return f, xe, dst, src, fluid, t


@pytest.fixture
def exact_oracle():
    surrogate_ref.ROUND_BF16 = False
    yield surrogate_ref
    surrogate_ref.ROUND_BF16 = True
    importlib.reload(surrogate_ref)


def test_oracle_gradients_match_finite_differences(exact_oracle):
    S = exact_oracle
    rng = np.random.default_rng(0)
    p = random_params(rng)
    f, xe, dst, src, fluid, t = random_graph(rng)
    net = S.Net(p)
    _, _, g = net.loss_and_grads(f, xe, dst, src, fluid, t)
    for k in sorted(p):
        idx = tuple(rng.integers(0, s) for s in p[k].shape)
        old = p[k][idx]
        eps = 1e-6
        p[k][idx] = old + eps
        lp = net.loss_and_grads(f, xe, dst, src, fluid, t)[0]
        p[k][idx] = old - eps
        lm = net.loss_and_grads(f, xe, dst, src, fluid, t)[0]
        p[k][idx] = old
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[k][idx]) <= 1e-4 * max(1e-6, abs(fd) + abs(g[k][idx])), k


def test_bf16_rounding_is_nearest_even():
    import surrogate_ref as S

    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.0e38], np.float32)
    r = S.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == np.float32(1.0 + 2 ** -7)
    assert r[3] == -2.5
