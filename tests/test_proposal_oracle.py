"""The CPU oracle of the learned support proposal (oracle/mlp_oracle.py),
pinned on its own: analytic gradients against central finite differences
(float64, no BF16 rounding), BF16 rounding against numpy's definition, and
the restricted pursuit against the full oracle OMP when every atom is a
candidate."""

import numpy as np
import pytest


@pytest.fixture(scope="module")
def mlp():
    from ksvd_loader import load_oracle
    load_oracle()
    import mlp_oracle
    return mlp_oracle


def test_bf16_rounding(mlp):
    x = np.array([1.0, 1.00390625, 1.005859375, -3.3, 0.0, 1e-30, 65504.0], np.float32)
    r = mlp.bf16(x)
    # values exactly representable stay, others go to the nearest BF16 (8-bit significand)
    assert r[0] == 1.0 and r[1] == 1.0  # 1 + 2^-8 is a tie: to even (1.0)
    assert r[2] == 1.0078125            # 1 + 1.5 * 2^-8 rounds up
    for v, q in zip(x, r):
        assert abs(q - float(v)) <= abs(float(v)) * 2.0 ** -8 + 1e-45


def test_gradient_finite_differences(mlp):
    rng = np.random.default_rng(3)
    n, K, B = 16, 24, 8
    P = mlp.num_params(n, K)
    params = rng.normal(scale=0.05, size=P)
    Y = rng.normal(loc=100.0, scale=30.0, size=(B, n)).astype(np.float32)
    sup = rng.integers(-1, K, size=(B, 5)).astype(np.int32)
    loss, g = mlp.loss_grad(params, Y, sup, K, emulate=False)
    assert g.shape == (P,)
    picks = rng.choice(P, size=40, replace=False)
    # also one entry of every block
    o = np.cumsum([0, 512 * n, 512, 512 * 512, 512, K * 512])
    picks = np.concatenate([picks, o + 3])
    h = 1e-5
    for i in picks:
        e = np.zeros(P)
        e[i] = h
        lp, _ = mlp.loss_grad(params + e, Y, sup, K, emulate=False)
        lm, _ = mlp.loss_grad(params - e, Y, sup, K, emulate=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (i, fd, g[i])


def test_restricted_with_all_candidates_is_full_omp(mlp, oracle, synth):
    img = synth.add_gaussian(synth.clean_image(48, 5), 20.0, 5)
    Y = oracle.extract_patches(img, 8, 8, 2, 2)
    D = oracle.init_dictionary(Y, 32, int_norm=True, dtype=np.float64)
    Ys = Y[:300]
    cand = np.tile(np.arange(32, dtype=np.int32), (Ys.shape[0], 1))
    ri, rc, _ = mlp.omp_restricted(Ys, D, cand, 5)
    fi, fc = oracle.omp(Ys.astype(np.float64), D, 5)
    assert np.mean(np.all(ri == fi, axis=1)) >= 0.999
    m = np.all(ri == fi, axis=1)
    np.testing.assert_allclose(rc[m], fc[m], rtol=1e-7, atol=1e-7)


def test_top_candidates_order(mlp):
    Z = np.array([[0.1, 0.5, 0.5, -1.0, 2.0]])
    np.testing.assert_array_equal(mlp.top_candidates(Z, 3), [[4, 1, 2]])
