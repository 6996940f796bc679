"""The CPU restatement of the path-guiding network (oracle/guide.py) checked
against the mathematics it restates: BF16 rounding known answers, a
normalised vMF mixture, the analytic output gradient against finite
differences, and the hash-grid indexing bounds."""
import numpy as np

from oracle import guide as G


def test_bf16_round_to_nearest_even():
    x = np.array([1.0, 1.00390625, 1.01171875, -2.5, 3.0e38, 1e-40], np.float32)
    r = G.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                  # halfway between 1 and 1 + 2^-7: the even one
    assert r[2] == np.float32(1.015625)  # halfway between 1 + 2^-7 and 1 + 2^-6: the even one
    assert r[3] == -2.5
    assert np.isfinite(r[4]) and abs(r[4] / 3.0e38 - 1) < 1 / 128
    assert (G.bf16(r) == r).all()


def _fib_sphere(n):
    i = np.arange(n) + 0.5
    z = 1 - 2 * i / n
    phi = np.pi * (1 + 5 ** 0.5) * i
    s = np.sqrt(1 - z * z)
    return np.stack([s * np.cos(phi), s * np.sin(phi), z], 1)


def test_mixture_density_integrates_to_one():
    rng = np.random.default_rng(3)
    o = rng.normal(0, 1.5, (6, 41))
    o[:, 3::5][:, :8] = rng.uniform(-4, 5, (6, 8))       # log κ from broad to sharp lobes
    D = _fib_sphere(400_000)
    for r in range(len(o)):
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        p = G.guide_pdf(np.repeat(o[r:r + 1], len(D), 0), np.repeat(n[None], len(D), 0), D)
        assert abs(p.mean() * 4 * np.pi - 1) < 2e-3


def test_output_gradient_matches_finite_differences():
    """Lobe outputs: the derivative of −w·log p_vmf; the α output: of
    −w·log p_mix."""
    rng = np.random.default_rng(5)
    n = 8
    o = rng.normal(0, 1, (n, 41))
    o[:, 3::5][:, :8] = rng.uniform(-3, 4, (n, 8))
    N = np.tile([0.0, 0.0, 1.0], (n, 1))
    D = rng.normal(size=(n, 3))
    D[:, 2] = np.abs(D[:, 2])
    D /= np.linalg.norm(D, axis=1, keepdims=True)
    w = rng.uniform(0.1, 2.0, n)
    _, g = G.loss_grad(o, N, D, w, 1.0)

    def lobe_loss(oo):                      # −w·log p_vmf: the lobes' objective
        mu, k, pi, _, _ = G.mixture(oo)
        c = np.einsum("nlj,nj->nl", mu, D)
        return -w * np.log((pi * G.vmf_norm(k) * np.exp(k * (c - 1))).sum(1))

    def mix_loss(oo):                       # −w·log p_mix: α's objective
        return G.loss_grad(oo, N, D, w, 1.0)[0]
    h = 1e-6
    for k in range(41):
        op, om = o.copy(), o.copy()
        op[:, k] += h
        om[:, k] -= h
        f = mix_loss if k == 40 else lobe_loss
        fd = (f(op) - f(om)) / (2 * h)
        assert np.allclose(g[:, k], fd, rtol=1e-4, atol=1e-6), k


def test_grid_indices_stay_in_the_table():
    res = G.resolutions()
    assert res[0] == 16 and 3900 < res[-1] < 4300
    rng = np.random.default_rng(1)
    for r in res:
        c = rng.integers(0, r + 1, (1000, 3)).astype(np.uint32)
        idx = G.grid_index(r, c[:, 0], c[:, 1], c[:, 2])
        assert idx.max() < G.TSIZE
        if (r + 1) ** 3 <= G.TSIZE:                       # dense levels are one-to-one
            assert len(np.unique(idx)) == len(np.unique(c, axis=0))


def test_adam_first_step_moves_by_the_learning_rate():
    p = np.zeros(5, np.float32)
    g = np.array([1e-3, -2.0, 0.0, 5e-7, -1e-5], np.float32)
    p1, m, v = G.adam(p, np.zeros(5, np.float32), np.zeros(5, np.float32), g, 1)
    assert np.allclose(p1[[0, 1, 4]], [-1e-2, 1e-2, 1e-2], rtol=1e-3)
    assert p1[2] == 0.0
