"""CPU checks of the radiance-cache restatement (oracle/mlp_ref.py): the
analytic fp64 gradient against central finite differences, the bf16-rounded
network against the exact one, and the encoding's range and layout."""
import numpy as np


def _data(rng, n, extent=16.0):
    q = np.zeros((n, 9), np.float32)
    q[:, :3] = rng.uniform(0, extent, size=(n, 3))
    nrm = rng.normal(size=(n, 3))
    q[:, 3:6] = nrm / np.linalg.norm(nrm, axis=1, keepdims=True)
    q[:, 6:9] = rng.uniform(0, 1, size=(n, 3))
    y = (q[:, 6:9] * (0.5 + 0.5 * np.sin(q[:, :1] * 0.7))).astype(np.float32)
    return q, y


def _init(rng):
    from oracle import mlp_ref as M
    ws = []
    for l, (k, n) in enumerate(M.SHAPES):
        w = rng.normal(size=(k, n)) * np.sqrt(2.0 / k)
        if l == 3:
            w[:, M.N_OUT:] = 0.0
            w *= 0.3
        ws.append(w)
    return M.pack(ws)


def test_encode_layout(orc):
    from oracle import mlp_ref as M
    rng = np.random.default_rng(1)
    q, _ = _data(rng, 64)
    f = M.encode(q, 16.0)
    assert f.shape == (64, 80)
    assert np.all(np.abs(f[:, :72]) <= 1.0)
    np.testing.assert_array_equal(f[:, 78], 1.0)
    np.testing.assert_array_equal(f[:, 79], 0.0)
    np.testing.assert_array_equal(f[:, 72:78], M.bf16_round(q[:, 3:9]))
    # octave k, axis 0: sin(2 pi 2^k frac(p / extent * 0.5)); the double-angle
    # recurrence stays within the bf16 step of the exact value
    for k in range(12):
        ref = np.sin(2 * np.pi * 2.0 ** k * ((q[:, 0] / 16.0 * 0.5) % 1.0))
        assert np.max(np.abs(f[:, 6 * k] - ref)) < 8e-3, k
        ref = np.cos(2 * np.pi * 2.0 ** k * ((q[:, 0] / 16.0 * 0.5) % 1.0))
        assert np.max(np.abs(f[:, 6 * k + 3] - ref)) < 8e-3, k


def test_bf16_round_ties_to_even():
    from oracle import mlp_ref as M
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: rounds to the even mantissa (1.0)
    x = np.array([1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -2.5, 0.0], np.float32)
    np.testing.assert_array_equal(M.bf16_round(x), np.array([1.0, 1.0 + 2 * 2.0 ** -7, -2.5, 0.0], np.float32))


def test_gradient64_matches_finite_differences(orc):
    from oracle import mlp_ref as M
    rng = np.random.default_rng(2)
    q, y = _data(rng, 48)
    feat = M.encode(q, 16.0).astype(np.float64)
    p = _init(rng)
    g = M.gradient64(feat, y, p)
    # the loss with the denominator frozen at p (the training objective's gradient)
    o0 = M.forward64(feat, p)[:, :M.N_OUT]
    den = o0 * o0 + 0.01

    def L(pp):
        o = M.forward64(feat, pp)[:, :M.N_OUT]
        return float(np.mean(np.sum((o - y) ** 2 / den, axis=1)))

    idx = rng.choice(np.flatnonzero(g != 0), size=60, replace=False)
    eps = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = eps
        fd = (L(p + e) - L(p - e)) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_bf16_network_close_to_exact(orc):
    from oracle import mlp_ref as M
    rng = np.random.default_rng(3)
    q, y = _data(rng, 256)
    feat = M.encode(q, 16.0)
    p = _init(rng)
    o, _, _ = M.forward(feat, p)
    o64 = M.forward64(feat, M.bf16_round(p))
    assert np.max(np.abs(o - o64)) < 0.05 * np.max(np.abs(o64))
    _, g = M.gradient(feat, y, p)
    g64 = M.gradient64(feat.astype(np.float64), y, M.bf16_round(p))
    assert np.linalg.norm(g - g64) < 0.05 * np.linalg.norm(g64)


def test_adam_step_moves_against_gradient():
    from oracle import mlp_ref as M
    w = np.ones(M.N_PARAMS, np.float32)
    g = np.full(M.N_PARAMS, 0.5, np.float32)
    w1, m1, v1 = M.adam(w, np.zeros_like(w), np.zeros_like(w), g, 1, 1e-2)
    pad = np.zeros(M.N_PARAMS, bool)
    pad[M.N_PARAMS - 1024:] = (np.arange(1024) % 16) >= 3
    # first step of Adam moves every weight by lr (bias-corrected m/sqrt(v) = sign(g))
    np.testing.assert_allclose(w1[~pad], 1.0 - 1e-2, rtol=1e-5)
    assert np.all(w1[pad] == 0.0)
