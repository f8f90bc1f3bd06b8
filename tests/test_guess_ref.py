"""The FP64 restatement of the learned-guess network (oracle/guess_mlp_ref.py), pinned on CPU
before it is trusted as the checker of the GPU's backward kernels: with the BF16 roundings
switched off its analytic gradient equals central finite differences of its own loss."""
import numpy as np

import guess_mlp_ref as MLP


def test_restatement_gradient_matches_central_differences():
    rng = np.random.default_rng(3)
    n = sum(fi * fo + fo for fi, fo in MLP.SIZES)
    p = rng.standard_normal(n) * 0.08
    rows = 40
    x = rng.standard_normal((rows, 64))
    t = rng.standard_normal((rows, 8)) * 0.3
    m = (rng.random((rows, 8)) < 0.7).astype(np.float64)
    inv = 1.0 / rows
    ident = lambda a: np.asarray(a, np.float64)  # noqa: E731
    loss, g = MLP.loss_and_grad(p, x, t, m, inv, rnd=ident)
    assert loss > 0.0
    # a few entries of every block: W1, b1, W2, b2, W3, b3, W4, b4
    starts, off = [], 0
    for fi, fo in MLP.SIZES:
        starts += [off, off + fi * fo]
        off += fi * fo + fo
    picks = [s + k for s in starts for k in (0, 3, 7)]
    h = 1e-5
    for k in picks:
        e = np.zeros(n)
        e[k] = h
        lp, _ = MLP.loss_and_grad(p + e, x, t, m, inv, rnd=ident)
        lm, _ = MLP.loss_and_grad(p - e, x, t, m, inv, rnd=ident)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[k]) <= 1e-7 + 1e-6 * abs(fd), (k, fd, g[k])


def test_bf16_rounding_is_round_to_nearest_even():
    vals = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 0.0], np.float32)
    r = MLP.bf16(vals)
    assert r[0] == 1.0 and r[1] == 1.0  # tie below: to even (1.0)
    assert r[2] == 1.0 + 2 ** -7  # 1 + 1.5 ulp -> 1 + 2 ulp
    assert r[3] == -2.5 and r[4] == 0.0
