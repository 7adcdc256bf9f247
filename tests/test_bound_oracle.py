"""Pins the learned bound's CPU oracle (oracle/bound_oracle.py), which has no counterpart in
the reference: its analytic gradient equals central finite differences of its own loss (with
the bfloat16 roundings switched off, which make the loss piecewise constant), one Adam step
follows the published update rule, and the bfloat16 rounding is round-to-nearest-even.
CPU only."""
import math

import numpy as np

from oracle import bound_oracle as BO


def _setup(seed=0, n=64):
    rng = np.random.default_rng(seed)
    p = np.zeros(BO.N_PARAMS)
    for off, cnt, fan in ((BO.OFF_W1, 768, 12), (BO.OFF_B1, 64, 12), (BO.OFF_W2, 4096, 64), (BO.OFF_B2, 64, 64),
                          (BO.OFF_W3, 64, 64), (BO.OFF_B3, 1, 64)):
        p[off:off + cnt] = rng.uniform(-1, 1, cnt) / math.sqrt(fan)
    raw = rng.normal(0.0, 2.0, (n, 12)).astype(np.float32)
    tgt = (raw[:, 10] + rng.normal(-0.5, 0.3, n)).astype(np.float32)
    norm = (raw.mean(0), raw.std(0), float((tgt - raw[:, 10]).mean()), float((tgt - raw[:, 10]).std()))
    return p, raw, tgt, norm


def test_gradient_matches_finite_differences():
    p, raw, tgt, norm = _setup()
    _, g = BO.loss_and_grad(p, raw, tgt, norm, rounding=False)
    rng = np.random.default_rng(1)
    picks = list(rng.choice(BO.N_PARAMS, 60, replace=False)) + [BO.OFF_B3, BO.OFF_W3, BO.OFF_B1, BO.OFF_W1]
    for i in picks:
        h = 1e-5
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp, _ = BO.loss_and_grad(pp, raw, tgt, norm, rounding=False)
        lm, _ = BO.loss_and_grad(pm, raw, tgt, norm, rounding=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_adam_step_rule():
    p = np.array([0.5, -1.0, 2.0])
    g = np.array([0.1, -0.2, 0.0])
    m, v = np.zeros(3), np.zeros(3)
    p1, m1, v1 = BO.adam(p, m, v, g, 1, 1e-2)
    # first bias-corrected step moves each weight by lr * sign(g) (up to eps)
    assert np.allclose(p1, p - 1e-2 * np.sign(g), atol=1e-6)
    assert np.allclose(m1, 0.1 * g) and np.allclose(v1, 0.001 * g * g)


def test_bf16_round_to_nearest_even():
    one = np.float32(1.0)
    ulp = np.float32(2.0 ** -7)  # bfloat16 spacing at 1
    assert BO.bf16(one + ulp / 2)[()] == one                  # tie -> even (1.0)
    assert BO.bf16(one + ulp + ulp / 2)[()] == one + 2 * ulp  # tie -> even (1 + 2 ulp)
    assert BO.bf16(one + ulp * 0.49)[()] == one
    assert BO.bf16(one + ulp * 0.51)[()] == one + ulp
