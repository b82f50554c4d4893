"""CPU checks of the screening network's oracle: BF16 rounding, the float64
gradient against central finite differences, and the unit enumeration."""
import numpy as np

import macis_b200 as mb
from oracle import screen_oracle as so


def test_bf16_rounding_half_to_even():
    x = np.array([1.0, 1 + 2.0 ** -8, 1 + 3 * 2.0 ** -8, 1 + 2.0 ** -7,
                  -2.5, 3.0e38, 1e-40], dtype=np.float32)
    r = so.bf16_round(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                       # tie -> even mantissa
    assert r[2] == np.float32(1 + 2.0 ** -6)  # tie -> even (upwards)
    assert r[3] == np.float32(1 + 2.0 ** -7)  # representable
    assert r[4] == -2.5
    assert np.isfinite(r[5])
    assert np.array_equal(so.bf16_value(so.bf16_bits(x)), r)


def test_float64_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    din, n = 64, 7
    _, npar = so.layout(din)
    P = rng.normal(0, 0.2, npar)
    X = rng.normal(0, 1, (n, din))
    t = rng.normal(0, 1, n)
    g, loss = so.gradients(P, X, t, din, bf16=False)
    y, _ = so.forward(P, X, din, bf16=False)
    assert abs(loss - np.sum((y - t) ** 2) / (2 * n)) < 1e-14
    off, _ = so.layout(din)
    idx = np.concatenate([rng.integers(a, b, 6) for a, b in off.values()])
    h = 1e-6
    for i in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += h
        Pm[i] -= h
        lp = so.gradients(Pp, X, t, din, bf16=False)[1]
        lm = so.gradients(Pm, X, t, din, bf16=False)[1]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_adam_first_step_is_sign_times_lr():
    P = np.zeros(4)
    G = np.array([1.0, -2.0, 0.5, 0.0])
    P1, M, V = so.adam(P, G, np.zeros(4), np.zeros(4), 1, 1e-3)
    # bias-corrected first step: -lr * g / (|g| + eps)
    assert np.allclose(P1[:3], -1e-3 * np.sign(G[:3]), rtol=1e-6)
    assert P1[3] == 0.0


def test_unit_count_formula():
    for na, nb, nva, nvb in [(3, 2, 5, 6), (1, 1, 1, 1), (4, 4, 0, 0)]:
        u = so._unit_list(na, nb, nva, nvb)
        assert len(u) == 2 + 2 * na * nva + nb * nvb
        assert u[0][0] == 0 and u[1][0] == 1


def test_unit_widths():
    for nbits in (64, 128, 256):
        assert mb.unit_width(nbits) == so.unit_width(nbits)
