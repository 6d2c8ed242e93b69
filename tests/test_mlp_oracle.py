"""CPU checks of the warm-start MLP oracle and of the warm start's host-side pieces."""
import math

import numpy as np
import pytest

from oracle import mlp_oracle as mo

SMALL = [(7, 3), (5, 7), (4, 5)]


def test_analytic_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = mo.init_params(1, SMALL) + 0.1 * rng.standard_normal(mo.num_params(SMALL))
    x = rng.standard_normal((6, 3))
    t = rng.standard_normal((6, 4))
    _, g = mo.loss_and_grad(p, x, t, shapes=SMALL)
    h = 1e-6
    fd = np.empty_like(p)
    for i in range(p.size):
        e = np.zeros_like(p)
        e[i] = h
        fd[i] = (mo.loss_and_grad(p + e, x, t, shapes=SMALL)[0] - mo.loss_and_grad(p - e, x, t, shapes=SMALL)[0]) / (2 * h)
    assert np.max(np.abs(fd - g)) <= 1e-8 * max(1.0, np.max(np.abs(g)))


def test_full_size_directional_derivative():
    rng = np.random.default_rng(1)
    p = mo.init_params(2)
    x = rng.standard_normal((16, 3))
    t = rng.standard_normal((16, 64)) * 0.3
    _, g = mo.loss_and_grad(p, x, t)
    v = rng.standard_normal(p.size)
    h = 1e-6
    fd = (mo.loss_and_grad(p + h * v, x, t)[0] - mo.loss_and_grad(p - h * v, x, t)[0]) / (2 * h)
    assert abs(fd - g @ v) <= 1e-7 * abs(fd)


def test_bf16_rounding():
    a = np.array([1.0, 1.00390625, 1.005859375, -3.0e-5, 65504.0], dtype=np.float32)
    r = mo.bf16(a)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == 1.0078125
    assert np.all(np.abs(r - a) <= np.abs(a) * 2.0 ** -8)


def test_adam_first_step_is_signed_lr():
    p = np.zeros(4)
    g = np.array([1e-3, -2.0, 5.0, 0.0])
    p1, m, v = mo.adam_step(p, g, np.zeros(4), np.zeros(4), 1, 0.01)
    assert np.allclose(p1[:3], -0.01 * np.sign(g[:3]), rtol=1e-4) and p1[3] == 0.0


def test_radial_samples_of_gaussian():
    from gp5_b200 import warmstart as ws
    N, n = 300.0, 64
    L = ws.box_length(N)
    x = ws.axis(n, L)
    s = 0.3 * N ** (1 / 3)
    g = np.exp(-x * x / (2 * s * s))
    psi = g[:, None, None] * g[None, :, None] * g[None, None, :]
    got = ws.radial_samples(psi, N)
    r = ws.radii(N)
    assert np.max(np.abs(got - np.exp(-r * r / (2 * s * s)))) < 1e-9


def test_profile_start_reproduces_gaussian():
    from gp5_b200 import warmstart as ws
    N, n = 300.0, 64
    s = 0.3 * N ** (1 / 3)
    r = ws.radii(N)
    psi = ws.profile_start(np.exp(-r * r / (2 * s * s)), N, n)
    ref = ws.gaussian_start(N, n)  # width 0.5 N^(1/3): build the 0.3 one by hand
    L = ws.box_length(N)
    x = ws.axis(n, L)
    g = np.exp(-x * x / (2 * s * s))
    ref = (g[:, None, None] * g[None, :, None] * g[None, None, :])
    ref = ref * math.sqrt(N / (np.sum(ref ** 2) * (L / n) ** 3))
    assert np.max(np.abs(psi - ref)) < 2e-4 * np.max(ref)
    assert abs(np.sum(np.abs(psi) ** 2) * (L / n) ** 3 - N) < 1e-9 * N


def test_sample_params_ranges_and_features():
    from gp5_b200 import warmstart as ws
    ps = ws.sample_params(500, 7)
    Ns = np.array([p["N"] for p in ps])
    assert Ns.min() >= 20 and Ns.max() <= 2000
    assert all(-3.2 <= p["c3"] <= -2.8 for p in ps)
    assert {p["omega"] for p in ps} == {0.0, 0.05, 0.1}
    f = ws.features(ps)
    assert f.shape == (500, 3) and np.all(np.abs(f) < 2.0)
    assert ws.sample_params(3, 7) == ps[:3]
