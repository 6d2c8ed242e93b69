"""The per-axis kinetic scheme of the merged RK step (GP5_KIN_SCHEME=1, Launch::step_axes: y and
z spectral second-derivative passes, the x term inside the stage boundary) against the default
3D-transform scheme: the same step to rounding (the sum of the three 1D terms is the 3D operator
because K^2 is separable)."""
import math
import os

import numpy as np
import pytest

from gp5_b200 import _abi

pytestmark = pytest.mark.gpu


def droplet(n, N=500.0, seed=3):
    L = 4.0 * N ** (1.0 / 3.0)
    x = -L / 2 + L / n * (np.arange(n) + 0.5)
    sig = 0.5 * N ** (1.0 / 3.0)
    g = np.exp(-x * x / (2 * sig * sig))
    psi = (g[:, None, None] * g[None, :, None] * g[None, None, :]).astype(np.complex128)
    psi *= np.exp(1j * 1e-3 * np.random.default_rng(seed).uniform(-1, 1, psi.shape))
    psi *= math.sqrt(N / (float(np.sum(np.abs(psi) ** 2)) * (L / n) ** 3))
    return np.asfortranarray(psi), L


def advance(scheme, n, prec, kind, imaginary, steps):
    psi, L = droplet(n)
    old = os.environ.get("GP5_KIN_SCHEME")
    os.environ["GP5_KIN_SCHEME"] = scheme  # read when the plan is created
    try:
        p = _abi.Plan((n,) * 3, (-L / 2,) * 3, (L / 2,) * 3, precision=prec)
    finally:
        if old is None:
            del os.environ["GP5_KIN_SCHEME"]
        else:
            os.environ["GP5_KIN_SCHEME"] = old
    f = _abi.Functional(p, _abi.GP5_FUNC_LHY, c3=-3.0, c4=2.5)
    st = _abi.Stepper(f, 0.15 * (L / n) ** 2 if imaginary else 2e-3, kind, imaginary=imaginary)
    if imaginary:
        st.set_renormalization([500.0])
    a = p.field(psi.astype(p.cdtype))
    st.advance(a, steps)
    out = a.download()
    prof = st.profile(a, nrep=1)
    a.close()
    st.close()
    f.close()
    p.close()
    return out, [k for k, _ in prof]


@pytest.mark.parametrize("n,prec,kind,imaginary", [
    (32, _abi.GP5_C128, _abi.GP5_STEP_RK4, True),
    (64, _abi.GP5_C128, _abi.GP5_STEP_RK4, False),
    (64, _abi.GP5_C128, _abi.GP5_STEP_EULER, False),
    (64, _abi.GP5_C64, _abi.GP5_STEP_RK4, False),
    (64, _abi.GP5_C64, _abi.GP5_STEP_RK4, True),
])
def test_per_axis_scheme_matches_the_3d_transform_scheme(n, prec, kind, imaginary):
    ref, kinds0 = advance("0", n, prec, kind, imaginary, 5)
    got, kinds1 = advance("1", n, prec, kind, imaginary, 5)
    tol = 1e-13 if prec == _abi.GP5_C128 else 2e-6
    assert float(np.max(np.abs(got - ref))) <= tol * float(np.max(np.abs(ref)))
    stages = 4 if kind == _abi.GP5_STEP_RK4 else 1
    # the per-axis step: y and z derivative passes and the boundary per stage, no prologue
    assert kinds1.count(12) == stages and kinds1.count(22) >= stages and kinds1.count(2) == stages
    assert 3 not in kinds1 and kinds0.count(3) == stages
