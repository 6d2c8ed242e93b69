"""The stage boundary fed by the bulk-copy ring (ring.cuh, k_boundary_ring) against the
register-load boundary of the same radix schedule: bitwise equal in real time (the ring changes
only where the operands come from), equal to the reduction order under renormalisation (its
tiles have other line counts, so the per-tile norm partials fold in another order); and the
bounded stage wait: a bound of 0 makes the wait run out, the call reports GP5_ERR_TIMEOUT and
the plan stays usable."""
import math

import numpy as np
import pytest

from gp5_b200 import _abi

pytestmark = pytest.mark.gpu

C128, C64 = _abi.GP5_C128, _abi.GP5_C64

# (n, precision, schedule) served by the ring's tile shapes (16 KB per stream and tile,
# 128 or 256 threads)
SERVED = [(32, C128, 0), (32, C128, 1), (64, C128, 0), (64, C128, 1), (128, C128, 1), (256, C128, 1),
          (32, C64, 0), (64, C64, 0), (128, C64, 0), (128, C64, 1), (256, C64, 0)]


def droplet(n, N=500.0, seed=7):
    L = 4.0 * N ** (1.0 / 3.0)
    x = -L / 2 + L / n * (np.arange(n) + 0.5)
    sig = 0.5 * N ** (1.0 / 3.0)
    g = np.exp(-x * x / (2 * sig * sig))
    psi = (g[:, None, None] * g[None, :, None] * g[None, None, :]).astype(np.complex128)
    psi *= np.exp(1j * 1e-3 * np.random.default_rng(seed).uniform(-1, 1, psi.shape))
    psi *= math.sqrt(N / (float(np.sum(np.abs(psi) ** 2)) * (L / n) ** 3))
    return np.asfortranarray(psi), L


def advance(n, prec, boundary, imaginary, steps, wait_ns=None):
    psi0, L = droplet(n)
    p = _abi.Plan((n,) * 3, (-L / 2,) * 3, (L / 2,) * 3, precision=prec)
    try:
        r = p.radix()
        p.set_radix(r[:5] + [boundary])
        assert p.radix()[5] == boundary
        if wait_ns is not None:
            p.set_wait_bound(wait_ns)
        f = _abi.Functional(p, _abi.GP5_FUNC_LHY, c3=-3.0, c4=2.5)
        dt = 0.15 * (L / n) ** 2 if imaginary else 2e-3
        st = _abi.Stepper(f, dt, _abi.GP5_STEP_RK4, imaginary=imaginary)
        if imaginary:
            st.set_renormalization([500.0])
        a = p.field(psi0.astype(p.cdtype))
        try:
            st.advance(a, steps)
            return a.download()
        finally:
            a.close()
            st.close()
            f.close()
    finally:
        p.close()


@pytest.mark.parametrize("n,prec,s", SERVED)
def test_ring_boundary_matches_register_loads_in_real_time(n, prec, s):
    steps = 2 if n == 256 else 5
    ref = advance(n, prec, s, False, steps)
    got = advance(n, prec, 2 | s, False, steps)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("n,prec,s", [c for c in SERVED if c[0] <= 128])
def test_ring_boundary_renormalised_imaginary_time(n, prec, s):
    ref = advance(n, prec, s, True, 6)
    got = advance(n, prec, 2 | s, True, 6)
    tol = 1e-13 if prec == C128 else 1e-5
    assert float(np.max(np.abs(got - ref))) <= tol * float(np.max(np.abs(ref)))


def test_ring_wait_timeout_reports_status_and_plan_stays_usable():
    n, prec, s = 64, C128, 0
    with pytest.raises(_abi.Gp5Error) as e:
        advance(n, prec, 2 | s, False, 2, wait_ns=0)
    assert e.value.status == _abi.GP5_ERR_TIMEOUT
    # the same configuration with the default bound runs and matches the register-load kernel
    got = advance(n, prec, 2 | s, False, 2, wait_ns=_abi.GP5_RING_WAIT_DEFAULT_NS)
    assert np.array_equal(got, advance(n, prec, s, False, 2))


def test_ring_choice_outside_its_shapes_falls_back():
    """Where the ring has no tile shape (c128 at 256 with schedule 0: 64 threads), the boundary
    runs the register-load kernel and the result is unchanged."""
    ref = advance(256, C128, 0, False, 1)
    got = advance(256, C128, 2, False, 1)
    assert np.array_equal(got, ref)
