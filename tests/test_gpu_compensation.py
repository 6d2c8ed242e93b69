"""complex64 state updates against complex128: the compensated update
(gp5cu_stepper_set_compensation) and the stochastically rounded one (the complex64 default,
gp5cu_stepper_set_stochastic_rounding), both against round-to-nearest."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def droplet(n=64, N=200.0):
    from gp5_b200 import warmstart as ws
    return ws.box_length(N), ws.gaussian_start(N, n, None)[..., None]


def run(prec, psi, L, steps, comp=False, renorm=None, dt=5e-5, rounding=None):
    from gp5_b200 import _abi
    n = psi.shape[0]
    p = _abi.Plan((n,) * 3, (-L / 2,) * 3, (L / 2,) * 3, precision=prec)
    f = _abi.Functional(p, _abi.GP5_FUNC_LHY, c3=-3.3)
    st = _abi.Stepper(f, dt, imaginary=renorm is not None)
    if renorm is not None:
        st.set_renormalization([renorm])
    if comp:
        st.set_compensation(True)
    if rounding is not None:
        st.set_stochastic_rounding(rounding == "stochastic")
    a = p.field(psi)
    st.advance(a, steps)
    return a.download(), f.observables(a)


def test_compensation_cuts_complex64_drift():
    L, psi = droplet()
    ref, o64 = run(0, psi, L, 600)
    plain, o32 = run(1, psi, L, 600, rounding="nearest")
    comp, o32c = run(1, psi, L, 600, comp=True)
    n0 = float(np.sum(np.abs(psi) ** 2) * (L / 64) ** 3)
    drift = abs(o32["norm"] / n0 - 1)
    drift_c = abs(o32c["norm"] / n0 - 1)
    assert abs(o64["norm"] / n0 - 1) < 1e-13
    assert drift_c < 0.25 * drift + 1e-9, (drift, drift_c)
    err = np.max(np.abs(plain - ref)) / np.max(np.abs(ref))
    err_c = np.max(np.abs(comp - ref)) / np.max(np.abs(ref))
    assert err_c <= err, (err, err_c)
    assert abs(o32c["energy"] / o64["energy"] - 1) <= abs(o32["energy"] / o64["energy"] - 1) + 1e-9


def test_compensation_rules():
    from gp5_b200 import _abi
    L, psi = droplet(32, 20.0)
    with pytest.raises(_abi.Gp5Error):
        run(0, psi, L, 1, comp=True)  # complex128 plans
    # with renormalisation the correction is inactive: bitwise the plain complex64 result
    a, _ = run(1, psi, L, 50, comp=True, renorm=20.0, dt=1e-3)
    b, _ = run(1, psi, L, 50, comp=False, renorm=20.0, dt=1e-3)
    assert np.array_equal(a, b)


def test_stochastic_rounding_is_the_default_and_cuts_complex64_drift():
    L, psi = droplet()
    ref, o64 = run(0, psi, L, 600)
    nearest, on = run(1, psi, L, 600, rounding="nearest")
    default, od = run(1, psi, L, 600)
    again, _ = run(1, psi, L, 600, rounding="stochastic")
    assert np.array_equal(default, again)  # the default, and deterministic
    n0 = float(np.sum(np.abs(psi) ** 2) * (L / 64) ** 3)
    drift_n = abs(on["norm"] / n0 - 1)
    drift_s = abs(od["norm"] / n0 - 1)
    assert drift_s < 0.5 * drift_n + 1e-9, (drift_n, drift_s)
    err_n = abs(on["energy"] / o64["energy"] - 1)
    err_s = abs(od["energy"] / o64["energy"] - 1)
    assert err_s < 0.5 * err_n + 1e-9, (err_n, err_s)
    # the state stays as close to complex128 as the round-to-nearest one
    assert np.max(np.abs(default - ref)) <= 2 * np.max(np.abs(nearest - ref)) + 1e-6 * np.max(np.abs(ref))


def test_stochastic_rounding_rules():
    from gp5_b200 import _abi
    L, psi = droplet(32, 20.0)
    with pytest.raises(_abi.Gp5Error):
        run(0, psi, L, 1, rounding="stochastic")  # complex128 plans
    run(0, psi, L, 1, rounding="nearest")  # turning it off is always allowed
    # the compensated update takes precedence: the same result with either rounding
    a, _ = run(1, psi, L, 20, comp=True, rounding="stochastic")
    b, _ = run(1, psi, L, 20, comp=True, rounding="nearest")
    assert np.array_equal(a, b)
