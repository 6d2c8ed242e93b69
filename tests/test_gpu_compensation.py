"""Compensated complex64 state update (gp5cu_stepper_set_compensation) against complex128."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def droplet(n=64, N=200.0):
    from gp5_b200 import warmstart as ws
    return ws.box_length(N), ws.gaussian_start(N, n, None)[..., None]


def run(prec, psi, L, steps, comp=False, renorm=None, dt=5e-5):
    from gp5_b200 import _abi
    n = psi.shape[0]
    p = _abi.Plan((n,) * 3, (-L / 2,) * 3, (L / 2,) * 3, precision=prec)
    f = _abi.Functional(p, _abi.GP5_FUNC_LHY, c3=-3.3)
    st = _abi.Stepper(f, dt, imaginary=renorm is not None)
    if renorm is not None:
        st.set_renormalization([renorm])
    if comp:
        st.set_compensation(True)
    a = p.field(psi)
    st.advance(a, steps)
    return a.download(), f.observables(a)


def test_compensation_cuts_complex64_drift():
    L, psi = droplet()
    ref, o64 = run(0, psi, L, 600)
    plain, o32 = run(1, psi, L, 600)
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
