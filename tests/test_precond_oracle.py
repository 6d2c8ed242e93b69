"""The preconditioned ground-state iteration (the batched solver's GP5_BATCH_PRECOND) restated
in the oracle: it reaches a fixed point of renormalised imaginary-time RK4 (the reference's
ground-state method, stepper.cpp:46-71) at residual 1e-8 in tens of iterations."""
import numpy as np
import pytest

from oracle import gp_oracle as o


@pytest.mark.parametrize("N,c3,n,seed", [(20.0, -3.0, 32, 1), (30.0, -3.1, 32, 2), (300.0, -2.9, 32, 3)])
def test_preconditioned_iteration_reaches_an_imaginary_time_fixed_point(N, c3, n, seed):
    L = 4.0 * N ** (1.0 / 3.0)
    geo = o.Geometry((n,) * 3, (-L / 2,) * 3, (L / 2,) * 3)
    psi0 = o.gaussian_with_noise(geo, 0.5 * N ** (1.0 / 3.0), 1e-3, seed=seed, N=N, phase_noise=True)
    func = o.Functional("lhy", c3=c3)
    psi, it, ob = o.precond_ground_state(func, geo, psi0, N)
    assert ob["residual"] <= 1e-8 and it <= 200, (it, ob["residual"])
    assert abs(ob["norm"] - N) <= 1e-10 * N
    assert ob["E"] < o.observables(func, psi0, geo)["E"]
    # renormalised imaginary-time RK4 leaves the state where it is
    dx = L / n
    st = o.Stepper(func, geo, 0.15 * dx * dx, normalizations=[N])
    psi2 = st.advance(psi.copy(), 100)
    ob2 = o.observables(func, psi2, geo)
    assert abs(ob2["E"] - ob["E"]) <= 1e-10 * abs(ob["E"])
    assert np.max(np.abs(np.abs(psi2) - np.abs(psi))) <= 1e-6 * np.max(np.abs(psi))


@pytest.mark.parametrize("N,c3,omega,n", [(20.0, -3.0, 0.1, 32), (200.0, -2.9, 0.1, 32)])
def test_preconditioned_iteration_converges_in_a_trap(N, c3, omega, n):
    """With a harmonic trap the shift takes half the potential's maximum: without it the slowly
    varying modes at the box corners overshoot and the iteration diverges for large boxes."""
    L = 4.0 * N ** (1.0 / 3.0)
    geo = o.Geometry((n,) * 3, (-L / 2,) * 3, (L / 2,) * 3)
    psi0 = o.gaussian_with_noise(geo, 0.5 * N ** (1.0 / 3.0), 1e-3, seed=5, N=N, phase_noise=True)
    func = o.Functional("lhy", c3=c3, V=o.harmonic_potential(geo, [(omega,) * 3]))
    psi, it, ob = o.precond_ground_state(func, geo, psi0, N, max_iter=400)
    assert ob["residual"] <= 1e-8, (it, ob["residual"])
    dx = L / n
    st = o.Stepper(func, geo, 0.15 * dx * dx, normalizations=[N])
    ob2 = o.observables(func, st.advance(psi.copy(), 50), geo)
    assert abs(ob2["E"] - ob["E"]) <= 1e-10 * abs(ob["E"])
