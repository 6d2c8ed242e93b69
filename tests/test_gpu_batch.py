"""Batched independent droplet solves (gp5cu_batch_*) against single solves and the oracle."""
import math

import numpy as np
import pytest

from oracle import gp_oracle as o

pytestmark = pytest.mark.gpu


def droplet_start(n, L, N, seed):
    geo = o.Geometry((n,) * 3, (-L / 2,) * 3, (L / 2,) * 3)
    return geo, o.gaussian_with_noise(geo, 0.5 * N ** (1 / 3), 1e-3, seed=seed, N=N, phase_noise=True)


SOLVES = [
    dict(n=32, L=12.0, N=20.0, c3=-3.0, c4=2.5, omega=0.0, dt=0.004),
    dict(n=64, L=20.0, N=200.0, c3=-2.9, c4=2.5, omega=0.1, dt=0.003),
    dict(n=32, L=14.0, N=40.0, c3=-3.1, c4=2.5, omega=0.05, dt=0.005),
    dict(n=64, L=24.0, N=500.0, c3=-3.2, c4=2.5, omega=0.0, dt=0.004),
    dict(n=32, L=10.0, N=25.0, c3=-2.8, c4=2.5, omega=0.0, dt=0.003),
]


@pytest.mark.parametrize("prec", [0, 1])
def test_batch_matches_single_solves(prec):
    from gp5_b200 import _abi as abi
    b = abi.Batch(SOLVES, precision=prec)
    starts = []
    for k, sd in enumerate(SOLVES):
        geo, psi = droplet_start(sd["n"], sd["L"], sd["N"], 100 + k)
        starts.append((geo, psi))
        b.set_state(k, psi)
    res = b.solve(tol=1e-30, check_every=10, max_steps=30)
    assert all(r["steps"] == 30 and not r["converged"] for r in res)
    for k, sd in enumerate(SOLVES):
        geo, psi = starts[k]
        p = abi.Plan(geo.shape, geo.left, geo.right, precision=prec)
        f = abi.Functional(p, abi.GP5_FUNC_LHY, c3=sd["c3"], c4=sd["c4"],
                           omegas=[(sd["omega"],) * 3] if sd["omega"] > 0 else None)
        st = abi.Stepper(f, sd["dt"])
        st.set_renormalization([sd["N"]])
        a = p.field(psi)
        for _ in range(3):
            st.advance(a, 10)
        single = a.download()
        batched = b.get_state(k)
        assert np.array_equal(single, batched), k
        if prec == 1:
            # a complex64 batch reports the observables of its state evaluated in complex128
            assert res[k]["steps_c64"] == 30
            p = abi.Plan(geo.shape, geo.left, geo.right)
            f = abi.Functional(p, abi.GP5_FUNC_LHY, c3=sd["c3"], c4=sd["c4"],
                               omegas=[(sd["omega"],) * 3] if sd["omega"] > 0 else None)
            a = p.field(single)
        ob = f.observables(a)
        assert abs(ob["residual"] - res[k]["residual"]) <= 1e-12 * max(ob["residual"], 1e-300) + 1e-300
        assert abs(ob["energy"] - res[k]["energy"]) <= 1e-12 * abs(ob["energy"])


def test_batch_vs_oracle():
    from gp5_b200 import _abi as abi
    sd = SOLVES[2]
    geo, psi = droplet_start(sd["n"], sd["L"], sd["N"], 7)
    b = abi.Batch([sd])
    b.set_state(0, psi)
    b.solve(tol=1e-30, check_every=5, max_steps=20)
    V = o.harmonic_potential(geo, [(sd["omega"],) * 3])
    st = o.Stepper(o.Functional("lhy", c3=sd["c3"], c4=sd["c4"], V=V), geo, sd["dt"], normalizations=[sd["N"]])
    ref = st.advance(psi.copy(), 20)
    got = b.get_state(0)
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-12


CONVERGE = [dict(n=32, L=4 * 20 ** (1 / 3), N=20.0, c3=-3.0, c4=2.5, omega=0.0, dt=0.01),
            dict(n=32, L=4 * 30 ** (1 / 3), N=30.0, c3=-3.1, c4=2.5, omega=0.0, dt=0.01),
            dict(n=64, L=4 * 70 ** (1 / 3), N=70.0, c3=-2.9, c4=2.5, omega=0.0, dt=0.15 * (4 * 70 ** (1 / 3) / 64) ** 2)]


def _converged_batch(prec):
    from gp5_b200 import _abi as abi
    b = abi.Batch(CONVERGE, precision=prec)
    starts = []
    for k, sd in enumerate(CONVERGE):
        geo, psi = droplet_start(sd["n"], sd["L"], sd["N"], 11 + k)
        starts.append(psi)
        b.set_state(k, psi)
    res = b.solve(tol=1e-8, check_every=100, max_steps=200000)
    return b, res, starts


def test_batch_converges_to_residual_and_packed_solves_match_single_solves():
    """Solves finish at different checks; the ones still running are packed into the first
    slots and the launches shrink to them.  Every final state is bitwise the single solve's
    after the same number of steps, and the observables agree with the oracle."""
    from gp5_b200 import _abi as abi
    b, res, starts = _converged_batch(abi.GP5_C128)
    assert len({r["steps"] for r in res[:2]}) == 2  # the 32^3 pair finishes at different checks
    for k, (r, sd) in enumerate(zip(res, CONVERGE)):
        assert r["converged"], r
        assert r["residual"] <= 1e-8
        assert r["steps_c64"] == 0
        geo = o.Geometry((sd["n"],) * 3, (-sd["L"] / 2,) * 3, (sd["L"] / 2,) * 3)
        got = b.get_state(k)
        ob = o.observables(o.Functional("lhy", c3=sd["c3"]), got, geo)
        assert abs(ob["E"] - r["energy"]) <= 1e-10 * abs(ob["E"])
        assert abs(ob["mu"] - r["mu"]) <= 1e-10 * abs(ob["mu"])
        assert abs(ob["norm"] - sd["N"]) <= 1e-9 * sd["N"]
        assert math.isclose(ob["residual"], r["residual"], rel_tol=1e-6)
        p = abi.Plan(geo.shape, geo.left, geo.right)
        st = abi.Stepper(abi.Functional(p, abi.GP5_FUNC_LHY, c3=sd["c3"], c4=sd["c4"]), sd["dt"])
        st.set_renormalization([sd["N"]])
        a = p.field(starts[k])
        for _ in range(r["steps"] // 100):
            st.advance(a, 100)
        assert np.array_equal(a.download(), got), k


def test_complex64_batch_converges_to_residual_like_complex128():
    """complex64 bulk, then complex128 to the tolerance: every solve reaches 1e-8 and its energy
    agrees with the complex128 batch's."""
    from gp5_b200 import _abi as abi
    _, r64, _ = _converged_batch(abi.GP5_C128)
    _, r32, _ = _converged_batch(abi.GP5_C64)
    for a, c in zip(r32, r64):
        assert a["converged"] and a["residual"] <= 1e-8, a
        assert 0 < a["steps_c64"] <= a["steps"]
        assert abs(a["energy"] - c["energy"]) <= 1e-9 * abs(c["energy"])
        assert abs(a["mu"] - c["mu"]) <= 1e-8 * abs(c["mu"])


@pytest.mark.parametrize("prec", [0, 1])
def test_preconditioned_batch_reaches_the_imaginary_time_ground_states(prec):
    """GP5_BATCH_PRECOND reaches the states that imaginary-time RK4 converges to (energy, mu
    and |psi|) in tens of iterations, where RK4 takes thousands of steps; a complex64 batch runs
    its bulk in complex64 and finishes in complex128.  The converged observables agree with the
    oracle's evaluation of the returned state."""
    from gp5_b200 import _abi as abi
    brk, rrk, starts = _converged_batch(abi.GP5_C128)
    b = abi.Batch(CONVERGE, precision=prec)
    b.set_method(abi.GP5_BATCH_PRECOND, 0.5)
    for k, psi in enumerate(starts):
        b.set_state(k, psi)
    res = b.solve(tol=1e-8, check_every=5, max_steps=2000)
    for k, (r, c, sd) in enumerate(zip(res, rrk, CONVERGE)):
        assert r["converged"] and r["residual"] <= 1e-8, r
        assert r["steps"] <= 200 and r["steps"] * 10 < c["steps"], (r["steps"], c["steps"])
        assert (r["steps_c64"] > 0) == (prec == 1)
        assert abs(r["energy"] - c["energy"]) <= 1e-9 * abs(c["energy"])
        # mu moves to first order with the state (the energy to second order): at residual
        # 1e-8 both solvers' states differ by about residual / gap
        assert abs(r["mu"] - c["mu"]) <= 1e-6 * abs(c["mu"])
        got = b.get_state(k)
        a = np.abs(brk.get_state(k))
        assert np.max(np.abs(np.abs(got) - a)) <= 1e-5 * np.max(a)
        geo = o.Geometry((sd["n"],) * 3, (-sd["L"] / 2,) * 3, (sd["L"] / 2,) * 3)
        ob = o.observables(o.Functional("lhy", c3=sd["c3"]), got, geo)
        assert abs(ob["E"] - r["energy"]) <= 1e-10 * abs(ob["E"])
        assert abs(ob["norm"] - sd["N"]) <= 1e-9 * sd["N"]
    with pytest.raises(abi.Gp5Error):
        b.set_method(abi.GP5_BATCH_PRECOND, 1.5)
    with pytest.raises(abi.Gp5Error):
        b.set_method(7, 0.5)
