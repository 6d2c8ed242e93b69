"""The bench workload at its full size (256^3 LHY droplet, N = 5000, L = 4 N^(1/3)): one RK4
step against the oracle, and size-independent properties of the transforms and of real-time
evolution."""
import math

import numpy as np
import pytest

from oracle import gp_oracle as o

pytestmark = pytest.mark.gpu

N_ATOMS, N_GRID = 5000.0, 256


def workload():
    L = 4.0 * N_ATOMS ** (1.0 / 3.0)
    geo = o.Geometry((N_GRID,) * 3, (-L / 2,) * 3, (L / 2,) * 3)
    psi = o.gaussian_with_noise(geo, 0.5 * N_ATOMS ** (1.0 / 3.0), 1e-3, seed=2024, N=N_ATOMS, phase_noise=True)
    return geo, psi


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.fixture(scope="module")
def setup():
    from gp5_b200 import _abi
    geo, psi = workload()
    return _abi, geo, psi


def test_one_rk4_step_matches_oracle_at_256cubed(setup):
    abi, geo, psi = setup
    p = abi.Plan(geo.shape, geo.left, geo.right)
    f = abi.Functional(p, abi.GP5_FUNC_LHY, c3=-3.3, c4=2.5)
    st = abi.Stepper(f, 5e-5, imaginary=False)
    a = p.field(psi)
    st.advance(a, 1)
    ref = o.Stepper(o.Functional("lhy", c3=-3.3, c4=2.5), geo, 5e-5, imaginary=False).advance(psi.copy(), 1)
    assert rel(a.download(), ref) < 1e-12


def test_fft_roundtrip_and_linearity_at_256cubed(setup):
    abi, geo, psi = setup
    p = abi.Plan(geo.shape, geo.left, geo.right)
    rng = np.random.default_rng(5)
    y = np.asfortranarray(rng.standard_normal(psi.shape) + 1j * rng.standard_normal(psi.shape))
    a, b, w = p.field(psi), p.field(y), p.field()
    p.fft(a, w, abi.GP5_FORWARD)
    fa = w.download()
    p.fft(w, w, abi.GP5_BACKWARD)
    assert rel(w.download() / N_GRID ** 3, psi) < 1e-13
    p.fft(b, w, abi.GP5_FORWARD)
    fb = w.download()
    c = p.field(np.asfortranarray(2.5 * psi - 1j * y))
    p.fft(c, w, abi.GP5_FORWARD)
    assert rel(w.download(), 2.5 * fa - 1j * fb) < 1e-13
    # Parseval: sum |F psi|^2 = N^3 sum |psi|^2
    assert abs(np.sum(np.abs(fa) ** 2) / (N_GRID ** 3 * np.sum(np.abs(psi) ** 2)) - 1) < 1e-13


@pytest.mark.parametrize("prec,tol_n,tol_e", [(0, 1e-12, 1e-9), (1, 1e-5, 1e-5)])
def test_real_time_conserves_norm_and_energy_at_256cubed(setup, prec, tol_n, tol_e):
    abi, geo, psi = setup
    p = abi.Plan(geo.shape, geo.left, geo.right, precision=prec)
    f = abi.Functional(p, abi.GP5_FUNC_LHY, c3=-3.3, c4=2.5)
    st = abi.Stepper(f, 5e-5, imaginary=False)
    a = p.field(psi)
    ob0 = f.observables(a)
    st.advance(a, 200)
    ob1 = f.observables(a)
    assert abs(ob1["norm"] / ob0["norm"] - 1) < tol_n
    assert abs(ob1["energy"] / ob0["energy"] - 1) < tol_e


def test_config2_droplet_ground_state_then_real_time():
    """The 128^3 LHY droplet (N = 500, L = 4 N^(1/3)): imaginary-time RK4 (dt = 5e-4,
    renormalised) to a residual of 1e-10, then 2000 real-time RK4 steps (dt = 1e-4).  A
    converged eigenstate only turns its phase in real time: |psi| stays put, the norm and the
    energy are conserved and the phase turns at the rate mu."""
    from gp5_b200 import _abi, warmstart as ws
    N, n = 500.0, 128
    L = ws.box_length(N)
    p = _abi.Plan((n,) * 3, (-L / 2,) * 3, (L / 2,) * 3)
    f = _abi.Functional(p, _abi.GP5_FUNC_LHY)
    st = _abi.Stepper(f, 5e-4)
    st.set_renormalization([N])
    a = p.field(ws.gaussian_start(N, n, seed=2024)[..., None])
    steps = 0
    ob = f.observables(a)
    while ob["residual"] > 1e-10 and steps < 400000:
        st.advance(a, 5000)
        steps += 5000
        ob = f.observables(a)
    assert ob["residual"] <= 1e-10, (steps, ob["residual"])
    gs = a.download()
    rt = _abi.Stepper(f, 1e-4, imaginary=False)
    rt.advance(a, 2000)
    ob2 = f.observables(a)
    psi = a.download()
    assert abs(ob2["norm"] / ob["norm"] - 1) < 1e-12
    assert abs(ob2["energy"] / ob["energy"] - 1) < 1e-10
    assert np.max(np.abs(np.abs(psi) - np.abs(gs))) <= 1e-7 * np.max(np.abs(gs))
    # phase turned by -mu t at the droplet centre (psi ~ e^{-i mu t} psi0)
    c = (n // 2, n // 2, n // 2, 0)
    turn = np.angle(psi[c] / gs[c])
    expected = -ob["mu"] * 2000 * 1e-4
    assert abs((turn - expected + np.pi) % (2 * np.pi) - np.pi) < 1e-6
