"""CPU checks of the oracle against the reference's own known answers.

Each test restates one of the reference's tests (lucaparisi91/GP5) on the oracle:
  fft_test.cpp:10-83    forward/backward round trip, TOL 1e-6 (traits.h:46)
  fft_test.cpp:85-153   spectral Laplacian of a Gaussian against the analytic value, 1e-6
  test.py:92-119        LHY H applied to exp(-r^2) against the analytic value, 1e-4
  test.py:123-147       normalise to 1
  test.py:10-69         geometry: space steps, cell-centred grid
plus the long-double direct DFT (oracle/dft_ld.c) pinning numpy's FFT on small grids.
"""
import math

import numpy as np
import pytest

from oracle import gp_oracle as o
from oracle import dft3_ld


def test_geometry_space_step_and_grid():
    geo = o.Geometry((100, 200, 50))  # test.py:10-18 (default box [-1, 1])
    assert geo.left == (-1, -1, -1) and geo.right == (1, 1, 1)
    assert geo.space_step(0) == 2 / 100 and geo.space_step(1) == 2 / 200 and geo.space_step(2) == 2 / 50
    X, Y, Z = o.grid(geo)  # test.py:35-40
    assert abs(X.min() - (geo.left[0] + geo.space_step(0) / 2)) < 1e-12
    assert abs(X.max() - (geo.right[0] - geo.space_step(0) / 2)) < 1e-12
    assert abs((X[1, 0, 0] - X[0, 0, 0]) - geo.space_step(0)) < 1e-12


def test_momentum_conventions():
    # even n: Nyquist -> -n/2 ; odd n: i <= (n-1)/2 positive (geometry.cpp:127-148)
    geo = o.Geometry((8, 7, 2), (0, 0, 0), (2 * math.pi, 2 * math.pi, 2 * math.pi))
    assert list(o.momentum_axis(geo, 0)) == [0, 1, 2, 3, -4, -3, -2, -1]
    assert list(o.momentum_axis(geo, 1)) == [0, 1, 2, 3, -3, -2, -1]


@pytest.mark.parametrize("shape", [(6, 10, 12), (8, 8, 8), (5, 7, 3), (30, 4, 2)])
def test_numpy_fft_matches_long_double_dft(shape):
    rng = np.random.default_rng(1)
    a = (rng.standard_normal(shape + (1,)) + 1j * rng.standard_normal(shape + (1,)))
    for direction in (o.FORWARD, o.BACKWARD):
        ref = dft3_ld(a, direction)
        got = o.fft3(a, direction)
        assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-14


def test_fft_forward_backward_roundtrip():
    # fft_test.cpp:10-83: N=(50,170,150), box [-1/2,1/2]^3, Gaussian sigma=(1,0.5,0.2)
    geo = o.Geometry((50, 170, 150), (-0.5,) * 3, (0.5,) * 3)
    f = o.new_field(geo)
    o.init_gaussian(geo, (1, 0.5, 0.2), f)
    back = o.fft3(o.fft3(f, o.FORWARD), o.BACKWARD) * (1.0 / geo.n_sites)
    assert np.max(np.abs(back - f)) < 1e-6


def test_laplacian_of_gaussian_analytic():
    # fft_test.cpp:85-153: N=(300,250,77), sigma=0.05, max |L - analytic| <= 1e-6
    geo = o.Geometry((300, 250, 77), (-0.5,) * 3, (0.5,) * 3)
    f = o.new_field(geo)
    sigma = 0.05
    o.init_gaussian(geo, sigma, f)
    lap = o.laplacian(f, geo)[..., 0]
    X, Y, Z = o.grid(geo)
    R2 = X * X + Y * Y + Z * Z
    alpha = 1 / (2 * sigma * sigma)
    L2 = np.exp(-alpha * R2) * (-R2 * alpha * 2 + 3) * (-2) * alpha
    assert np.max(np.abs(L2 - lap)) <= 1e-6


def test_lhy_apply_gaussian_analytic():
    # test.py:92-119: 100^3, box [-4,4]^3, psi = exp(-r^2)
    geo = o.Geometry((100, 100, 100), (-4,) * 3, (4,) * 3)
    X, Y, Z = o.grid(geo)
    r2 = X * X + Y * Y + Z * Z
    psi = o.new_field(geo)
    psi[..., 0] = np.exp(-r2) + 0j
    out = o.Functional("lhy").apply(psi, geo)[..., 0]
    p = np.exp(-r2)
    expected = (3 - 2 * r2) * p + (-3 * p ** 2 + 5 / 2 * p ** 3) * p
    assert np.max(np.abs(expected - out.real)) < 1e-4


def test_renormalize():
    # test.py:123-147
    geo = o.Geometry((50, 50, 50), (-5,) * 3, (5,) * 3)
    X, Y, Z = o.grid(geo)
    psi = o.new_field(geo)
    psi[..., 0] = np.exp(-(X * X + Y * Y + Z * Z))
    o.normalize(1, psi, 0, geo)
    assert abs(o.norm(psi, 0, geo) - 1) < 1e-12


def test_rk4_euler_consistency_small_dt():
    # one RK4 step and 16 Euler steps of dt/16 agree to O(dt^2) for a smooth state
    geo = o.Geometry((12, 12, 12), (-4,) * 3, (4,) * 3)
    psi = o.gaussian_with_noise(geo, 1.0, 0.0, seed=0, N=1.0)
    f = o.Functional("gp", couplings=[[1.0]], V=o.harmonic_potential(geo, [(1, 1, 1)]))
    rk = o.Stepper(f, geo, 1e-3, "RK4", True).advance(psi.copy(), 1)
    eu = o.Stepper(f, geo, 1e-3 / 16, "eulero", True).advance(psi.copy(), 16)
    assert np.max(np.abs(rk - eu)) / np.max(np.abs(rk)) < 1e-4


def test_energy_definitions_consistent():
    # E(psi) derivative along psi equals 2 Re<psi|H psi> (e_int' = f) for LHY and GP
    geo = o.Geometry((16, 16, 16), (-6,) * 3, (6,) * 3)
    psi = o.gaussian_with_noise(geo, 1.5, 1e-3, seed=3, N=20.0, phase_noise=True)
    for f in (o.Functional("lhy"),
              o.Functional("gp", couplings=[[2.0]], V=o.harmonic_potential(geo, [(1, 0.5, 2)]))):
        eps = 1e-6
        Ep = o.observables(f, psi * (1 + eps), geo)["E"]
        Em = o.observables(f, psi * (1 - eps), geo)["E"]
        dE = (Ep - Em) / (2 * eps)
        ob = o.observables(f, psi, geo)
        assert abs(dE - 2 * ob["mu"] * ob["norm"]) / abs(dE) < 1e-6


@pytest.mark.slow
def test_lhy_mu_protocol_near_reference_golden():
    """python/test/regressionTests/LHY_imaginary.py with its committed golden (mu file).

    The committed script's protocol, restated exactly, converges to -0.38366638; the
    committed number is -0.38372999.  The norm-decay estimator carries an O(dt) bias of
    ~6.6e-4 (the converged state's <H>/N is -0.38432), and the golden sits 6.4e-5 away
    from the restatement: it is pinned here to 1e-4, not bitwise.
    """
    mu, blocks, _ = o.lhy_mu_protocol()
    assert abs(mu - (-0.3837299937094331)) < 1e-4
    assert abs(mu - (-0.3836663826072363)) < 1e-12


def test_rk4_imaginary_stability_bound_on_corner_modes():
    """Renormalised imaginary-time RK4 blows up once dt passes 2.785 / (1.5 (pi/dx)^2)
    ~ 0.188 dx^2: white noise excites the cube-corner modes K^2 = 3 (pi/dx)^2, whose RK4
    amplification leaves [-1, 1].  (The batched ground-state runs use 0.15 dx^2.)"""
    geo = o.Geometry((16, 16, 16), (-4,) * 3, (4,) * 3)
    psi = o.gaussian_with_noise(geo, 1.5, 1e-3, seed=4, N=20.0, phase_noise=True)
    dx = geo.space_step(0)
    f = o.Functional("lhy")
    grow = []
    for fac in (0.15, 0.2):
        st = o.Stepper(f, geo, fac * dx * dx, normalizations=[20.0])
        e0 = o.observables(f, psi, geo)["ekin"]
        e1 = o.observables(f, st.advance(psi.copy(), 300), geo)["ekin"]
        grow.append(e1 / e0)
    assert grow[0] < 1.0 and grow[1] > 3.0


def test_decompose_squares_reference_case():
    # tst/cluster_test.cpp:34-58 on the oracle's restatement of src/cluster.cpp:17-83
    import oracle
    data = np.zeros((100, 100, 100, 1), complex)
    data[10:51, 10:51, 10:51, 0] = 1
    lab, k = oracle.decompose(data, 0.5)
    assert k == 1 and (lab[10:51, 10:51, 10:51] == 1).all()
    assert (lab[0:10] == -1).all() and (lab[51:] == -1).all()
    data[:] = 0
    data[10:21, 10:21, 10:21] = 1
    data[50:61, 10:21, 10:21] = 1
    lab, k = oracle.decompose(data, 0.5)
    assert k == 2 and (lab[10:21, 10:21, 10:21] == 1).all() and (lab[50:61, 10:21, 10:21] == 2).all()


def test_decompose_periodic_diagonal_order_and_cutoff():
    import oracle
    d = np.zeros((12, 10, 8, 2), complex)
    d[0, 3, 3, 0] = d[11, 3, 3, 0] = 1           # joined through the x boundary
    d[5, 5, 5, 0] = d[6, 6, 6, 0] = 1            # joined through a corner (26-neighbours)
    d[2, 0, 0, 0] = 1                            # scanned before (5,...) with i slowest
    d[8, 9, 7, 0] = 0.5 + 0.5j                   # |psi|^2 = 0.5: not above the cutoff
    lab, k = oracle.decompose(d, 0.5)
    assert k == 3
    assert lab[0, 3, 3, 0] == lab[11, 3, 3, 0] == 1
    assert lab[2, 0, 0, 0] == 2 and lab[5, 5, 5, 0] == lab[6, 6, 6, 0] == 3
    assert lab[8, 9, 7, 0] == -1 and (lab[..., 1] == 0).all()


def test_threaded_elementwise_oracle_is_bitwise_serial():
    """set_elementwise_threads only spreads the element-wise expressions over z-slabs: the
    results must not change by a bit."""
    geo = o.Geometry((48, 40, 36), (-6,) * 3, (6,) * 3)
    psi = o.gaussian_with_noise(geo, 1.5, 1e-3, seed=5, N=40.0, phase_noise=True)
    psi2 = np.concatenate([psi, 0.5 * psi], axis=3)
    V = np.asfortranarray(np.random.default_rng(1).uniform(0, 1, psi.shape))
    phase = np.asfortranarray(np.random.default_rng(2).uniform(-3, 3, psi.shape))
    cases = [
        lambda: o.Stepper(o.Functional("lhy", c3=-3.3, V=V), geo, 1e-3, imaginary=False).advance(psi.copy(), 2),
        lambda: o.Stepper(o.Functional("gp", couplings=np.array([[1.0, 0.3], [0.3, 2.0]]), masses=[1.0, 2.0]),
                          geo, 1e-3, normalizations=[40.0, 10.0]).advance(psi2.copy(), 2),
        lambda: o.Stepper(o.Functional("lhy"), geo, 1e-3, "eulero", False,
                          constraint_phase=phase).advance(psi.copy(), 2),
    ]
    try:
        serial = [c() for c in cases]
        o.set_elementwise_threads(4)
        threaded = [c() for c in cases]
    finally:
        o.set_elementwise_threads(1)
    for a, b in zip(serial, threaded):
        assert np.array_equal(a, b)
