"""GPU parity tests: the CUDA path, called through the C ABI, against the CPU oracle.

Tolerances (relative to max |oracle|): complex128 transforms 1e-13, one RK4 step 1e-12
(the one-step target), 1000 imaginary-time steps: psi 1e-10, E and mu 1e-10; complex64
transforms 2e-6.  The reference's own analytic tests keep their tolerances (1e-6, 1e-4).
"""
import math
import os

import numpy as np
import pytest

from oracle import gp_oracle as o

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def abi():
    from gp5_b200 import _abi
    _abi.lib()
    return _abi


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(np.asarray(b))), 1e-300))


def rand_field(shape, seed, ncomp=1):
    rng = np.random.default_rng(seed)
    s = tuple(shape) + (ncomp,)
    return np.asfortranarray(rng.uniform(-1, 1, s) + 1j * rng.uniform(-1, 1, s))


def make(abi, shape, left=(-1, -1, -1), right=(1, 1, 1), ncomp=1, prec=0):
    return abi.Plan(shape, left, right, ncomp=ncomp, precision=prec)


# ---------------------------------------------------------------- initial state
@pytest.mark.parametrize("prec,tol", [(0, 1e-15), (1, 1e-7)])
def test_init_gaussian_vs_oracle(abi, prec, tol):
    """gp5cu_init_gaussian against the oracle's initGaussian (geometry.cpp:251-276) on an
    anisotropic box and widths; the other component keeps its values."""
    geo = o.Geometry((30, 20, 17), (-10.0, -6.0, -3.5), (10.0, 8.0, 4.0))
    sigma = (5.0, 2.5, 1.25)
    p = make(abi, geo.shape, geo.left, geo.right, ncomp=2, prec=prec)
    start = rand_field(geo.shape, 11, ncomp=2)
    f = p.field(start)
    p.init_gaussian(f, sigma, comp=0)
    got = f.download()
    ref = start.copy()
    o.init_gaussian(geo, sigma, ref, comp=0)
    assert rel(got[..., 0], ref[..., 0]) < tol
    assert np.all(got[..., 0].imag == 0)
    if prec == 0:
        assert np.array_equal(got[..., 1], ref[..., 1])
    else:
        assert rel(got[..., 1], ref[..., 1]) < 1e-7
    with pytest.raises(abi.Gp5Error):
        p.init_gaussian(f, (1.0, 0.0, 1.0))


# ---------------------------------------------------------------- transforms
@pytest.mark.parametrize("prec,tol", [(0, 1e-13), (1, 2e-6)])
def test_fft_golden_mixed_radix(abi, prec, tol):
    z = np.load(os.path.join(GOLD, "fft_6x10x12.npz"))
    p = make(abi, (6, 10, 12), prec=prec)
    src, dst = p.field(z["a"]), p.field()
    p.fft(src, dst, abi.GP5_FORWARD)
    assert rel(dst.download(), z["fwd"]) < tol
    p.fft(src, dst, abi.GP5_BACKWARD)
    assert rel(dst.download(), z["bwd"]) < tol


@pytest.mark.parametrize("prec,tol", [(0, 1e-13), (1, 2e-6)])
def test_fft_golden_register_engine(abi, prec, tol):
    z = np.load(os.path.join(GOLD, "fft_32x64x8.npz"))
    p = make(abi, (32, 64, 8), prec=prec)
    src, dst = p.field(z["a"]), p.field()
    p.fft(src, dst, abi.GP5_FORWARD)
    assert rel(dst.download(), z["fwd"]) < tol


SHAPES = [(32, 32, 32), (64, 64, 64), (128, 64, 32), (256, 32, 16), (512, 16, 4), (30, 30, 30),
          (16, 24, 30), (77, 11, 13), (34, 17, 5), (64, 100, 48), (3, 256, 5)]


@pytest.mark.parametrize("shape", SHAPES)
def test_fft_vs_oracle(abi, shape):
    a = rand_field(shape, 7)
    p = make(abi, shape)
    src, dst = p.field(a), p.field()
    for d in (abi.GP5_FORWARD, abi.GP5_BACKWARD):
        p.fft(src, dst, d)
        assert rel(dst.download(), o.fft3(a, d)) < 1e-13, d


@pytest.mark.parametrize("shape", [(64, 64, 64), (30, 30, 30), (256, 16, 32)])
def test_fft_in_place_and_fp32(abi, shape):
    a = rand_field(shape, 8)
    p = make(abi, shape)
    f = p.field(a)
    p.fft(f, f, abi.GP5_FORWARD)
    assert rel(f.download(), o.fft3(a, o.FORWARD)) < 1e-13
    p32 = make(abi, shape, prec=1)
    g, h = p32.field(a), p32.field()
    p32.fft(g, h, abi.GP5_FORWARD)
    assert rel(h.download(), o.fft3(a, o.FORWARD)) < 2e-6


def test_fft_roundtrip_reference_case(abi):
    # fft_test.cpp:10-83
    geo = o.Geometry((50, 170, 150), (-0.5,) * 3, (0.5,) * 3)
    f = o.new_field(geo)
    o.init_gaussian(geo, (1, 0.5, 0.2), f)
    p = make(abi, geo.shape, geo.left, geo.right)
    a, b = p.field(f), p.field()
    p.fft(a, b, abi.GP5_FORWARD)
    p.fft(b, a, abi.GP5_BACKWARD)
    back = a.download() / geo.n_sites
    assert np.max(np.abs(back - f)) < 1e-6
    assert rel(back, f) < 1e-13


def test_laplacian_reference_analytic(abi):
    # fft_test.cpp:85-153: N=(300,250,77) (odd axis 7*11), sigma 0.05, <= 1e-6
    geo = o.Geometry((300, 250, 77), (-0.5,) * 3, (0.5,) * 3)
    f = o.new_field(geo)
    sigma = 0.05
    o.init_gaussian(geo, sigma, f)
    p = make(abi, geo.shape, geo.left, geo.right)
    a, b = p.field(f), p.field()
    p.laplacian(a, b)
    lap = b.download()[..., 0]
    X, Y, Z = o.grid(geo)
    R2 = X * X + Y * Y + Z * Z
    al = 1 / (2 * sigma * sigma)
    L2 = np.exp(-al * R2) * (-R2 * al * 2 + 3) * (-2) * al
    assert np.max(np.abs(L2 - lap)) <= 1e-6
    assert rel(lap, o.laplacian(f, geo)[..., 0]) < 1e-12


# ---------------------------------------------------------------- functionals
def test_lhy_apply_reference_analytic(abi):
    # test.py:92-119
    geo = o.Geometry((100, 100, 100), (-4,) * 3, (4,) * 3)
    X, Y, Z = o.grid(geo)
    r2 = X * X + Y * Y + Z * Z
    psi = o.new_field(geo)
    psi[..., 0] = np.exp(-r2) + 0j
    p = make(abi, geo.shape, geo.left, geo.right)
    f = abi.Functional(p, abi.GP5_FUNC_LHY)
    a, b = p.field(psi), p.field()
    f.apply(a, b)
    out = b.download()
    pe = np.exp(-r2)
    expected = (3 - 2 * r2) * pe + (-3 * pe ** 2 + 5 / 2 * pe ** 3) * pe
    assert np.max(np.abs(expected - out[..., 0].real)) < 1e-4
    assert rel(out, o.Functional("lhy").apply(psi, geo)) < 1e-12


def test_lhy_H_golden(abi):
    z = np.load(os.path.join(GOLD, "lhy_H_16x12x10.npz"))
    p = make(abi, (16, 12, 10), tuple(z["left"]), tuple(z["right"]))
    f = abi.Functional(p, abi.GP5_FUNC_LHY)
    a, b = p.field(z["psi"]), p.field()
    f.apply(a, b)
    assert rel(b.download(), z["H"]) < 1e-12


@pytest.mark.parametrize("shape", [(64, 64, 64), (48, 40, 36)])
def test_gp_harmonic_H_vs_oracle(abi, shape):
    geo = o.Geometry(shape, (-10,) * 3, (10,) * 3)
    psi = o.gaussian_with_noise(geo, 1.0, 1e-3, seed=1, N=1.0)
    p = make(abi, shape, geo.left, geo.right)
    f = abi.Functional(p, abi.GP5_FUNC_GP, couplings=[[1.0]], omegas=[(1.0, 1.0, 1.0)])
    a, b = p.field(psi), p.field()
    f.apply(a, b)
    of = o.Functional("gp", couplings=[[1.0]], V=o.harmonic_potential(geo, [(1, 1, 1)]))
    assert rel(b.download(), of.apply(psi, geo)) < 1e-12


def test_two_component_functionals(abi):
    geo = o.Geometry((24, 20, 16), (-6,) * 3, (6,) * 3)
    rng = np.random.default_rng(5)
    psi = o.new_field(geo, 2)
    o.init_gaussian(geo, 1.5, psi, 0)
    o.init_gaussian(geo, 2.0, psi, 1)
    psi = psi * np.exp(1j * 1e-2 * rng.uniform(-1, 1, psi.shape))
    p = make(abi, geo.shape, geo.left, geo.right, ncomp=2)
    a, b = p.field(psi), p.field()
    G = np.array([[1.0, 0.3], [0.3, 0.7]])
    f = abi.Functional(p, abi.GP5_FUNC_GP, couplings=G, masses=(1.0, 2.0), omegas=[(1, 1, 1), (0.5, 0.7, 0.9)])
    f.apply(a, b)
    of = o.Functional("gp", couplings=G, masses=(1.0, 2.0),
                      V=o.harmonic_potential(geo, [(1, 1, 1), (0.5, 0.7, 0.9)], 2))
    assert rel(b.download(), of.apply(psi, geo)) < 1e-12
    fu = abi.Functional(p, abi.GP5_FUNC_LHY_UNLOCKED, alpha=0.8, beta=0.6, eta=-1.1)
    fu.apply(a, b)
    ou = o.Functional("lhy_unlocked", alpha=0.8, beta=0.6, eta=-1.1)
    assert rel(b.download(), ou.apply(psi, geo)) < 1e-12


def test_potential_array(abi):
    geo = o.Geometry((32, 20, 24), (-5,) * 3, (5,) * 3)
    psi = o.gaussian_with_noise(geo, 1.2, 1e-2, seed=2, N=3.0)
    X, Y, Z = o.grid(geo)
    V = np.asfortranarray((0.3 * X * X + np.sin(Y) + 0.1 * Z)[..., None])
    p = make(abi, geo.shape, geo.left, geo.right)
    vdev = p.field(V.astype(np.complex128))  # device copy; real part read below via a real buffer
    # a real (double) array: reinterpret the first half of a complex field buffer
    vreal = np.asfortranarray(V.astype(np.float64))
    vbuf = p.field()
    tmp = np.zeros(p.field_shape, dtype=np.complex128, order="F")
    tmp.reshape(-1, order="F").view(np.float64)[: vreal.size] = vreal.reshape(-1, order="F")
    vbuf.upload(tmp)
    f = abi.Functional(p, abi.GP5_FUNC_LHY, potential_ptr=vbuf.ptr.value)
    a, b = p.field(psi), p.field()
    f.apply(a, b)
    assert rel(b.download(), o.Functional("lhy", V=V).apply(psi, geo)) < 1e-12
    del vdev


# ---------------------------------------------------------------- norms
def test_norm_normalize_maxdensity(abi):
    geo = o.Geometry((50, 50, 50), (-5,) * 3, (5,) * 3)
    X, Y, Z = o.grid(geo)
    psi = o.new_field(geo)
    psi[..., 0] = np.exp(-(X * X + Y * Y + Z * Z))
    p = make(abi, geo.shape, geo.left, geo.right)
    a = p.field(psi)
    assert abs(p.norm(a) - o.norm(psi, 0, geo)) / o.norm(psi, 0, geo) < 1e-13
    p.normalize(a, 1.0)
    assert abs(p.norm(a) - 1.0) < 1e-13  # test.py:141
    ref = psi.copy()
    o.normalize(1.0, ref, 0, geo)
    assert rel(a.download(), ref) < 1e-14
    assert abs(p.max_density(a) - np.max(np.abs(ref) ** 2)) < 1e-15 * np.max(np.abs(ref) ** 2) * 4


# ---------------------------------------------------------------- steppers
def test_steps_golden(abi):
    z = np.load(os.path.join(GOLD, "gp_steps_12x10x8.npz"))
    p = make(abi, (12, 10, 8), tuple(z["left"]), tuple(z["right"]))
    f = abi.Functional(p, abi.GP5_FUNC_GP, couplings=[[1.0]], omegas=[(1.0, 1.0, 1.0)])
    rk = abi.Stepper(f, 1e-3, abi.GP5_STEP_RK4, imaginary=True)
    a = p.field(z["psi"])
    rk.advance(a, 1)
    assert rel(a.download(), z["rk4_imag"]) < 1e-12
    eu = abi.Stepper(f, 1e-3, abi.GP5_STEP_EULER, imaginary=False)
    b = p.field(z["psi"])
    eu.advance(b, 1)
    assert rel(b.download(), z["euler_real"]) < 1e-12
    assert abs(rk.time - 1e-3) < 1e-18


def test_rk4_renorm_golden(abi):
    z = np.load(os.path.join(GOLD, "lhy_rk4_renorm_10x12x14.npz"))
    p = make(abi, (10, 12, 14), tuple(z["left"]), tuple(z["right"]))
    f = abi.Functional(p, abi.GP5_FUNC_LHY)
    st = abi.Stepper(f, 2e-3)
    st.set_renormalization([25.0])
    a = p.field(z["psi"])
    st.advance(a, 3)
    assert rel(a.download(), z["out"]) < 1e-12


def config1(n=64):
    geo = o.Geometry((n, n, n), (-10,) * 3, (10,) * 3)
    psi = o.gaussian_with_noise(geo, 1.0, 1e-3, seed=2024, N=1.0)
    of = o.Functional("gp", couplings=[[1.0]], V=o.harmonic_potential(geo, [(1, 1, 1)]))
    return geo, psi, of


def test_rk4_one_step_config1(abi):
    geo, psi, of = config1()
    p = make(abi, geo.shape, geo.left, geo.right)
    f = abi.Functional(p, abi.GP5_FUNC_GP, couplings=[[1.0]], omegas=[(1, 1, 1)])
    st = abi.Stepper(f, 1e-3)
    a = p.field(psi)
    st.advance(a, 1)
    ref = o.Stepper(of, geo, 1e-3).advance(psi.copy(), 1)
    assert rel(a.download(), ref) < 1e-12


def test_rk4_1000_steps_config1(abi):
    """Config 1: 64^3 harmonic GP, imaginary RK4 dt=1e-3, 1000 steps; psi, E, mu vs oracle."""
    geo, psi, of = config1()
    p = make(abi, geo.shape, geo.left, geo.right)
    f = abi.Functional(p, abi.GP5_FUNC_GP, couplings=[[1.0]], omegas=[(1, 1, 1)])
    st = abi.Stepper(f, 1e-3)
    a = p.field(psi)
    st.advance(a, 1000)
    got = a.download()
    ref = o.Stepper(of, geo, 1e-3).advance(psi.copy(), 1000)
    assert rel(got, ref) < 1e-10
    go = f.observables(a)
    ob = o.observables(of, ref, geo)
    for k in ("energy", "mu"):
        rk = "E" if k == "energy" else k
        assert abs(go[k] - ob[rk]) / abs(ob[rk]) < 1e-10, (k, go[k], ob[rk])
    assert abs(go["residual"] - ob["residual"]) < 1e-8
    assert abs(st.time - 1.0) < 1e-9


def test_real_time_lhy_steps(abi):
    geo = o.Geometry((32, 32, 32), (-8,) * 3, (8,) * 3)
    psi = o.gaussian_with_noise(geo, 2.0, 1e-3, seed=9, N=60.0, phase_noise=True)
    p = make(abi, geo.shape, geo.left, geo.right)
    f = abi.Functional(p, abi.GP5_FUNC_LHY, c3=-3.3)
    st = abi.Stepper(f, 1e-3, imaginary=False)
    a = p.field(psi)
    st.advance(a, 20)
    ref = o.Stepper(o.Functional("lhy", c3=-3.3), geo, 1e-3, imaginary=False).advance(psi.copy(), 20)
    assert rel(a.download(), ref) < 1e-12


def test_phase_constraint_and_two_component_step(abi):
    geo = o.Geometry((16, 16, 12), (-5,) * 3, (5,) * 3)
    rng = np.random.default_rng(3)
    psi = o.new_field(geo, 2)
    o.init_gaussian(geo, 1.5, psi, 0)
    o.init_gaussian(geo, 1.8, psi, 1)
    phase = np.asfortranarray(rng.uniform(-3, 3, psi.shape))
    p = make(abi, geo.shape, geo.left, geo.right, ncomp=2)
    G = np.array([[1.0, 0.2], [0.2, 0.5]])
    f = abi.Functional(p, abi.GP5_FUNC_GP, couplings=G)
    st = abi.Stepper(f, 1e-3)
    st.set_renormalization([2.0, 3.0])
    # the phase is a real array in the plan precision: pack it into a device buffer
    pbuf = p.field()
    tmp = np.zeros(p.field_shape, dtype=np.complex128, order="F")
    tmp.reshape(-1, order="F").view(np.float64)[: phase.size] = phase.reshape(-1, order="F")
    pbuf.upload(tmp)
    st.set_phase_constraint(pbuf)
    a = p.field(psi)
    st.advance(a, 2)
    of = o.Functional("gp", couplings=G)
    ref = o.Stepper(of, geo, 1e-3, normalizations=[2.0, 3.0], constraint_phase=phase).advance(psi.copy(), 2)
    assert rel(a.download(), ref) < 1e-12


def test_observables_vs_oracle(abi):
    geo = o.Geometry((40, 36, 32), (-8,) * 3, (8,) * 3)
    psi = o.gaussian_with_noise(geo, 2.0, 1e-2, seed=4, N=80.0, phase_noise=True)
    p = make(abi, geo.shape, geo.left, geo.right)
    a = p.field(psi)
    for f, of in ((abi.Functional(p, abi.GP5_FUNC_LHY), o.Functional("lhy")),
                  (abi.Functional(p, abi.GP5_FUNC_GP, couplings=[[0.7]], omegas=[(1, 0.8, 1.2)]),
                   o.Functional("gp", couplings=[[0.7]], V=o.harmonic_potential(geo, [(1, 0.8, 1.2)])))):
        g = f.observables(a)
        r = o.observables(of, psi, geo)
        assert abs(g["norm"] - r["norm"]) / r["norm"] < 1e-13
        for k, rk in (("energy", "E"), ("ekin", "ekin"), ("eint", "eint"), ("mu", "mu")):
            assert abs(g[k] - r[rk]) / max(abs(r[rk]), 1e-300) < 1e-12, k
        assert abs(g["residual"] - r["residual"]) / r["residual"] < 1e-10


def test_lhy_mu_protocol_30cubed(abi):
    """python/test/regressionTests/LHY_imaginary.py on the GPU: the oracle restatement converges
    to -0.38366638260724; the reference's committed golden is -0.38372999 (within 1e-4)."""
    geo = o.Geometry((30, 30, 30), (-10,) * 3, (10,) * 3)
    psi0 = o.new_field(geo)
    o.init_gaussian(geo, 5.0, psi0)
    p = make(abi, geo.shape, geo.left, geo.right)
    a = p.field(psi0)
    N = 370.0
    p.normalize(a, N)
    f = abi.Functional(p, abi.GP5_FUNC_LHY)
    dt = 0.01 * geo.space_step(0) ** 2
    st = abi.Stepper(f, dt)
    old, mu, it = 0.0, 1e18, 0
    while abs(mu - old) > 1e-9 and it < 40:
        it += 1
        for _ in range(1000):
            p.normalize(a, N)
            st.advance(a, 1)
        old, mu = mu, 0.5 * math.log(N / p.norm(a)) / dt
        p.normalize(a, N)
    assert abs(mu - (-0.3836663826072363)) < 1e-10
    assert abs(mu - (-0.3837299937094331)) < 1e-4


# ---------------------------------------------------------------- precision / determinism
def test_fp32_step_error_vs_fp64(abi):
    geo = o.Geometry((64, 64, 64), (-10,) * 3, (10,) * 3)
    psi = o.gaussian_with_noise(geo, 2.5, 1e-3, seed=6, N=200.0, phase_noise=True)
    out = []
    for prec in (0, 1):
        p = make(abi, geo.shape, geo.left, geo.right, prec=prec)
        f = abi.Functional(p, abi.GP5_FUNC_LHY, c3=-3.3)
        st = abi.Stepper(f, 5e-4, imaginary=False)
        a = p.field(psi)
        st.advance(a, 10)
        out.append((a.download(), f.observables(a)))
    assert rel(out[1][0], out[0][0]) < 1e-5
    assert abs(out[1][1]["energy"] - out[0][1]["energy"]) / abs(out[0][1]["energy"]) < 1e-6
    assert abs(out[1][1]["norm"] - out[0][1]["norm"]) / out[0][1]["norm"] < 1e-6


def test_bitwise_deterministic(abi):
    geo = o.Geometry((64, 32, 48), (-6,) * 3, (6,) * 3)
    psi = o.gaussian_with_noise(geo, 1.5, 1e-2, seed=10, N=40.0, phase_noise=True)
    res = []
    for _ in range(2):
        p = make(abi, geo.shape, geo.left, geo.right)
        f = abi.Functional(p, abi.GP5_FUNC_LHY)
        st = abi.Stepper(f, 1e-3)
        st.set_renormalization([40.0])
        a = p.field(psi)
        st.advance(a, 5)
        res.append((a.download(), f.observables(a)))
    assert np.array_equal(res[0][0], res[1][0])
    assert res[0][1] == res[1][1]


def test_host_buffer_entry_point(abi):
    geo, psi, of = config1(32)
    p = make(abi, geo.shape, geo.left, geo.right)
    f = abi.Functional(p, abi.GP5_FUNC_GP, couplings=[[1.0]], omegas=[(1, 1, 1)])
    st = abi.Stepper(f, 1e-3)
    host = np.asfortranarray(psi.copy())
    out = np.empty_like(host)
    st.advance_host(host, out, 3)
    ref = o.Stepper(of, geo, 1e-3).advance(psi.copy(), 3)
    assert rel(out, ref) < 1e-12


def test_errors_are_reported(abi):
    with pytest.raises(abi.Gp5Error) as e:
        abi.Plan((1, 8, 8), (-1,) * 3, (1,) * 3)
    assert e.value.status == abi.GP5_ERR_ARG
    with pytest.raises(abi.Gp5Error) as e:
        abi.Plan((2 * 67, 4, 4), (-1,) * 3, (1,) * 3)  # prime factor 67 > 61
    assert e.value.status == abi.GP5_ERR_UNSUPPORTED
    p = make(abi, (8, 8, 8))
    with pytest.raises(abi.Gp5Error):
        abi.Functional(p, abi.GP5_FUNC_LHY_UNLOCKED)  # needs two components
    f = abi.Functional(p, abi.GP5_FUNC_LHY)
    a = p.field()
    with pytest.raises(abi.Gp5Error):
        f.apply(a, a)  # src == dst


def test_nonfinite_is_reported(abi):
    geo = o.Geometry((16, 16, 16), (-4,) * 3, (4,) * 3)
    psi = o.gaussian_with_noise(geo, 1.0, 0.0, seed=0, N=1.0)
    psi[3, 3, 3, 0] = np.nan
    p = make(abi, geo.shape, geo.left, geo.right)
    f = abi.Functional(p, abi.GP5_FUNC_LHY)
    st = abi.Stepper(f, 1e-3)
    st.set_renormalization([1.0])
    a = p.field(psi)
    with pytest.raises(abi.Gp5Error) as e:
        st.advance(a, 1)
    assert e.value.status == abi.GP5_ERR_NONFINITE


def test_two_component_laplacian_reference_case(abi):
    """tst/fft_test.cpp:156-215 (derivative_multipleComponents, a smoke test there): two
    components, N = (200, 100, 100), box [-1,1]x[-1/2,1/2]^2, Gaussians of width 0.05 and
    0.02; here checked against the analytic Laplacian of each component and the oracle."""
    geo = o.Geometry((200, 100, 100), (-1.0, -0.5, -0.5), (1.0, 0.5, 0.5))
    f = o.new_field(geo, 2)
    o.init_gaussian(geo, 0.05, f, 0)
    o.init_gaussian(geo, 0.02, f, 1)
    p = make(abi, geo.shape, geo.left, geo.right, ncomp=2)
    a, b = p.field(f), p.field()
    p.laplacian(a, b)
    got = b.download()
    assert rel(got, o.laplacian(f, geo)) < 1e-12
    X, Y, Z = o.grid(geo)
    R2 = X * X + Y * Y + Z * Z
    for c, s in ((0, 0.05), (1, 0.02)):
        al = 1 / (2 * s * s)
        ref = np.exp(-al * R2) * (-R2 * al * 2 + 3) * (-2) * al
        assert np.max(np.abs(got[..., c].real - ref)) <= 1e-6 * np.max(np.abs(ref)), c
