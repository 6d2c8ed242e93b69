"""The reference's Python tests (python/test/test.py) run against this package's ``gp`` API
(pybind11 gpCpp over the C ABI), single process.  test_geo needs no GPU; the others do."""
import math
import os

import numpy as np
import pytest

from oracle import gp_oracle as o


def test_geo():
    from gp5_b200 import gp
    geo = gp.geometry((100, 200, 50))  # test.py:10-18
    assert geo.shape == [100, 200, 50]
    assert geo.left == [-1, -1, -1]
    assert geo.right == [1, 1, 1]
    assert geo.spaceStep[0] == 2 / 100
    assert geo.spaceStep[1] == 2 / 200
    assert geo.spaceStep[2] == 2 / 50


@pytest.mark.gpu
def test_field():
    from gp5_b200 import gp
    geo = gp.geometry((100, 200, 50))  # test.py:20-45
    psi = gp.field(geo, nComponents=1, processorGrid=[1, 1, 1])
    assert psi.localShape == [100, 200, 50]
    for d in range(3):
        assert psi.array.shape[d] == psi.localShape[d]
    X, Y, Z = psi.grid()
    assert abs(np.min(X) - (geo.left[0] + geo.spaceStep[0] / 2)) < 1e-12
    assert abs(np.max(X) - (geo.right[0] - geo.spaceStep[0] / 2)) < 1e-12
    assert abs(X[1, 0, 0, 0] - X[0, 0, 0, 0] - geo.spaceStep[0]) < 1e-12
    psi.array = (X ** 2 + Y ** 2 + Z ** 2)
    assert abs(np.sum(psi.array - (X ** 2 + Y ** 2 + Z ** 2))) < 1e-9


@pytest.mark.gpu
def test_LHY():
    from gp5_b200 import gp
    geo = gp.geometry((100, 200, 50))
    psi = gp.field(geo, nComponents=1, processorGrid=[1, 1, 1])
    model = gp.LHY(psi)
    assert model.nComponents == 1
    psi2 = gp.field(geo, nComponents=2)
    with pytest.raises(ValueError):
        gp.LHY(psi2)


@pytest.mark.gpu
def test_LHY_apply():
    from gp5_b200 import gp
    geo = gp.geometry((100, 100, 100), left=[-4, -4, -4], right=[4, 4, 4])  # test.py:92-119
    psi1 = gp.field(geo, nComponents=1, processorGrid=[1, 1, 1])
    psi2 = gp.field(geo, nComponents=1, processorGrid=[1, 1, 1])
    model = gp.LHY(psi1)
    X, Y, Z = psi1.grid()
    r = np.sqrt(X ** 2 + Y ** 2 + Z ** 2)
    psi1.array = np.exp(-r ** 2) + 1j * 0
    model.apply(psi1, psi2, t=0)
    alpha = 1
    p1 = np.real(psi1.array)
    psi_expected = alpha * (3 - 2 * alpha * r ** 2) * p1 + (-3 * p1 ** 2 + 5 / 2 * p1 ** 3) * p1
    assert np.max(np.abs(psi_expected - np.real(psi2.array))) < 1e-4


@pytest.mark.gpu
def test_renormalize():
    from gp5_b200 import gp
    geo = gp.geometry((50, 50, 50), left=[-5, -5, -5], right=[5, 5, 5])  # test.py:123-147
    psi = gp.field(geo, nComponents=1, processorGrid=[1, 1, 1])
    X, Y, Z = psi.grid()
    r = np.sqrt(X ** 2 + Y ** 2 + Z ** 2)
    psi0 = np.exp(-r ** 2)
    psi.array = psi0
    psi.normalize(1, component=0)
    assert abs(psi.norm(0) - 1) < 1e-7
    psi.array = psi0
    psi.normalize([1])
    N = psi.norm()
    assert len(N) == 1
    assert abs(N[0] - 1) < 1e-7


@pytest.mark.gpu
def test_stepper_matches_oracle():
    """test.py:149-197 (50^3, box [-32,32], N=370, RK4 dt=0.1 dx^2), 4 blocks of 100 steps
    with normalisation before each step; mu of every block against the oracle."""
    from gp5_b200 import gp
    geo = gp.geometry((50, 50, 50), left=[-32, -32, -32], right=[32, 32, 32])
    psi = gp.field(geo, nComponents=1, processorGrid=[1, 1, 1])
    X, Y, Z = psi.grid()
    r = np.sqrt(X ** 2 + Y ** 2 + Z ** 2)
    psi.array = np.exp(-r ** 2 / (2 * 5 ** 2))
    N = 370
    psi.normalize([N])
    model = gp.LHY(psi)
    stepper = gp.stepper(timeStep=0.1 * geo.spaceStep[0] ** 2, name="RK4", model=model)

    ogeo = o.Geometry((50, 50, 50), (-32,) * 3, (32,) * 3)
    opsi = psi.array.copy()
    ost = o.Stepper(o.Functional("lhy"), ogeo, 0.1 * ogeo.space_step(0) ** 2)
    maxd = gp.maxDensity()
    for _ in range(4):
        for _ in range(100):
            psi.normalize([N])
            stepper.advance(psi, nSteps=1)
            o.normalize(N, opsi, 0, ogeo)
            opsi = ost.advance(opsi, 1)
        mu = 0.5 * np.log(N / psi.norm(0)) / stepper.timeStep
        omu = o.mu_from_norm_decay(N, o.norm(opsi, 0, ogeo), ost.dt)
        assert abs(mu - omu) < 1e-9 * abs(omu)
        psi.normalize([N])
        o.normalize(N, opsi, 0, ogeo)
        d0 = maxd(psi)
        assert abs(d0 - np.max(np.abs(opsi)) ** 2) < 1e-10 * d0
    assert abs(stepper.time - 400 * stepper.timeStep) < 1e-12


@pytest.mark.gpu
def test_io(tmp_path):
    from gp5_b200 import gp
    geo = gp.geometry((50, 50, 50), left=[-32, -32, -32], right=[32, 32, 32])  # test.py:200-217
    psi = gp.field(geo, nComponents=1, processorGrid=[1, 1, 1])
    X, Y, Z = psi.grid()
    r = np.sqrt(X ** 2 + Y ** 2 + Z ** 2)
    psi0 = np.exp(-r ** 2 / (2 * 5 ** 2))
    psi.array = psi0
    fn = os.path.join(str(tmp_path), "test.npy")
    psi.save(fn)
    psi.array = psi0 * 0
    psi.load(fn)
    assert abs(np.sum(np.abs(psi.array - psi0))) < 1e-12


@pytest.mark.gpu
def test_gp_model_observables_and_precision():
    from gp5_b200 import gp
    geo = gp.geometry((64, 64, 64), left=[-10] * 3, right=[10] * 3)
    psi = gp.field(geo)
    X, Y, Z = psi.grid()
    psi.array = np.exp(-(X ** 2 + Y ** 2 + Z ** 2) / 2)
    psi.normalize([1.0])
    model = gp.GP(psi, couplings=[[1.0]], omegas=[[1.0, 1.0, 1.0]])
    ob = model.observables(psi)
    ogeo = o.Geometry((64, 64, 64), (-10,) * 3, (10,) * 3)
    of = o.Functional("gp", couplings=[[1.0]], V=o.harmonic_potential(ogeo, [(1, 1, 1)]))
    r = o.observables(of, psi.array, ogeo)
    assert abs(ob["energy"] - r["E"]) < 1e-12 * abs(r["E"])
    assert abs(ob["mu"] - r["mu"]) < 1e-12 * abs(r["mu"])
    psi32 = gp.field(geo, precision="c64")
    psi32.array = psi.array
    m32 = gp.GP(psi32, couplings=[[1.0]], omegas=[[1.0, 1.0, 1.0]])
    st = gp.stepper(m32, 1e-3)
    st.advance(psi32, 10)
    st64 = gp.stepper(model, 1e-3)
    st64.advance(psi, 10)
    assert np.max(np.abs(psi32.array - psi.array)) < 1e-5 * np.max(np.abs(psi.array))


@pytest.mark.gpu
def test_field_save_load_hdf5(tmp_path):
    """gp.field.save / load of .hdf5 files (python/gp/gp.py:101-162 -> gpCpp.field.save / load,
    src/gpCpp.cpp:105-118) in the reference's layout (src/io.cpp: dataset "field",
    [nComp][Nz][Ny][Nx] of double[2]), through the library's own HDF5 writer and reader."""
    from gp5_b200 import _abi, gp
    geo = gp.geometry((12, 10, 8), left=[-3, -2, -1], right=[3, 2, 1])
    psi = gp.field(geo, nComponents=2)
    rng = np.random.default_rng(4)
    a = rng.standard_normal((12, 10, 8, 2)) + 1j * rng.standard_normal((12, 10, 8, 2))
    psi.array = a
    p = str(tmp_path / "sub" / "state.hdf5")
    psi.save(p)
    assert _abi.h5_field_shape(p) == ((12, 10, 8), 2)
    assert np.array_equal(_abi.h5_read_dataset(p, "field"), np.transpose(a, (3, 2, 1, 0)))
    other = gp.field(geo, nComponents=2)
    other.load(p)
    assert np.array_equal(other.array, a)
    wrong = gp.field(gp.geometry((12, 10, 6)), nComponents=2)
    with pytest.raises(RuntimeError):
        wrong.load(p)
