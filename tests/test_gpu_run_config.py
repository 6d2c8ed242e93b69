"""The YAML front end run on the GPU against the oracle's stepper."""
import numpy as np
import pytest

from oracle import gp_oracle as o

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_trapped_gp_imaginary_rk4(tmp_path):
    from gp5_b200 import run as R
    from test_run_config import base_cfg
    c = base_cfg()
    s = R.build_spec(c)
    geo = o.Geometry(tuple(s["shape"]), tuple(s["left"]), tuple(s["right"]))
    psi = o.gaussian_with_noise(geo, 1.5, 1e-3, seed=4, N=50.0)
    np.save(tmp_path / "init.npy", psi)
    r = R.run(c, base=str(tmp_path), log=lambda *_: None)
    assert len(r["files"]) == 2 and r["steps"] == 20
    assert all(f.endswith(".hdf5") for f in r["files"])  # out_<k>.hdf5, as the reference writes
    out1 = R.read_array(r["files"][1])
    assert np.array_equal(R.read_array(r["files"][0]), psi)
    V = o.harmonic_potential(geo, [(1.0, 0.8, 1.2)])
    f = o.Functional("gp", couplings=np.array([[0.7]]), masses=[1.0], V=V)
    ref = o.Stepper(f, geo, 1e-3, "RK4", True, normalizations=[50.0]).advance(psi.copy(), 10)
    assert rel(out1, ref) < 1e-12


def test_unlocked_droplet_with_file_potential_and_phase(tmp_path):
    from gp5_b200 import run as R
    from test_run_config import base_cfg
    c = base_cfg()
    c["wavefunction"] = {"nComponents": 2, "normalization": [20, 30]}
    c["functional"] = {"d": {"name": "UnlockedLHYDroplet", "eta": -4, "alpha": 0.88, "beta": 1.0},
                       "V": {"name": "externalPotential",
                             "V": {"f": {"name": "potentialFromFile", "filename": "V.npy"},
                                   "v": {"name": "vortex"}}}}
    c["evolution"].update(stepper="eulero", reNormalize=False, imaginaryTime=False, timeStep=5e-4)
    c["evolution"]["constraint"] = {"p": {"name": "phaseConstraint", "file": "phase.npy"}}
    s = R.build_spec(c)
    geo = o.Geometry(tuple(s["shape"]), tuple(s["left"]), tuple(s["right"]))
    rng = np.random.default_rng(1)
    psi = o.new_field(geo, 2)
    o.init_gaussian(geo, 1.5, psi, 0)
    o.init_gaussian(geo, 2.0, psi, 1)
    psi = np.asfortranarray(psi * 0.3)
    Vf = np.asfortranarray(rng.uniform(0, 0.5, psi.shape))
    phase = np.asfortranarray(rng.uniform(-3, 3, psi.shape))
    np.save(tmp_path / "init.npy", psi)
    np.save(tmp_path / "V.npy", Vf)
    np.save(tmp_path / "phase.npy", phase)
    r = R.run(c, base=str(tmp_path), log=lambda *_: None)
    X, Y, Z = o.grid(geo)
    V = Vf + (0.5 / (X * X + Y * Y))[..., None]
    f = o.Functional("lhy_unlocked", alpha=0.88, beta=1.0, eta=-4.0, V=V)
    ref = o.Stepper(f, geo, 5e-4, "eulero", False, constraint_phase=phase).advance(psi.copy(), 10)
    assert rel(R.read_array(r["files"][1]), ref) < 1e-12
