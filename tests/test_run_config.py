"""The YAML front end (gp5_b200/run.py): configuration parsing and host-side arrays on CPU."""
import math
import os

import numpy as np
import pytest

from gp5_b200 import run as R
from gp5_b200 import _abi


def base_cfg():
    return {
        "mesh": {"shape": [24, 20, 16]},
        "domain": {"left": [-6, -5, -4], "right": [6, 5, 4]},
        "parallel": {"processorGrid": [1, 1, 1], "fftOrdering": [2, 0, 1]},
        "wavefunction": {"nComponents": 1, "normalization": [50]},
        "functional": {"gp": {"name": "gpFunctional", "masses": [1.0], "coupling": [[0.7]]},
                       "V": {"name": "externalPotential",
                             "V": {"h": {"name": "harmonic", "omegas": [[1.0, 0.8, 1.2]]}}}},
        "evolution": {"timeStep": 1e-3, "imaginaryTime": True, "stepper": "RK4", "maxTime": 0.015,
                      "reNormalize": True},
        "initialCondition": {"file": "init.npy"},
        "output": {"folder": "out", "nIterations": 10},
    }


def test_spec_from_config():
    s = R.build_spec(base_cfg())
    assert s["shape"] == [24, 20, 16] and s["ncomp"] == 1 and s["normalizations"] == [50.0]
    f = s["functional"]
    assert f["kind"] == _abi.GP5_FUNC_GP and f["couplings"] == [[0.7]] and f["masses"] == [1.0]
    assert f["potentials"] == [("harmonic", [[1.0, 0.8, 1.2]])]
    assert s["stepper"] == _abi.GP5_STEP_RK4 and s["imaginary"] and s["renormalize"]
    assert s["every"] == 10 and s["max_time"] == 0.015 and s["constraint"] is None


def test_two_component_couplings_are_transposed_like_the_reference():
    c = base_cfg()
    c["wavefunction"] = {"nComponents": 2, "normalization": [1, 2]}
    c["functional"]["gp"]["coupling"] = [[1.0, 0.2], [0.3, 2.0]]
    c["functional"]["V"]["V"]["h"]["omegas"] = [[1, 1, 1], [2, 2, 2]]
    s = R.build_spec(c)
    # couplings(i, j) = coupling[j][i] (src/functional.cpp:172-190)
    assert s["functional"]["couplings"] == [[1.0, 0.3], [0.2, 2.0]]


@pytest.mark.parametrize("edit,msg", [
    (lambda c: c["functional"]["gp"].update(name="other"), "Unkown functional"),
    (lambda c: c["functional"]["V"]["V"]["h"].update(name="other"), "Unkown potential"),
    (lambda c: c["functional"]["gp"].update(coupling=[[1, 2], [3, 4]]), "Incompatible number of components"),
    (lambda c: c["parallel"].update(processorGrid=[2, 1, 1]), "processorGrid"),
    (lambda c: c["evolution"].update(stepper="leapfrog"), "allowed steppers")])
def test_config_errors(edit, msg):
    c = base_cfg()
    edit(c)
    with pytest.raises(R.ConfigError, match=msg):
        R.build_spec(c)


def test_potential_sum_and_files(tmp_path):
    c = base_cfg()
    vfile = tmp_path / "V.npy"
    extra = np.asfortranarray(np.random.default_rng(0).uniform(0, 1, (24, 20, 16, 1)))
    np.save(vfile, extra)
    c["functional"]["V"]["V"] = {"a": {"name": "harmonic", "omegas": [[1.0, 0.8, 1.2]]},
                                 "b": {"name": "vortex"},
                                 "c": {"name": "potentialFromFile", "filename": str(vfile)}}
    s = R.build_spec(c)
    V = R.potential_array(s)
    x, y, z = R._positions(s)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    ref = (X * X + 0.64 * Y * Y + 1.44 * Z * Z) * 0.5 + 0.5 / (X * X + Y * Y) + extra[..., 0]
    assert np.max(np.abs(V[..., 0] - ref)) < 1e-12
    p = R.write_array(str(tmp_path / "f"), extra.astype(complex))
    assert p.endswith("f.hdf5")
    back = R.read_array(p)
    assert np.array_equal(back, extra) and back.flags["F_CONTIGUOUS"]
    p = R.write_array(str(tmp_path / "g.npy"), extra.astype(complex))
    assert np.array_equal(R.read_array(p), extra)
    # a potential given as an HDF5 file in the reference's layout
    R.write_array(str(tmp_path / "V.hdf5"), extra.astype(complex))
    c["functional"]["V"]["V"]["c"]["filename"] = str(tmp_path / "V.hdf5")
    assert np.max(np.abs(R.potential_array(R.build_spec(c))[..., 0] - ref)) < 1e-12
    with pytest.raises(R.ConfigError, match="cannot open"):
        R.read_array(str(tmp_path / "x.hdf5"))


class _FakeField:
    def __init__(self, plan, host=None):
        self.plan = plan
        self.a = np.zeros(plan.field_shape, complex) if host is None else np.array(host, complex)
        self.ptr = type("P", (), {"value": 0})()

    def download(self):
        return self.a.copy()

    def upload(self, host):
        self.a = np.array(host, complex)


class _FakePlan:
    def __init__(self, shape, left, right, ncomp=1, precision=0, device=0):
        self.field_shape = tuple(shape) + (ncomp,)
        self.precision = precision
        self.h = None

    def field(self, host=None):
        return _FakeField(self, host)


class _FakeFunctional:
    def __init__(self, plan, kind, **kw):
        self.kw = kw


class _FakeStepper:
    calls = []

    def __init__(self, func, dt, kind, imaginary=True):
        self.dt = dt

    def set_renormalization(self, N):
        pass

    def set_phase_constraint(self, p):
        pass

    def advance(self, f, n):
        _FakeStepper.calls.append(n)
        f.a = f.a + n  # a trace of the steps taken


@pytest.mark.parametrize("max_time", [0.015, 0.02, 0.0])
def test_run_loop_outputs_and_time(tmp_path, monkeypatch, max_time):
    monkeypatch.setattr(R._abi, "Plan", _FakePlan)
    monkeypatch.setattr(R._abi, "Functional", _FakeFunctional)
    monkeypatch.setattr(R._abi, "Stepper", _FakeStepper)
    _FakeStepper.calls = []
    c = base_cfg()
    c["evolution"]["maxTime"] = max_time
    np.save(tmp_path / "init.npy", np.zeros((24, 20, 16, 1), complex))
    r = R.run(c, base=str(tmp_path), log=lambda *_: None)
    # the reference's loop: while t <= maxTime { save; nIterations x (advance; t += dt) }
    t, k = 0.0, 0
    while t <= max_time:
        for _ in range(10):
            t += 1e-3
        k += 1
    assert len(r["files"]) == k and r["steps"] == 10 * k and r["time"] == t
    assert _FakeStepper.calls == [10] * k
    for j, fpath in enumerate(r["files"]):
        assert fpath.endswith(f"out_{j}.hdf5") and os.path.dirname(fpath) == str(tmp_path / "out")
        assert np.all(R.read_array(fpath) == 10 * j)  # out_j is saved before block j advances
