"""YAML front end: the reference's `gp` executable (src/main.cpp:14-249) as a driver over the
C ABI, with the same configuration keys.

    python -m gp5_b200.run config.yaml [--device 0]

Keys (src/main.cpp:32-166, src/functional.cpp:154-258, src/externalPotential.cpp:84-122,
src/constraint.cpp:19-37):
  mesh.shape, domain.left/right, parallel.processorGrid (must be [1,1,1]: one GPU holds the
  grid; parallel.fftOrdering is accepted and ignored), wavefunction.nComponents /
  normalization, functional.<any>: {name: gpFunctional (coupling, masses) | LHYDroplet (c3, c4:
  extension, defaults -3 and 5/2) | UnlockedLHYDroplet (alpha, beta, eta) | externalPotential
  (V.<any>: {name: harmonic (omegas) | vortex | potentialFromFile (filename)})},
  evolution.timeStep / imaginaryTime / stepper (RK4 | eulero) / maxTime / reNormalize /
  constraint.<any>: {name: phaseConstraint, file}, initialCondition.file, output.folder /
  nIterations.

Loop (src/main.cpp:176-205): while t <= maxTime: save the state to <folder>/out_<k>; advance
nIterations steps (t += timeStep per step); k += 1.

Files: fields, potentials and phases are HDF5 files in the reference's layout (src/io.cpp:
dataset "field", complex elements, dims [nComp][Nz][Ny][Nx]), read and written by the
library's own HDF5 code (gp5cu_h5_*); the states are saved as <folder>/out_<k>.hdf5 like the
reference's executable (src/main.cpp:193).  A .npy path holds the same payload as a
(nx, ny, nz, ncomp) numpy array.
"""
from __future__ import annotations

import math
import os
from typing import Optional

import numpy as np

from . import _abi


class ConfigError(RuntimeError):
    pass


def _vec(x, n, what):
    v = list(x)
    if len(v) != n:
        raise ConfigError(f"{what}: expected {n} values")
    return v


def build_spec(cfg: dict) -> dict:
    """Validated run description from a parsed configuration (no GPU work)."""
    shape = [int(v) for v in _vec(cfg["mesh"]["shape"], 3, "mesh.shape")]
    left = [float(v) for v in _vec(cfg["domain"]["left"], 3, "domain.left")]
    right = [float(v) for v in _vec(cfg["domain"]["right"], 3, "domain.right")]
    par = cfg.get("parallel", {}) or {}
    pg = [int(v) for v in par.get("processorGrid", [1, 1, 1])]
    if int(np.prod(pg)) != 1:
        raise ConfigError("one GPU holds the whole grid: processorGrid must be [1,1,1]")
    wf = cfg["wavefunction"]
    nc = int(wf["nComponents"])
    norms = [float(v) for v in wf.get("normalization", [])]

    func = dict(kind=None, couplings=None, masses=None, c3=-3.0, c4=2.5, alpha=0.0, beta=0.0, eta=0.0,
                potentials=[])
    for _, fc in (cfg.get("functional") or {}).items():
        name = fc["name"]
        if name == "gpFunctional":
            func["kind"] = _abi.GP5_FUNC_GP
            if "coupling" in fc:
                g = fc["coupling"]
                if len(g) != nc or any(len(row) != nc for row in g):
                    raise ConfigError("Incompatible number of components")
                # couplings(i, j) = coupling[j][i] (src/functional.cpp:172-190)
                func["couplings"] = [[float(g[j][i]) for j in range(nc)] for i in range(nc)]
            if "masses" in fc:
                func["masses"] = [float(m) for m in fc["masses"]]
        elif name == "LHYDroplet":
            func["kind"] = _abi.GP5_FUNC_LHY
            func["c3"] = float(fc.get("c3", -3.0))
            func["c4"] = float(fc.get("c4", 2.5))
        elif name == "UnlockedLHYDroplet":
            func["kind"] = _abi.GP5_FUNC_LHY_UNLOCKED
            func["alpha"], func["beta"], func["eta"] = float(fc["alpha"]), float(fc["beta"]), float(fc["eta"])
        elif name == "externalPotential":
            for _, pc in (fc.get("V") or {}).items():
                pname = pc["name"]
                if pname == "harmonic":
                    om = [[float(w) for w in _vec(row, 3, "omegas")] for row in pc["omegas"]]
                    if len(om) < nc:
                        raise ConfigError("Incompatible number of components")
                    func["potentials"].append(("harmonic", om))
                elif pname == "vortex":
                    func["potentials"].append(("vortex", None))
                elif pname == "potentialFromFile":
                    func["potentials"].append(("file", str(pc["filename"])))
                else:
                    raise ConfigError("Unkown potential")
        else:
            raise ConfigError(" Unkown functional")
    if func["kind"] is None:
        raise ConfigError("no functional in the configuration")

    ev = cfg["evolution"]
    name = ev["stepper"]
    if name not in ("RK4", "eulero"):
        raise ConfigError("allowed steppers: RK4, eulero")
    constraint = None
    for _, cc in (ev.get("constraint") or {}).items():
        if cc["name"] == "phaseConstraint":
            constraint = str(cc["file"])
            break
    out = cfg["output"]
    return dict(shape=shape, left=left, right=right, ncomp=nc, normalizations=norms, functional=func,
                stepper=_abi.GP5_STEP_RK4 if name == "RK4" else _abi.GP5_STEP_EULER,
                dt=float(ev["timeStep"]), imaginary=bool(ev["imaginaryTime"]),
                renormalize=bool(ev.get("reNormalize", False)), max_time=float(ev["maxTime"]),
                constraint=constraint, init=str(cfg["initialCondition"]["file"]),
                folder=str(out["folder"]), every=int(out["nIterations"]))


def read_array(path: str, base: str = "") -> np.ndarray:
    """A field, potential or phase file (gp::load, src/io.cpp:154-256) as a (nx, ny, nz, ncomp)
    complex array; .npy files hold the same payload."""
    p = path if os.path.isabs(path) or not base else os.path.join(base, path)
    if p.endswith((".hdf5", ".h5")):
        try:
            return _abi.h5_load_field(p)
        except _abi.Gp5Error as e:
            raise ConfigError(f"{p}: {e}") from e
    return np.load(p)


def write_array(path: str, a: np.ndarray) -> str:
    """Saves a field (gp::save, src/io.cpp:56-152): HDF5 unless the path ends in .npy; a path
    without an extension gets .hdf5 (out_<k>.hdf5, src/main.cpp:193).  Returns the file name."""
    if path.endswith(".npy"):
        np.save(path, np.asfortranarray(a))
        return path
    p = path if path.endswith((".hdf5", ".h5")) else path + ".hdf5"
    _abi.h5_save_field(p, np.asarray(a))
    return p


def _positions(spec):
    return [spec["left"][d] + (np.arange(spec["shape"][d]) + 0.5) * (spec["right"][d] - spec["left"][d]) /
            spec["shape"][d] for d in range(3)]


def potential_array(spec, base: str = "") -> Optional[np.ndarray]:
    """sumPotential (src/externalPotential.cpp:59-72): the listed potentials added to 0 in order;
    None when there is none."""
    pots = spec["functional"]["potentials"]
    if not pots:
        return None
    nx, ny, nz = spec["shape"]
    nc = spec["ncomp"]
    x, y, z = _positions(spec)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    V = np.zeros((nx, ny, nz, nc))
    for kind, arg in pots:
        if kind == "harmonic":
            for c in range(nc):
                w = arg[c]
                V[..., c] += (w[0] * w[0] * X * X + w[1] * w[1] * Y * Y + w[2] * w[2] * Z * Z) * 0.5
        elif kind == "vortex":
            V += (0.5 / (X * X + Y * Y))[..., None]
        else:
            V += np.real(read_array(arg, base)).reshape(nx, ny, nz, nc, order="F")
    return np.asfortranarray(V)


def _real_buffer(plan: "_abi.Plan", real: np.ndarray):
    """A real array in the plan precision packed into a device field buffer."""
    buf = plan.field()
    tmp = np.zeros(plan.field_shape, dtype=np.complex128, order="F")
    flat = tmp.reshape(-1, order="F")
    if plan.precision == _abi.GP5_C128:
        flat.view(np.float64)[: real.size] = np.asarray(real, np.float64).reshape(-1, order="F")
        buf.upload(tmp)
    else:
        host = np.zeros(plan.field_shape, dtype=np.complex64, order="F")
        host.reshape(-1, order="F").view(np.float32)[: real.size] = np.asarray(real, np.float32).reshape(-1, order="F")
        _abi.check(_abi.lib().gp5cu_upload(plan.h, buf.ptr, _abi.C.c_void_p(host.ctypes.data)))
    return buf


def run(cfg, device: int = 0, precision: int = _abi.GP5_C128, base: str = "", log=print) -> dict:
    """Runs a configuration (a dict or a YAML path); returns the output files and final time."""
    if isinstance(cfg, str):
        import yaml
        base = base or os.path.dirname(os.path.abspath(cfg))
        with open(cfg) as fh:
            cfg = yaml.safe_load(fh)
    spec = build_spec(cfg)
    f = spec["functional"]
    plan = _abi.Plan(spec["shape"], spec["left"], spec["right"], ncomp=spec["ncomp"], precision=precision,
                     device=device)
    V = potential_array(spec, base)
    vbuf = None
    kw = dict(couplings=f["couplings"], masses=f["masses"], c3=f["c3"], c4=f["c4"], alpha=f["alpha"],
              beta=f["beta"], eta=f["eta"])
    if V is not None and len(f["potentials"]) == 1 and f["potentials"][0][0] == "harmonic":
        kw["omegas"] = f["potentials"][0][1]  # the device forms the same harmonic values
    elif V is not None:
        vbuf = _real_buffer(plan, V)
        kw["potential_ptr"] = vbuf.ptr.value
    func = _abi.Functional(plan, f["kind"], **kw)
    st = _abi.Stepper(func, spec["dt"], spec["stepper"], imaginary=spec["imaginary"])
    if spec["renormalize"]:
        st.set_renormalization(spec["normalizations"])
    pbuf = None
    if spec["constraint"]:
        phase = np.real(read_array(spec["constraint"], base))
        pbuf = _real_buffer(plan, phase)
        st.set_phase_constraint(pbuf)
    psi = np.asarray(read_array(spec["init"], base), dtype=np.complex128)
    psi = np.asfortranarray(psi.reshape(tuple(spec["shape"]) + (spec["ncomp"],), order="F"))
    field = plan.field(psi)
    folder = spec["folder"] if os.path.isabs(spec["folder"]) or not base else os.path.join(base, spec["folder"])
    os.makedirs(folder, exist_ok=True)
    t, k, files = 0.0, 0, []
    while t <= spec["max_time"]:
        log(f"Time: {t}")
        files.append(write_array(os.path.join(folder, f"out_{k}"), field.download()))
        st.advance(field, spec["every"])
        for _ in range(spec["every"]):
            t += spec["dt"]
        k += 1
    return dict(files=files, time=t, steps=k * spec["every"])


def main(argv=None):
    import argparse

    ap = argparse.ArgumentParser(description="Run a GP5 YAML configuration on the GPU.")
    ap.add_argument("config")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--complex64", action="store_true", help="FP32 bulk arithmetic (FP64 reductions)")
    a = ap.parse_args(argv)
    r = run(a.config, device=a.device, precision=_abi.GP5_C64 if a.complex64 else _abi.GP5_C128)
    print(f"{len(r['files'])} outputs, {r['steps']} steps, t = {r['time']}")


if __name__ == "__main__":
    main()
