"""Python front end with the names and behaviour of the reference's ``gp`` package
(python/gp/gp.py:11-223), over the pybind11 ``gpCpp`` module of this package.

Differences from the reference:
  * one process, one GPU: mpi4py and netCDF4 are optional (imported only when used);
  * ``field.array`` returns a host copy of the device state (assign to it to upload);
  * ``field(..., precision="c64")`` selects complex64 bulk arithmetic;
  * ``GP`` (harmonic GP model) and ``model.observables`` (E, mu, residual) are extensions;
  * ``save``/``load`` of .hdf5/.h5 files use the reference's HDF5 layout (dataset "field",
    element double[2], dims [nComp][Nz][Ny][Nx], src/io.cpp:41-135) through gpCpp.field.save
    and gpCpp.field.load, which read and write the format without libhdf5 or h5py; a .npy file
    name stores the same payload as a numpy array.
"""
from __future__ import annotations

import os
import re
from pathlib import Path

import numpy as np

from . import gpCpp

_PREC = {"c128": gpCpp.C128, "complex128": gpCpp.C128, "c64": gpCpp.C64, "complex64": gpCpp.C64}


class geometry:
    def __init__(self, shape, left=(-1, -1, -1), right=(1, 1, 1)):
        self._geometryCpp = gpCpp.geometry(list(left), list(right), list(shape))

    @property
    def left(self):
        return self._geometryCpp.getLeft()

    @property
    def right(self):
        return self._geometryCpp.getRight()

    @property
    def shape(self):
        return self._geometryCpp.getShape()

    @property
    def spaceStep(self):
        return [(self.right[d] - self.left[d]) / self.shape[d] for d in range(len(self.shape))]


class field:
    def __init__(self, geo, nComponents=1, processorGrid=(1, 1, 1), fftOrdering=(2, 0, 1), precision="c128",
                 device=0):
        self._nComponents = nComponents
        self._geometry = geo
        self._fieldCpp = gpCpp.field(geo._geometryCpp, nComponents, list(processorGrid), list(fftOrdering),
                                     _PREC[precision], device)

    @property
    def localShape(self):
        return self._fieldCpp.getLocalShape()

    @property
    def array(self):
        return self._fieldCpp.getTensor()

    @array.setter
    def array(self, x):
        x = np.asarray(x)
        if x.ndim == 3:
            x = x[..., None]
        self._fieldCpp.setTensor(np.asfortranarray(x.astype(np.complex128)))

    @property
    def nComponents(self):
        return self._nComponents

    def norm(self, component=None):
        if component is not None:
            return self._fieldCpp.getNorm(component)
        return [self.norm(c) for c in range(self.nComponents)]

    def normalize(self, N, component=None):
        if component is not None:
            self._fieldCpp.normalize(component, N)
        else:
            for Nc, c in zip(N, range(self.nComponents)):
                self.normalize(Nc, component=c)

    @property
    def offset(self):
        return self._fieldCpp.getOffset()

    def grid(self):
        """Cell-centred X, Y, Z of shape (nx, ny, nz, nComponents) (gp.py:77-95)."""
        meshShape = self.localShape
        left = self._geometry.left
        deltax = self._geometry.spaceStep
        axes = [(np.arange(0, meshShape[d]) + 0.5) * deltax[d] + left[d] + self.offset[d] * deltax[d]
                for d in range(3)]
        axes.append([1.0 for _ in range(self._nComponents)])
        X, Y, Z, _ = np.meshgrid(*axes, indexing="ij")
        return X, Y, Z

    def save(self, filename, format=None):
        if format is None:
            if re.match(r".*\.nc$", filename):
                format = "netCDF4"
            elif re.match(r".*\.(hdf5|h5)$", filename):
                format = "hdf5"
            elif re.match(r".*\.npy$", filename):
                format = "npy"
        if format is None:
            raise RuntimeError("Could not guess format.")
        Path(os.path.dirname(filename) or ".").mkdir(parents=True, exist_ok=True)
        if format == "netCDF4":
            self.saveNetCDF(filename)
        elif format == "hdf5":
            self.saveHDF5(filename)
        elif format == "npy":
            np.save(filename, self.array)
        else:
            raise RuntimeError("Unknown format {}".format(format))

    def saveHDF5(self, filename):
        """gp.field.saveHDF5 (python/gp/gp.py:127-131) through gpCpp.field.save: the
        reference's HDF5 layout (src/io.cpp:56-152), written by the library itself."""
        Path(os.path.dirname(filename) or ".").mkdir(parents=True, exist_ok=True)
        self._fieldCpp.save(filename)

    def saveNetCDF(self, filename):
        from netCDF4 import Dataset

        psi = self.array
        rho = np.abs(psi) ** 2
        phi = np.angle(psi)
        root = Dataset(filename, "w")
        root.createDimension("X", psi.shape[0])
        root.createDimension("Y", psi.shape[1])
        root.createDimension("Z", psi.shape[2])
        for c in range(psi.shape[3]):
            v = root.createVariable("rho{:d}".format(c), "f8", ("X", "Y", "Z"))
            v[:, :, :] = rho[:, :, :, c]
        for c in range(psi.shape[3]):
            v = root.createVariable("phi{:d}".format(c), "f8", ("X", "Y", "Z"))
            v[:, :, :] = phi[:, :, :, c]
        root.close()

    def load(self, filename):
        """gp.field.load (python/gp/gp.py:161-162): HDF5 files in the reference's layout
        (src/io.cpp:154-256) through gpCpp.field.load; .npy files hold the same payload."""
        if re.match(r".*\.(hdf5|h5)$", filename):
            self._fieldCpp.load(filename)
        else:
            self.array = np.load(filename)

    def maxDensity(self):
        return self._fieldCpp.maxDensity()


class _model:
    def apply(self, psi1, psi2, t=0):
        self._funcCpp.apply(psi1._fieldCpp, psi2._fieldCpp, t)

    def observables(self, psi):
        """Energy, chemical potential and residual of psi (extension)."""
        return self._funcCpp.observables(psi._fieldCpp)

    @property
    def nComponents(self):
        return self._funcCpp.nComponents()


class LHY(_model):
    def __init__(self, psi, c3=-3.0, c4=2.5):
        if psi.nComponents != 1:
            raise ValueError("Field should have one component")
        self._funcCpp = gpCpp.LHY(psi._fieldCpp, c3, c4)


class GP(_model):
    """gpFunctional (src/functional.cpp:13-102): couplings g_ij, masses, harmonic omegas."""

    def __init__(self, psi, couplings=None, masses=None, omegas=None):
        self._funcCpp = gpCpp.GP(psi._fieldCpp, couplings or [], masses or [], omegas or [])


class stepper:
    def __init__(self, model, timeStep, name="RK4", imaginary=True, renormalize=False, compensate=False):
        """name: str, allowed: RK4, eulero.  compensate (extension): compensated state update for
        complex64 fields (the part of psi below FP32 resolution is carried between steps)."""
        self._timeStep = timeStep
        self._name = name
        self._imaginary = imaginary
        self._stepperCpp = gpCpp.timeStepper(timeStep, name, imaginary)
        self._model = model
        self._stepperCpp.setFunctional(model._funcCpp)
        self._renormalize = False
        self._stepperCpp.unsetRenormalization()
        if compensate:
            self._stepperCpp.setCompensation(True)

    def setCompensation(self, on):
        self._stepperCpp.setCompensation(bool(on))

    def setStochasticRounding(self, on):
        """Extension: stochastically rounded complex64 state update (on by default for complex64
        fields; False rounds to nearest)."""
        self._stepperCpp.setStochasticRounding(bool(on))

    def setRenormalization(self, N):
        self._stepperCpp.setRenormalization(list(N))

    def advance(self, psi, nSteps=1):
        self._stepperCpp.advance(psi._fieldCpp, nSteps)

    @property
    def time(self):
        return self._stepperCpp.getTime()

    @property
    def timeStep(self):
        return self._timeStep


class maxDensity:
    def __init__(self):
        pass

    def __call__(self, psi, root=0):
        return psi.maxDensity()
