"""CPU oracle of the GP5 hot path: test infrastructure, never the product.

Only tests/, the smoke check and bench.py's CPU-baseline leg import it.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_DFT_LIB = os.path.join(_HERE, "_build", "libdft_ld.so")


def build():
    """Compile the long-double DFT (oracle/dft_ld.c) with the committed Makefile."""
    import subprocess
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def dft3_ld(psi: np.ndarray, direction: int) -> np.ndarray:
    """Long-double direct 3D DFT of a (nx, ny, nz, ncomp) field, unnormalised."""
    if not os.path.exists(_DFT_LIB):
        build()
    lib = ctypes.CDLL(_DFT_LIB)
    a = np.asarray(psi, dtype=np.complex128)
    nx, ny, nz, nc = a.shape
    src = np.asfortranarray(a).ravel(order="F").view(np.float64).copy()
    dst = np.empty_like(src)
    lib.dft3_ld(ctypes.c_int(nx), ctypes.c_int(ny), ctypes.c_int(nz), ctypes.c_int(nc),
                src.ctypes.data_as(ctypes.c_void_p), dst.ctypes.data_as(ctypes.c_void_p),
                ctypes.c_int(direction))
    return dst.view(np.complex128).reshape((nx, ny, nz, nc), order="F")


_CLUSTER_LIB = os.path.join(_HERE, "_build", "libcluster.so")


def decompose(psi: np.ndarray, cutoff: float, comp: int = 0):
    """Droplet labels of gp::decompose::decompose (src/cluster.cpp:17-83): int32 array of the
    field's shape (nx, ny, nz, ncomp), Fortran order; returns (labels, number of clusters)."""
    if not os.path.exists(_CLUSTER_LIB):
        build()
    lib = ctypes.CDLL(_CLUSTER_LIB)
    a = np.asarray(psi, dtype=np.complex128)
    if a.ndim == 3:
        a = a[..., None]
    nx, ny, nz, nc = a.shape
    src = np.asfortranarray(a).ravel(order="F").view(np.float64).copy()
    out = np.zeros(nx * ny * nz * nc, dtype=np.int32)
    lib.decompose.restype = ctypes.c_int
    k = lib.decompose(ctypes.c_int(nx), ctypes.c_int(ny), ctypes.c_int(nz), ctypes.c_int(comp),
                      src.ctypes.data_as(ctypes.c_void_p), ctypes.c_double(cutoff),
                      out.ctypes.data_as(ctypes.c_void_p))
    if k < 0:
        raise MemoryError("decompose: stack allocation failed")
    return out.reshape((nx, ny, nz, nc), order="F"), k
