"""HDF5 field files in the reference's layout (gp5cu_h5_*), host side only.

The reference writes one dataset "field" in the root group with element
H5Tarray(double, [2]) and dims [nComp][Nz][Ny][Nx] (src/io.cpp:45, 77-90, 135), contiguous
storage, so the raw data is the field's own x-fastest memory order.  libhdf5 and h5py are not
installed here; the reader is pinned on a file the HDF5 library itself wrote (scipy's MATLAB
7.3 test file, an HDF5 file behind a 512-byte user block), and the writer is checked field by
field against the format it must produce and through round trips."""
import os
import struct

import numpy as np
import pytest

from gp5_b200 import _abi

SIG = b"\x89HDF\r\n\x1a\n"


def _field(shape, ncomp, seed):
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.standard_normal(shape + (ncomp,)) + 1j * rng.standard_normal(shape + (ncomp,)))


@pytest.mark.parametrize("shape,ncomp", [((8, 6, 4), 1), ((7, 5, 3), 2), ((1, 1, 1), 1), ((32, 30, 28), 2)])
def test_round_trip(tmp_path, shape, ncomp):
    psi = _field(shape, ncomp, sum(shape) + ncomp)
    p = str(tmp_path / "f.hdf5")
    _abi.h5_save_field(p, psi)
    assert _abi.h5_field_shape(p) == (shape, ncomp)
    back = _abi.h5_load_field(p)
    assert back.shape == shape + (ncomp,)
    assert np.array_equal(back, psi)


def test_written_layout_is_the_reference_layout(tmp_path):
    """Superblock 0, dataset "field" with dims [nComp][Nz][Ny][Nx], element array(2) of IEEE
    float64 little-endian, contiguous raw data = the field bytes in x-fastest order at the
    end of the file."""
    shape, ncomp = (5, 4, 3), 2
    psi = _field(shape, ncomp, 3)
    p = str(tmp_path / "f.h5")
    _abi.h5_save_field(p, psi)
    b = open(p, "rb").read()
    assert b[:8] == SIG and b[8] == 0  # signature, superblock version 0
    assert b[13] == 8 and b[14] == 8  # offsets and lengths of 8 bytes
    eof = struct.unpack_from("<Q", b, 40)[0]
    assert eof == len(b)
    raw = psi.tobytes(order="F")
    assert b[-len(raw):] == raw
    info = _abi.h5_read_dataset(p, "field")
    assert info.shape == (ncomp, shape[2], shape[1], shape[0])
    assert np.array_equal(info, np.transpose(psi, (3, 2, 1, 0)))
    # datatype message: class 10 (array) version 2, size 16, one dimension of 2, base float64
    i = b.index(bytes([0x2A, 0, 0, 0, 16, 0, 0, 0, 1, 0, 0, 0, 2, 0, 0, 0]))
    assert b[i + 20:i + 28] == bytes([0x11, 0x20, 63, 0, 8, 0, 0, 0])
    # dataspace message: version 1, rank 4, dims nComp, Nz, Ny, Nx
    dims = struct.pack("<4Q", ncomp, shape[2], shape[1], shape[0])
    j = b.index(dims)
    assert b[j - 8:j - 6] == bytes([1, 4])
    # the dataset is named "field" in the root group's local heap
    assert b"field\x00" in b[:j]


def test_reader_on_a_file_written_by_the_hdf5_library():
    """scipy's testhdf5_7.4_GLNX86.mat is an HDF5 file (libhdf5, via MATLAB) behind a
    512-byte user block: superblock 0 with base address 512, a symbol-table root group, a
    version-1 layout message.  Its one dataset, testdouble, holds 0, pi/4, ..., 2 pi with HDF5
    dims [9, 1]."""
    import scipy

    p = os.path.join(os.path.dirname(scipy.__file__), "io", "matlab", "tests", "data", "testhdf5_7.4_GLNX86.mat")
    if not os.path.exists(p):
        pytest.skip("scipy's HDF5 test file is not installed")
    v = _abi.h5_read_dataset(p, "testdouble")
    assert v.shape == (9, 1)
    assert np.array_equal(v[:, 0], np.arange(9) * (np.pi / 4))
    with pytest.raises(_abi.Gp5Error) as e:
        _abi.h5_field_shape(p)
    assert e.value.status == _abi.GP5_ERR_ARG
    assert b"members: testdouble" in _abi.lib().gp5cu_last_error()


def test_load_rejects_a_shape_mismatch_and_bad_files(tmp_path):
    p = str(tmp_path / "f.hdf5")
    _abi.h5_save_field(p, _field((4, 4, 4), 1, 1))
    out = np.empty((4, 4, 2, 1), dtype=np.complex128, order="F")
    rc = _abi.lib().gp5cu_h5_load_field(p.encode(), _abi.C.c_void_p(out.ctypes.data),
                                        (_abi.C.c_int * 3)(4, 4, 2), 1)
    assert rc == _abi.GP5_ERR_ARG
    bad = tmp_path / "bad.hdf5"
    bad.write_bytes(b"not an hdf5 file" * 40)
    with pytest.raises(_abi.Gp5Error) as e:
        _abi.h5_load_field(str(bad))
    assert e.value.status == _abi.GP5_ERR_IO
    with pytest.raises(_abi.Gp5Error) as e:
        _abi.h5_load_field(str(tmp_path / "missing.hdf5"))
    assert e.value.status == _abi.GP5_ERR_IO
    trunc = tmp_path / "trunc.hdf5"
    trunc.write_bytes(open(p, "rb").read()[:300])
    with pytest.raises(_abi.Gp5Error) as e:
        _abi.h5_load_field(str(trunc))
    assert e.value.status == _abi.GP5_ERR_IO
