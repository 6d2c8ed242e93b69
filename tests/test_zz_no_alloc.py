"""The allocation-free norm, gp5cu_norm_noalloc, against the plan-based gp5cu_norm and the oracle.

gp5cu_norm_noalloc serves callers that cannot allocate device memory when they need a norm
(their fields live in another allocator's memory, or the device is full): it keeps its
partial sums in a static device array instead of a plan's buffers.  This file is collected
last so that a run stopping at the first failure has already run every other test; it
passes alone in a fresh process and after the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import gp_oracle as o

pytestmark = pytest.mark.gpu


def _dV(plan):
    dV = 1.0
    for d in range(3):
        dV *= (plan.right[d] - plan.left[d]) / plan.shape[d]
    return dV


def _noalloc_norm(abi, ptr, precision, shape, ncomp, comp, dV):
    out = C.c_double()
    abi.check(abi.lib().gp5cu_norm_noalloc(C.c_void_p(ptr), precision, (C.c_int * 3)(*shape), ncomp, comp, dV,
                                           None, C.byref(out)))
    return out.value


@pytest.mark.parametrize("prec,shape,ncomp", [(0, (64, 48, 40), 1), (1, (32, 30, 28), 2), (0, (7, 5, 3), 2),
                                              (0, (256, 256, 256), 1)])
def test_norm_noalloc_matches_plan_norm_and_oracle_twice(prec, shape, ncomp):
    from gp5_b200 import _abi as abi

    geo = o.Geometry(shape, (-6,) * 3, (6,) * 3)
    rng = np.random.default_rng(31)
    psi = np.asfortranarray(rng.uniform(-1, 1, shape + (ncomp,)) + 1j * rng.uniform(-1, 1, shape + (ncomp,)))
    plan = abi.Plan(geo.shape, geo.left, geo.right, ncomp=ncomp, precision=prec)
    f = plan.field(psi)
    stored = f.download()  # the values as the device holds them (complex64 rounding included)
    tol = 1e-13 if prec == 0 else 1e-12  # both sum the stored values in FP64
    for comp in range(ncomp):
        ref = plan.norm(f, comp)
        oracle = o.norm(stored, comp, geo)
        first = _noalloc_norm(abi, f.ptr.value, prec, shape, ncomp, comp, _dV(plan))
        second = _noalloc_norm(abi, f.ptr.value, prec, shape, ncomp, comp, _dV(plan))  # shared scratch reused
        assert abs(first - ref) <= tol * abs(ref)
        assert abs(first - oracle) <= tol * abs(oracle)
        assert first == second


def test_norm_noalloc_allocates_nothing():
    """Free device memory is the same before and after a first call on a shape not seen before."""
    import torch

    from gp5_b200 import _abi as abi

    geo = o.Geometry((40, 36, 33), (-3,) * 3, (3,) * 3)
    plan = abi.Plan(geo.shape, geo.left, geo.right)
    psi = np.asfortranarray(np.random.default_rng(5).uniform(-1, 1, geo.shape + (1,)) + 0j)
    f = plan.field(psi)
    # a first call on another shape loads the module (its static array included)
    warm = abi.Plan((8, 8, 8), (-1,) * 3, (1,) * 3)
    wf = warm.field(np.ones((8, 8, 8, 1), dtype=np.complex128))
    _noalloc_norm(abi, wf.ptr.value, 0, (8, 8, 8), 1, 0, 1.0)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    got = _noalloc_norm(abi, f.ptr.value, 0, geo.shape, 1, 0, geo.dV)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert abs(got - o.norm(psi, 0, geo)) <= 1e-13 * abs(got)


def test_norm_noalloc_complex64_view_on_an_8_byte_boundary():
    """Component 1 of a complex64 field with an odd site count starts 8 bytes past a 16-byte
    boundary; the call takes it as a one-component field."""
    from gp5_b200 import _abi as abi

    shape = (7, 5, 3)  # 105 sites
    geo = o.Geometry(shape, (-2,) * 3, (2,) * 3)
    rng = np.random.default_rng(9)
    psi = np.asfortranarray(rng.uniform(-1, 1, shape + (2,)) + 1j * rng.uniform(-1, 1, shape + (2,)))
    plan = abi.Plan(shape, geo.left, geo.right, ncomp=2, precision=abi.GP5_C64)
    f = plan.field(psi)
    ptr1 = f.ptr.value + 105 * 8
    assert ptr1 % 16 == 8
    got = _noalloc_norm(abi, ptr1, abi.GP5_C64, shape, 1, 0, geo.dV)
    assert abs(got - plan.norm(f, 1)) <= 1e-12 * abs(got)
    assert abs(got - o.norm(f.download(), 1, geo)) <= 1e-12 * abs(got)


def test_norm_noalloc_rejects_fields_beyond_the_limit():
    from gp5_b200 import _abi as abi

    plan = abi.Plan((8, 8, 8), (-1,) * 3, (1,) * 3)
    f = plan.field()
    out = C.c_double()
    for shape in ((512, 256, 256), (1 << 21, 1 << 21, 1 << 21), (2**31 - 1, 2**31 - 1, 2**31 - 1)):
        rc = abi.lib().gp5cu_norm_noalloc(f.ptr, 0, (C.c_int * 3)(*shape), 1, 0, 1.0, None, C.byref(out))
        assert rc == abi.GP5_ERR_ARG
        assert b"static scratch limit" in abi.lib().gp5cu_last_error()
    # a complex128 field must be 16-byte aligned
    rc = abi.lib().gp5cu_norm_noalloc(C.c_void_p(f.ptr.value + 8), 0, (C.c_int * 3)(4, 4, 4), 1, 0, 1.0, None,
                                      C.byref(out))
    assert rc == abi.GP5_ERR_ARG
