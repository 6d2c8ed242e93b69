"""The allocation-free norm, gp5cu_norm_noalloc, against the plan-based gp5cu_norm.

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


def _noalloc_norm(abi, plan, field, comp=0):
    out = C.c_double()
    shape = (C.c_int * 3)(*plan.shape)
    dV = 1.0
    for d in range(3):
        dV *= (plan.right[d] - plan.left[d]) / plan.shape[d]
    abi.check(abi.lib().gp5cu_norm_noalloc(field.ptr, plan.precision, shape, plan.ncomp, comp, dV, None,
                                           C.byref(out)))
    return out.value


@pytest.mark.parametrize("prec,shape,ncomp", [(0, (64, 48, 40), 1), (1, (32, 30, 28), 2), (0, (256, 256, 256), 1)])
def test_norm_noalloc_matches_plan_norm_twice(prec, shape, ncomp):
    from gp5_b200 import _abi as abi

    geo = o.Geometry(shape, (-6,) * 3, (6,) * 3)
    rng = np.random.default_rng(31)
    psi = np.asfortranarray(rng.uniform(-1, 1, shape + (ncomp,)) + 1j * rng.uniform(-1, 1, shape + (ncomp,)))
    plan = abi.Plan(geo.shape, geo.left, geo.right, ncomp=ncomp, precision=prec)
    f = plan.field(psi)
    tol = 1e-13 if prec == 0 else 1e-12  # both sum the stored values in FP64
    for comp in range(ncomp):
        ref = plan.norm(f, comp)
        first = _noalloc_norm(abi, plan, f, comp)
        second = _noalloc_norm(abi, plan, f, comp)  # the shared scratch keeps the last call
        assert abs(first - ref) <= tol * abs(ref)
        assert abs(second - ref) <= tol * abs(ref)
        assert first == second


def test_norm_noalloc_rejects_fields_beyond_the_limit():
    from gp5_b200 import _abi as abi

    plan = abi.Plan((8, 8, 8), (-1,) * 3, (1,) * 3)
    f = plan.field()
    out = C.c_double()
    too_big = (C.c_int * 3)(512, 256, 256)
    rc = abi.lib().gp5cu_norm_noalloc(f.ptr, 0, too_big, 1, 0, 1.0, None, C.byref(out))
    assert rc == abi.GP5_ERR_ARG
    assert b"static scratch limit" in abi.lib().gp5cu_last_error()
