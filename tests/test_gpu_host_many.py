"""Pipelined host-state stepping (gp5cu_stepper_advance_host_many) against one state at a time."""
import numpy as np
import pytest

from oracle import gp_oracle as o

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec,imag", [(0, False), (1, False), (0, True)])
def test_host_many_matches_single_states(prec, imag):
    from gp5_b200 import _abi as abi
    geo = o.Geometry((32, 32, 32), (-6,) * 3, (6,) * 3)
    plan = abi.Plan(geo.shape, geo.left, geo.right, precision=prec)
    func = abi.Functional(plan, abi.GP5_FUNC_LHY, c3=-3.1)
    st = abi.Stepper(func, 1e-3, abi.GP5_STEP_RK4, imaginary=imag)
    if imag:
        st.set_renormalization([50.0])
    cdt = np.complex128 if prec == 0 else np.complex64
    states = [np.asfortranarray(o.gaussian_with_noise(geo, 1.5 + 0.1 * k, 1e-3, seed=k, N=50.0,
                                                      phase_noise=True).astype(cdt)) for k in range(5)]
    outs = [np.empty_like(s) for s in states]
    t0 = st.time
    st.advance_host_many(states, outs, 3)
    assert abs(st.time - (t0 + 3e-3)) < 1e-15
    for s, got in zip(states, outs):
        ref = np.empty_like(s)
        st.advance_host(s, ref, 3)
        assert np.array_equal(got, ref)
    # fewer states than device states
    two = [np.empty_like(s) for s in states[:2]]
    st.advance_host_many(states[:2], two, 3)
    assert all(np.array_equal(a, b) for a, b in zip(two, outs[:2]))
    # outputs may alias inputs
    same = [s.copy(order="F") for s in states[:3]]
    st.advance_host_many(same, same, 3)
    assert all(np.array_equal(a, b) for a, b in zip(same, outs[:3]))
