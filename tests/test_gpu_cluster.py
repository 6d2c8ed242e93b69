"""Droplet decomposition on the GPU (gp5cu_decompose) against the oracle's restatement of
gp::decompose::decompose (src/cluster.cpp:17-83): labels must be identical."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _smooth_blobs(shape, seed, ncomp=1):
    """thresholdable random field: a few periodic Gaussian blobs (some across the boundary)"""
    rng = np.random.default_rng(seed)
    grids = np.meshgrid(*[np.arange(n) for n in shape], indexing="ij")
    out = np.zeros(shape + (ncomp,), complex)
    for c in range(ncomp):
        for _ in range(7):
            ctr = rng.uniform(0, 1, 3) * np.array(shape)
            w = rng.uniform(1.5, 4.0)
            r2 = 0
            for g, n, x0 in zip(grids, shape, ctr):
                dx = np.abs(g - x0)
                dx = np.minimum(dx, n - dx)
                r2 = r2 + dx * dx
            out[..., c] += np.exp(-r2 / (2 * w * w)) * np.exp(1j * rng.uniform(0, 6.28))
    return np.asfortranarray(out)


@pytest.mark.parametrize("prec", [0, 1])
def test_squares_reference_case(prec):
    from gp5_b200 import _abi
    p = _abi.Plan((100, 100, 100), (-1.0,) * 3, (1.0,) * 3, precision=prec)
    data = np.zeros((100, 100, 100, 1), complex, order="F")
    data[10:51, 10:51, 10:51, 0] = 1
    lab, k = p.decompose(p.field(data), 0.5)
    ref, kr = oracle.decompose(data, 0.5)
    assert k == kr == 1 and np.array_equal(lab, ref)
    data[:] = 0
    data[10:21, 10:21, 10:21] = 1
    data[50:61, 10:21, 10:21] = 1
    lab, k = p.decompose(p.field(data), 0.5)
    ref, kr = oracle.decompose(data, 0.5)
    assert k == kr == 2 and np.array_equal(lab, ref)


@pytest.mark.parametrize("shape,ncomp,comp,prec", [((64, 64, 64), 1, 0, 0), ((48, 40, 36), 2, 1, 0),
                                                    ((64, 32, 128), 1, 0, 1), ((2, 3, 4), 1, 0, 0),
                                                    ((30, 50, 7), 2, 0, 1)])
def test_random_blobs_match_oracle(shape, ncomp, comp, prec):
    from gp5_b200 import _abi
    p = _abi.Plan(shape, (-1.0,) * 3, (1.0,) * 3, ncomp=ncomp, precision=prec)
    psi = _smooth_blobs(shape, sum(shape) + comp, ncomp)
    if prec == 1:
        psi = psi.astype(np.complex64).astype(np.complex128)  # the values the plan holds
    f = p.field(psi)
    for cut in (0.05, 0.3, 0.8):
        lab, k = p.decompose(f, cut, comp)
        ref, kr = oracle.decompose(psi, cut, comp)
        assert k == kr and np.array_equal(lab, ref), (cut, k, kr)


def test_empty_full_and_diagonal_cases():
    from gp5_b200 import _abi
    shape = (12, 10, 8)
    p = _abi.Plan(shape, (-1.0,) * 3, (1.0,) * 3, ncomp=2)
    d = np.zeros(shape + (2,), complex, order="F")
    lab, k = p.decompose(p.field(d), 0.1)
    assert k == 0 and (lab[..., 0] == -1).all() and (lab[..., 1] == 0).all()
    lab, k = p.decompose(p.field(np.ones_like(d)), 0.1)
    assert k == 1 and (lab[..., 0] == 1).all()
    d[0, 3, 3, 0] = d[11, 3, 3, 0] = 1
    d[5, 5, 5, 0] = d[6, 6, 6, 0] = 1
    d[2, 0, 0, 0] = 1
    d[8, 9, 7, 0] = 0.5 + 0.5j
    lab, k = p.decompose(p.field(d), 0.5)
    ref, kr = oracle.decompose(d, 0.5)
    assert k == kr == 3 and np.array_equal(lab, ref)


def test_gpcpp_decomposition_class():
    from gp5_b200 import gpCpp
    geo = gpCpp.geometry([-1.0] * 3, [1.0] * 3, [40, 40, 40])
    f = gpCpp.field(geo, 1, [1, 1, 1], [2, 0, 1])
    psi = _smooth_blobs((40, 40, 40), 3)
    f.setTensor(psi)
    lab = gpCpp.decomposition().decompose(f, 0.2)
    ref, _ = oracle.decompose(psi, 0.2)
    assert lab.dtype == np.int32 and lab.shape == (40, 40, 40, 1) and np.array_equal(lab, ref)
