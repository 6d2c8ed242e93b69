"""Property-based CPU checks (hypothesis) of host logic and of the oracle's labelling."""
import math
import os
import sys

import numpy as np
from hypothesis import given, settings, strategies as st

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@settings(max_examples=40, deadline=None)
@given(st.integers(2, 9), st.integers(2, 9), st.integers(2, 9), st.integers(0, 2 ** 31 - 1),
       st.floats(0.1, 0.9))
def test_oracle_labels_are_periodic_26_components_in_scan_order(nx, ny, nz, seed, fill):
    rng = np.random.default_rng(seed)
    d = (rng.uniform(0, 1, (nx, ny, nz, 1)) < fill).astype(complex)
    lab, k = oracle.decompose(d, 0.5)
    L = lab[..., 0]
    fg = np.abs(d[..., 0]) ** 2 > 0.5
    assert np.array_equal(L == -1, ~fg) and (L[fg] >= 1).all() and (L[fg] <= k).all()
    # every pair of 26-neighbours above the cutoff carries one label (periodic wrap)
    for di in (-1, 0, 1):
        for dj in (-1, 0, 1):
            for dk in (-1, 0, 1):
                sh = np.roll(L, (di, dj, dk), axis=(0, 1, 2))
                both = fg & (sh > 0)
                assert np.array_equal(L[both], sh[both])
    # numbering: clusters appear in increasing order along the scan (i slowest, k fastest)
    seen = []
    for v in np.transpose(L, (0, 1, 2)).reshape(-1):  # C order of (i, j, k): k fastest
        if v > 0 and v not in seen:
            seen.append(v)
    assert seen == list(range(1, k + 1))


@settings(max_examples=25, deadline=None)
@given(st.floats(20.0, 2000.0), st.sampled_from([16, 24, 32]), st.integers(0, 2 ** 31 - 1))
def test_profile_start_is_normalised_symmetric_fortran(N, n, seed):
    from gp5_b200 import warmstart as ws
    r = ws.radii(N)
    rng = np.random.default_rng(seed)
    s = np.exp(-(r / (0.6 * N ** (1 / 3))) ** 2) * (1 + 0.05 * rng.uniform(-1, 1, r.size))
    psi = ws.profile_start(s, N, n)
    dx = ws.box_length(N) / n
    assert psi.dtype == np.complex128 and psi.flags["F_CONTIGUOUS"] and psi.shape == (n, n, n)
    assert abs(np.sum(np.abs(psi) ** 2) * dx ** 3 / N - 1) < 1e-12
    for ax in range(3):
        assert np.allclose(psi, np.flip(psi, axis=ax), rtol=0, atol=1e-14 * np.max(np.abs(psi)))
    assert np.all(psi.real >= 0) and np.all(psi.imag == 0)


@settings(max_examples=10, deadline=None)
@given(st.integers(1, 40), st.integers(0, 3))
def test_bench_grid_rule(count, rank):
    sys.path.insert(0, ROOT)
    import bench
    for sd in bench.batch_solves(count, rank=rank):
        assert sd["n"] in (32, 64, 128)
        assert sd["L"] / sd["n"] <= 0.25 or sd["n"] == 128
        smaller = [m for m in (32, 64, 128) if m < sd["n"]]
        assert all(sd["L"] / m > 0.25 for m in smaller)
        assert math.isclose(sd["dt"], 0.15 * (sd["L"] / sd["n"]) ** 2)
