"""The tile-shape autotuner (gp5cu_plan_autotune / get_tiles / set_tiles): every shape of the
strided y/z passes gives bit-identical results, and the tuner's choice is one of them."""
import itertools

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _field(shape, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(shape + (1,)) + 1j * rng.standard_normal(shape + (1,))
    return np.asfortranarray(a)


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("shape", [(64, 32, 128), (256, 64, 64), (32, 512, 32)])
def test_every_tile_shape_gives_identical_transforms(prec, shape):
    from gp5_b200 import _abi
    p = _abi.Plan(shape, (-4.0,) * 3, (4.0,) * 3, precision=prec)
    chosen = p.tiles()
    assert all(t in (0, 128, 256, 512) for t in chosen)
    src = p.field(_field(shape, 1))
    dst = p.field()
    ref = None
    for th in (0, 128, 256, 512):
        try:
            p.set_tiles([th] * 5)
        except _abi.Gp5Error:
            continue  # the axis's lines do not split into this many threads
        p.fft(src, dst, _abi.GP5_FORWARD)
        fwd = dst.download()
        p.laplacian(src, dst)
        lap = dst.download()
        if ref is None:
            ref = (fwd, lap)
        else:
            assert np.array_equal(fwd, ref[0]) and np.array_equal(lap, ref[1]), th


def test_tuned_stepper_matches_default_bitwise():
    from gp5_b200 import _abi
    shape = (64, 64, 64)
    psi0 = _field(shape, 2) * 1e-2
    out = []
    for tiles in ([0] * 5, [512, 512, 512, 512, 256], None):
        p = _abi.Plan(shape, (-6.0,) * 3, (6.0,) * 3)
        if tiles is None:
            p.autotune()
        else:
            p.set_tiles(tiles)
        f = _abi.Functional(p, _abi.GP5_FUNC_LHY)
        st = _abi.Stepper(f, 1e-3, imaginary=False)
        a = p.field(psi0)
        st.advance(a, 5)
        out.append(a.download())
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[0], out[2])


def test_set_tiles_rejects_bad_shapes():
    from gp5_b200 import _abi
    p = _abi.Plan((30, 50, 64), (-1.0,) * 3, (1.0,) * 3)
    with pytest.raises(_abi.Gp5Error):
        p.set_tiles([100, 0, 0, 0, 0])
    with pytest.raises(_abi.Gp5Error):
        p.set_tiles([256, 0, 0, 0, 0])  # y = 50 uses the shared-memory engine
    p.set_tiles([0, 0, 256, 256, 256])
    assert p.tiles() == [0, 0, 256, 256, 256]


def test_tuning_cache_file_is_written_and_reused(tmp_path):
    import json
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    path = tmp_path / "tune.json"
    code = ("import sys; sys.path.insert(0, %r); from gp5_b200 import _abi; "
            "p = _abi.Plan((64, 64, 64), (-1.0,) * 3, (1.0,) * 3); print(p.tiles())" % root)
    env = dict(os.environ, GP5_AUTOTUNE_CACHE=str(path))
    r1 = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert r1.returncode == 0, r1.stderr
    d = json.loads(path.read_text())
    keys = [k for k in d if "|64x64x64|c1|c128|s1|" in k]
    assert len(keys) == 1 and d[keys[0]] == eval(r1.stdout.strip().splitlines()[-1])
    d[keys[0]] = [512, 256, 512, 256, 256]
    path.write_text(json.dumps(d))
    r2 = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert r2.returncode == 0, r2.stderr
    assert eval(r2.stdout.strip().splitlines()[-1]) == [512, 256, 512, 256, 256]


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("shape", [(64, 32, 128), (256, 64, 64), (32, 512, 32), (128, 128, 256)])
def test_both_radix_schedules_match_the_oracle(prec, shape):
    """Schedules 0 and 1 (other radices, other elements per thread) each give the unnormalised
    DFT and the spectral Laplacian to rounding: 1e-13 (complex128) / 2e-6 (complex64) of the
    long-double-checked numpy transform and of the oracle."""
    from gp5_b200 import _abi
    from oracle import gp_oracle as o
    geo = o.Geometry(shape, (-4.0,) * 3, (4.0,) * 3)
    psi = _field(shape, 3)
    ref_fwd = np.fft.fftn(psi, axes=(0, 1, 2))
    ref_lap = o.laplacian(psi, geo)
    tol = 1e-13 if prec == 0 else 2e-6
    for s in (0, 1):
        p = _abi.Plan(shape, geo.left, geo.right, precision=prec)
        p.set_radix([s] * 6)
        assert p.radix() == [s] * 6
        src, dst = p.field(psi), p.field()
        p.fft(src, dst, _abi.GP5_FORWARD)
        got = dst.download()
        assert np.max(np.abs(got - ref_fwd)) <= tol * np.max(np.abs(ref_fwd)), s
        p.laplacian(src, dst)
        got = dst.download()
        assert np.max(np.abs(got - ref_lap)) <= tol * np.max(np.abs(ref_lap)), s


@pytest.mark.parametrize("n", [32, 64, 128, 256])
def test_radix_one_stage_boundary_rk4_step_matches_the_oracle(n):
    """One renormalised imaginary-time RK4 step and one real-time step with every pass, the
    stage boundary included, on schedule 1, against the oracle at 1e-12."""
    from gp5_b200 import _abi
    from oracle import gp_oracle as o
    L = 4 * 100.0 ** (1 / 3)
    geo = o.Geometry((n, n, n), (-L / 2,) * 3, (L / 2,) * 3)
    psi = o.gaussian_with_noise(geo, 0.5 * 100.0 ** (1 / 3), 1e-3, seed=n, N=100.0, phase_noise=True)
    for imag in (True, False):
        p = _abi.Plan(geo.shape, geo.left, geo.right)
        p.set_radix([1] * 6)
        f = _abi.Functional(p, _abi.GP5_FUNC_LHY, c3=-3.1)
        st = _abi.Stepper(f, 0.15 * (L / n) ** 2 if imag else 1e-3, imaginary=imag)
        ost = o.Stepper(o.Functional("lhy", c3=-3.1), geo, st.dt, "RK4", imag)
        if imag:
            st.set_renormalization([100.0])
            ost.normalizations = [100.0]
        a = p.field(psi)
        st.advance(a, 1)
        ref = ost.advance(psi.copy(), 1)
        got = a.download()
        assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref)), imag


def test_plans_of_one_grid_share_their_radix_schedules():
    """The schedules are chosen once per grid and precision: a forced re-tune and a later plan
    keep them (so batched and single solves round alike)."""
    from gp5_b200 import _abi
    a = _abi.Plan((64, 64, 32), (-1.0,) * 3, (1.0,) * 3)
    r = a.radix()
    a.autotune()
    b = _abi.Plan((64, 64, 32), (-2.0,) * 3, (2.0,) * 3)
    assert a.radix() == r and b.radix() == r
    with pytest.raises(_abi.Gp5Error):
        a.set_radix([2, 0, 0, 0, 0, 0])
