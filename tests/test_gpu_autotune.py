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
