"""The trained warm start (gp5_b200/data/warmstart_mlp.npz): tensor-core inference against the
FP64 oracle network, and the imaginary-time steps it saves over the Gaussian start."""
import numpy as np
import pytest

from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


def test_inference_matches_oracle_network():
    from gp5_b200 import warmstart as ws
    model = ws.WarmStart.load()
    params = ws.sample_params(64, ws.TEST_SEED)
    got = model.predict(params)
    w = np.load(ws.DEFAULT_WEIGHTS)["params"].astype(np.float64)
    ref, _ = mo.forward(w, ws.features(params), quantize=True)
    assert np.max(np.abs(got - ref)) <= 2e-3 * np.max(np.abs(ref))
    model.close()


def test_warm_start_saves_steps_with_same_ground_state():
    """Four unseen droplets (N > 200) on 64^3 grids: steps to a 1e-8 residual from the
    network's start against the Gaussian, converged energies within 1e-10."""
    from gp5_b200 import warmstart as ws
    model = ws.WarmStart.load()
    params = [p for p in ws.sample_params(64, ws.TEST_SEED) if p["N"] > 200][:4]
    pred = model.predict(params)
    _, rg = ws.solve_ground_states(params, 64, tol=1e-8, check_every=100,
                                   starts=lambda p, n, k: ws.gaussian_start(p["N"], n, None))
    _, rw = ws.solve_ground_states(params, 64, tol=1e-8, check_every=100,
                                   starts=lambda p, n, k: ws.profile_start(pred[k], p["N"], n, None))
    assert all(r["converged"] for r in rg + rw)
    sg = sum(r["steps"] for r in rg)
    sw = sum(r["steps"] for r in rw)
    assert sg >= 1.3 * sw, (sg, sw)
    for a, b in zip(rg, rw):
        assert abs(a["energy"] - b["energy"]) <= 1e-10 * abs(a["energy"])
    model.close()
