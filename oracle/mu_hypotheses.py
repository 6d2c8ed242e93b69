"""The reference's mu regression protocol under alternative readings (test infrastructure).

python/test/regressionTests/LHY_imaginary.py:8-49 converges mu = 0.5 ln(N/||psi||^2)/dt over
1000-step blocks of imaginary-time RK4 (normalising before every step) until two blocks agree
to 1e-9; its committed result is python/test/regressionTests/mu:1 = -0.3837299937094331.  The
oracle's faithful restatement (gp_oracle.lhy_mu_protocol) lands 6.4e-5 from it.  This script
runs the protocol under each alternative that could move the result and prints one JSON line
per variant:

  restated      the script as committed (30^3, box [-10,10]^3, sigma 5, N 370, dt 0.01 dx^2)
  dt=...        other time steps (the estimator carries an O(dt) bias)
  N=371         another atom number
  grid=32       a 32^3 grid on the same box
  euler         the Euler stepper instead of RK4
  spb=100       100-step blocks (the stepsPerBlock of python/test/test.py:172)
  spacing29     the spacing L/(n - 1) (box widened to +-10*30/29)
  exact         the discrete ground state's mu = <psi|H psi>/N (preconditioned iteration to
                residual 1e-12): the dt -> 0 limit of the protocol
  permuted      the data with its axes permuted (y, z, x): the P3DFFT path with
                fftOrdering [2,0,1] (gp.py:35-38) only permutes the k-space axes, and on this
                cubic grid and box it must reproduce 'restated' to rounding

Usage: python -m oracle.mu_hypotheses [variant ...]   (all variants when none is given;
each takes 1-3 minutes of CPU).
"""
from __future__ import annotations

import json
import math
import sys

import numpy as np

from oracle import gp_oracle as o

GOLDEN = -0.3837299937094331  # python/test/regressionTests/mu:1


def _protocol_euler():
    geo = o.Geometry((30,) * 3, (-10.0,) * 3, (10.0,) * 3)
    psi = o.new_field(geo)
    o.init_gaussian(geo, 5.0, psi)
    o.normalize(370.0, psi, 0, geo)
    st = o.Stepper(o.Functional("lhy"), geo, 0.01 * geo.space_step(0) ** 2, "eulero", True)
    old, mu, it = 0.0, 1e18, 0
    while abs(mu - old) > 1e-9 and it < 200:
        it += 1
        for _ in range(1000):
            o.normalize(370.0, psi, 0, geo)
            psi = st.advance(psi, 1)
        old = mu
        mu = o.mu_from_norm_decay(370.0, o.norm(psi, 0, geo), st.dt)
        o.normalize(370.0, psi, 0, geo)
    return mu, it


def _protocol_permuted():
    """The restated protocol with the field stored as (y, z, x): every FFT, K^2 and norm then
    runs over permuted axes, as the P3DFFT path's permuted k-space ordering would."""
    geo = o.Geometry((30,) * 3, (-10.0,) * 3, (10.0,) * 3)
    psi = o.new_field(geo)
    o.init_gaussian(geo, 5.0, psi)
    psi = np.asfortranarray(np.transpose(psi, (1, 2, 0, 3)))
    o.normalize(370.0, psi, 0, geo)
    st = o.Stepper(o.Functional("lhy"), geo, 0.01 * geo.space_step(0) ** 2, "RK4", True)
    old, mu, it = 0.0, 1e18, 0
    while abs(mu - old) > 1e-9 and it < 1000:
        it += 1
        for _ in range(1000):
            o.normalize(370.0, psi, 0, geo)
            psi = st.advance(psi, 1)
        old = mu
        mu = o.mu_from_norm_decay(370.0, o.norm(psi, 0, geo), st.dt)
        o.normalize(370.0, psi, 0, geo)
    return mu, it


def run(name: str):
    dx = 20.0 / 30
    if name == "restated":
        mu, it, _ = o.lhy_mu_protocol()
    elif name.startswith("dt="):
        mu, it, _ = o.lhy_mu_protocol(dt_factor=float(name[3:]) / dx ** 2)
    elif name.startswith("N="):
        mu, it, _ = o.lhy_mu_protocol(N=float(name[2:]))
    elif name.startswith("grid="):
        n = int(name[5:])
        mu, it, _ = o.lhy_mu_protocol(shape=(n,) * 3)
    elif name.startswith("spb="):
        mu, it, _ = o.lhy_mu_protocol(steps_per_block=int(name[4:]))
    elif name == "spacing29":
        # the spacing L/(n - 1) of a vertex-based grid: the box widened to +-10*30/29
        mu, it, _ = o.lhy_mu_protocol(box=10.0 * 30 / 29)
    elif name == "exact":
        # the discrete ground state itself (no time step): mu = <psi|H psi>/N at residual 1e-12
        geo = o.Geometry((30,) * 3, (-10.0,) * 3, (10.0,) * 3)
        psi = o.new_field(geo)
        o.init_gaussian(geo, 5.0, psi)
        o.normalize(370.0, psi, 0, geo)
        _, it, ob = o.precond_ground_state(o.Functional("lhy"), geo, psi, 370.0, tol=1e-12, max_iter=5000)
        mu = ob["mu"]
    elif name == "euler":
        mu, it = _protocol_euler()
    elif name == "permuted":
        mu, it = _protocol_permuted()
    else:
        raise SystemExit(f"unknown variant {name}")
    return {"variant": name, "mu": mu, "blocks": it, "minus_golden": mu - GOLDEN}


VARIANTS = ["restated", "dt=0.001", "dt=0.002", "dt=0.004", f"dt={0.02 * (20.0 / 30) ** 2!r}", "N=371", "grid=32",
            "euler", "spb=100", "permuted", "spacing29", f"dt={0.01 * (20.0 / 29) ** 2!r}", "exact"]

if __name__ == "__main__":
    for v in sys.argv[1:] or VARIANTS:
        print(json.dumps(run(v)), flush=True)
    sys.exit(0 if math.isfinite(GOLDEN) else 1)
