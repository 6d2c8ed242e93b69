"""Host-side logic of the warm start (no GPU): the chunked ground-state driver and the
periodic image-sum placement of radial samples."""
import math

import numpy as np

from gp5_b200 import warmstart as ws


class FakeBatch:
    """Stands in for _abi.Batch: solve i converges after need[i] steps in total."""
    need = {}
    created = []
    methods = []

    def __init__(self, descs, precision=0, device=0, devices=None):
        self.descs = descs
        self.states = [None] * len(descs)
        FakeBatch.created.append(len(descs))

    def set_state(self, k, psi):
        self.states[k] = np.array(psi, copy=True)

    def solve(self, tol, check_every, max_steps):
        out = []
        for k, d in enumerate(self.descs):
            key = d["N"]
            done = int(self.states[k].flat[0].real)
            left = FakeBatch.need[key] - done
            steps = min(max(left, 0), max_steps)
            steps = int(math.ceil(steps / check_every) * check_every) if steps < max_steps else max_steps
            self.states[k].flat[0] = done + steps
            conv = done + steps >= FakeBatch.need[key]
            out.append(dict(steps=steps, converged=int(conv), residual=0.0 if conv else 1.0,
                            energy=-key, mu=-1.0, norm=key))
        return out

    def set_method(self, method, theta=0.5):
        FakeBatch.methods.append((method, theta))

    def get_state(self, k):
        return self.states[k][..., None]

    def close(self):
        pass


def test_chunks_count_steps_and_keep_order(monkeypatch):
    """Each chunk goes to one batch (the batched solver takes finished solves out of its
    launches itself); results come back in the order of params."""
    params = [dict(N=float(20 + k), c3=-3.0, omega=0.0) for k in range(7)]
    FakeBatch.need = {p["N"]: s for p, s in zip(params, [300, 5000, 900, 45000, 100, 2500, 12000])}
    FakeBatch.created = []
    monkeypatch.setattr(ws._abi, "Batch", FakeBatch)
    starts = lambda p, n, i: np.zeros((4, 4, 4), complex)
    states, res = ws.solve_ground_states(params, 4, tol=1e-8, chunk=3, starts=starts, check_every=100,
                                         max_steps=100000, devices=[0, 1])
    assert [r["steps"] for r in res] == [300, 5000, 900, 45000, 100, 2500, 12000]
    assert all(r["converged"] for r in res)
    assert [r["energy"] for r in res] == [-p["N"] for p in params]
    assert FakeBatch.created == [3, 3, 1]


def test_preconditioned_method_reaches_every_chunk(monkeypatch):
    """method=GP5_BATCH_PRECOND is set on every chunk's batch with the step 0.5; the default
    leaves the batches on imaginary-time RK4."""
    params = [dict(N=float(30 + k), c3=-3.0, omega=0.0) for k in range(5)]
    FakeBatch.need = {p["N"]: 40 for p in params}
    FakeBatch.created, FakeBatch.methods = [], []
    monkeypatch.setattr(ws._abi, "Batch", FakeBatch)
    starts = lambda p, n, i: np.zeros((4, 4, 4), complex)
    _, res = ws.solve_ground_states(params, 4, tol=1e-8, chunk=2, starts=starts, check_every=5,
                                    method=ws._abi.GP5_BATCH_PRECOND)
    assert FakeBatch.methods == [(ws._abi.GP5_BATCH_PRECOND, 0.5)] * 3
    assert [r["steps"] for r in res] == [40] * 5
    FakeBatch.methods = []
    ws.solve_ground_states(params, 4, tol=1e-8, chunk=2, starts=starts)
    assert FakeBatch.methods == []


def test_unconverged_at_max_steps(monkeypatch):
    params = [dict(N=21.0, c3=-3.0, omega=0.0), dict(N=22.0, c3=-3.0, omega=0.0)]
    FakeBatch.need = {21.0: 700, 22.0: 10 ** 9}
    FakeBatch.created = []
    monkeypatch.setattr(ws._abi, "Batch", FakeBatch)
    starts = lambda p, n, i: np.zeros((4, 4, 4), complex)
    _, res = ws.solve_ground_states(params, 4, tol=1e-8, starts=starts, max_steps=4000)
    assert res[0]["steps"] == 700 and res[0]["converged"]
    assert res[1]["steps"] == 4000 and not res[1]["converged"]


def _periodic_droplet(N, n, kappa=0.7):
    """sum over images of a smooth core with a screened-Coulomb tail (the shape of a small
    droplet's ground state in the periodic box)."""
    L = ws.box_length(N)
    x = ws.axis(n, L)
    R = ws.radii(N)[-1]
    rc = 0.4 * R

    def f(d):
        core = np.exp(-(d / rc) ** 2)
        tail = 0.02 * np.exp(-kappa * d) / np.maximum(d, 0.5) * (1 - np.exp(-(d / rc) ** 4))
        return core + tail

    out = np.zeros((n, n, n))
    for a in (-1, 0, 1):
        for b in (-1, 0, 1):
            for c in (-1, 0, 1):
                d = np.sqrt((x[:, None, None] - a * L) ** 2 + (x[None, :, None] - b * L) ** 2
                            + (x[None, None, :] - c * L) ** 2)
                out += f(d)
    return out * math.sqrt(N / (np.sum(out ** 2) * (L / n) ** 3))


def test_image_sum_placement_reproduces_periodic_droplet():
    N, n = 40.0, 48
    psi = _periodic_droplet(N, n)
    S = ws.radial_samples(psi, N)
    got = ws.profile_start(S, N, n)
    err = np.max(np.abs(got - psi)) / np.max(psi)
    # a purely radial placement misses the image-induced corner tails
    r = ws.radii(N)
    L = ws.box_length(N)
    x = ws.axis(n, L)
    Rg = np.sqrt(x[:, None, None] ** 2 + x[None, :, None] ** 2 + x[None, None, :] ** 2)
    radial = np.interp(np.minimum(Rg, r[-1]), r, S)
    radial = radial * math.sqrt(N / (np.sum(radial ** 2) * (L / n) ** 3))
    err_radial = np.max(np.abs(radial - psi)) / np.max(psi)
    assert err < 2e-3 and err < 0.2 * err_radial, (err, err_radial)
    assert got.flags["F_CONTIGUOUS"] and got.dtype == np.complex128
    assert abs(np.sum(np.abs(got) ** 2) * (L / n) ** 3 - N) < 1e-9 * N


def test_free_profile_recovers_the_isolated_profile():
    """Axis samples of a periodic image sum of a known isolated profile (smooth core, screened-
    Coulomb tail) deconvolve back to that profile and its tail rate."""
    N, kappa = 60.0, 0.7
    r = ws.radii(N)
    R, L = r[-1], ws.box_length(N)
    rc = 0.25 * R  # the tail dominates the last samples, as for a droplet

    def f(d):
        d = np.asarray(d, float)
        core = np.exp(-(d / rc) ** 2)
        tail = 0.03 * np.exp(-kappa * d) / np.maximum(d, 1e-12)
        w = 1 - np.exp(-(d / rc) ** 6)
        return core + w * tail

    # the isolated profile seen through the front end's tail model beyond R
    samples_iso = f(r)
    axis = np.zeros_like(r)
    for m in ws._AXIS_IMAGES:
        d = np.sqrt((r - m[0] * L) ** 2 + (m[1] * L) ** 2 + (m[2] * L) ** 2)
        axis += np.where(d <= R, f(np.minimum(d, R)),
                         f(R) * (R / np.maximum(d, R)) * np.exp(-kappa * (np.maximum(d, R) - R)))
    got, k = ws.free_profile(axis, N)
    assert 0.5 * kappa < k < 1.5 * kappa  # log-slope estimate (the core still leaks into it)
    assert np.max(np.abs(got - samples_iso)) < 1e-5 * np.max(samples_iso)


def test_lsq_samples_recover_an_image_sum_placement():
    """A field that is itself a profile_start placement is fitted: the least-squares samples
    place back onto the same field (32^3, a flat-topped droplet-like profile; the round trip
    re-estimates the tail rate, hence not to rounding)."""
    N, n = 60.0, 32
    r = ws.radii(N)
    R0 = 0.6 * N ** (1.0 / 3.0)
    s0 = 0.9 / (1.0 + np.exp((r - R0) / 0.5))  # flat top with a smooth edge
    psi = ws.profile_start(s0, N, n)
    s1 = ws.lsq_samples(psi, N)
    back = ws.profile_start(s1, N, n)
    assert np.max(np.abs(back - psi)) <= 1e-4 * np.max(np.abs(psi))


def test_lsq_samples_fit_better_than_the_axis_samples():
    """For a field that is not an image sum (a Gaussian product), the least-squares samples
    place closer to it than its own axis samples do."""
    N, n = 60.0, 32
    psi = ws.gaussian_start(N, n, None)
    err = lambda s: float(np.sqrt(np.mean(np.abs(ws.profile_start(s, N, n) - psi) ** 2)))
    assert err(ws.lsq_samples(psi, N)) <= err(ws.radial_samples(psi, N))
