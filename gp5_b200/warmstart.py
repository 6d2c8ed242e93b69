"""Learned warm start for LHY droplet ground states.

A small MLP (gp5cu_mlp_*: 3 -> 256 -> 256 -> 256 -> 64, GELU, BF16 tensor-core GEMMs with
FP32 accumulation) maps a solve's parameters (log N, cubic coefficient c3, trap frequency
omega) to 64 radial samples of the ground state psi(r) on [0, 2 N^(1/3)].  The samples are
interpolated onto the solve's grid, normalised to N, and imaginary time refines the result to
the requested residual exactly as it would refine a Gaussian.  The Gaussian of width
0.5 N^(1/3) (the start of python/test/regressionTests/LHY_imaginary.py:14) stays the
fallback.

The network is trained on ground states that the batched solver (gp5cu_batch_*) produces.
No reference counterpart: the reference has no learned component.
"""
from __future__ import annotations

import math
import os
from typing import Iterable, List, Optional, Sequence

import numpy as np

from . import _abi

N_SAMPLES = 64
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "warmstart_mlp.npz")
OMEGAS = (0.0, 0.05, 0.1)
C4 = 2.5


# ---- solve parameters ------------------------------------------------------------------------
def sample_params(count: int, seed: int, omegas: Sequence[float] = OMEGAS) -> List[dict]:
    """Seeded droplet parameters: N log-uniform in [20, 2000], c3 ~ U[-3.2, -2.8], omega drawn
    from `omegas`, c4 = 2.5."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        N = float(np.exp(rng.uniform(math.log(20.0), math.log(2000.0))))
        c3 = float(rng.uniform(-3.2, -2.8))
        om = float(omegas[int(rng.integers(len(omegas)))])
        out.append(dict(N=N, c3=c3, omega=om))
    return out


def box_length(N: float) -> float:
    """L = 4 N^(1/3): the box is [-L/2, L/2]^3."""
    return 4.0 * N ** (1.0 / 3.0)


def smallest_grid(N: float, grids: Sequence[int] = (32, 64, 128), max_dx: float = 0.25) -> int:
    """The smallest grid with L/n <= max_dx, else the largest."""
    L = box_length(N)
    return next((m for m in grids if L / m <= max_dx), grids[-1])


def solve_desc(p: dict, n: int, dt_factor: float = 0.15) -> dict:
    """Batch solve descriptor on an n^3 grid.  dt = 0.15 dx^2: imaginary-time RK4 is stable on
    the cube-corner modes K^2 = 3 (pi/dx)^2 up to dt ~ 0.188 dx^2."""
    L = box_length(p["N"])
    dx = L / n
    return dict(n=n, L=L, N=p["N"], c3=p["c3"], c4=p.get("c4", C4), omega=p.get("omega", 0.0),
                dt=dt_factor * dx * dx)


# ---- states ----------------------------------------------------------------------------------
def axis(n: int, L: float) -> np.ndarray:
    """Cell-centred positions of [-L/2, L/2] (geometry.cpp's grid convention)."""
    return -L / 2 + L / n * (np.arange(n) + 0.5)


def _normalise(psi: np.ndarray, N: float, dx: float) -> np.ndarray:
    return psi * math.sqrt(N / (float(np.sum(np.abs(psi) ** 2)) * dx ** 3))


def _phase_noise(psi: np.ndarray, seed: Optional[int], amp: float) -> np.ndarray:
    if seed is None or amp == 0.0:
        return psi
    return psi * np.exp(1j * amp * np.random.default_rng(seed).uniform(-1, 1, psi.shape))


def gaussian_start(N: float, n: int, seed: Optional[int] = None, amp: float = 1e-3) -> np.ndarray:
    """Gaussian of width 0.5 N^(1/3) with seeded phase noise of amplitude amp, normalised to N;
    complex128 (n, n, n), Fortran order (x fastest)."""
    L = box_length(N)
    x = axis(n, L)
    sig = 0.5 * N ** (1.0 / 3.0)
    g = np.exp(-x * x / (2 * sig * sig))
    psi = (g[:, None, None] * g[None, :, None] * g[None, None, :]).astype(np.complex128)
    psi = _phase_noise(psi, seed, amp)
    return np.asfortranarray(_normalise(psi, N, L / n))


def radii(N: float) -> np.ndarray:
    """The 64 sample radii r_j = j * 2 N^(1/3) / 63."""
    return np.linspace(0.0, 2.0 * N ** (1.0 / 3.0), N_SAMPLES)


def radial_samples(psi: np.ndarray, N: float) -> np.ndarray:
    """|psi| at the sample radii along the six half-axes through the box centre, averaged.

    psi: (n, n, n) or (n, n, n, 1) on the cell-centred grid of [-L/2, L/2]^3.  The centre is
    not a grid point, so the values are the field's Fourier interpolant (exact for a
    band-limited field)."""
    a = np.asarray(psi)
    if a.ndim == 4:
        a = a[..., 0]
    n = a.shape[0]
    L = box_length(N)
    dx = L / n
    x0 = -L / 2 + dx / 2
    P = np.fft.fftn(a)
    k = 2 * np.pi * np.fft.fftfreq(n, dx)
    e0 = np.exp(-1j * k * x0)  # other axes evaluated at 0
    r = radii(N)
    acc = np.zeros(N_SAMPLES)
    lines = (np.einsum("ijk,j,k->i", P, e0, e0), np.einsum("ijk,i,k->j", P, e0, e0),
             np.einsum("ijk,i,j->k", P, e0, e0))
    for c in lines:
        for sgn in (1.0, -1.0):
            ph = np.exp(1j * np.outer(sgn * r - x0, k))
            acc += np.abs(ph @ c) / n ** 3
    return acc / 6.0


_BASIS = None


def _basis():
    """Cubic-spline basis on the normalised sample radii u_j = j/63 (zero slope at u = 0,
    not-a-knot at u = 1): f(u) = B(u) @ samples."""
    global _BASIS
    if _BASIS is None:
        from scipy.interpolate import CubicSpline

        u = np.linspace(0.0, 1.0, N_SAMPLES)
        _BASIS = CubicSpline(u, np.eye(N_SAMPLES), bc_type=((1, np.zeros(N_SAMPLES)), "not-a-knot"))
    return _BASIS


def _profile_matrix(d: np.ndarray, R: float, kappa: float) -> np.ndarray:
    """(len(d), 64) matrix M with f(d) = M @ samples: the spline up to R, and beyond R a
    screened-Coulomb (Yukawa) tail f(R) (R/d) exp(-kappa (d - R))."""
    d = np.asarray(d, dtype=np.float64)
    inside = d <= R
    M = np.where(inside[:, None], _basis()(np.minimum(d, R) / R), 0.0)
    do = np.maximum(d, R)
    M[:, -1] += np.where(inside, 0.0, (R / do) * np.exp(-kappa * (do - R)))
    return M


def _tail_kappa(f: np.ndarray, r: np.ndarray) -> float:
    """Decay rate of r f(r) over samples 54..60 (log-linear least squares), clipped to [0.1, 5]."""
    sl = slice(-10, -3)
    y = np.log(np.maximum(r[sl] * np.abs(f[sl]), 1e-300))
    return float(np.clip(-np.polyfit(r[sl], y, 1)[0], 0.1, 5.0))


_AXIS_IMAGES = [(a, b, c) for a in range(-2, 3) for b in range(-2, 3) for c in range(-2, 3)]
_GRID_IMAGES = [(a, b, c) for a in range(-1, 2) for b in range(-1, 2) for c in range(-1, 2)]


def free_profile(samples: np.ndarray, N: float, iters: int = 4):
    """The isolated-droplet profile f whose periodic image sum sum_m f(|x - m L|) has the given
    samples along the axes; returns (f samples at radii(N), tail decay rate kappa).

    A ground state in the periodic box [-L/2, L/2]^3 is, where its density is small, a solution
    of the linear equation (-1/2 lap - mu) psi = 0, so its tail is a lattice sum of screened
    Coulomb tails, one per periodic image of the droplet.  Along the axis the image terms are
    a small correction, so the 64 x 64 system (spline inside R = L/2, Yukawa tail outside,
    images up to two boxes away) is diagonally dominant; kappa is re-estimated from the
    solution's own tail at each of the `iters` passes."""
    a = np.maximum(np.asarray(samples, dtype=np.float64), 0.0)
    r = radii(N)
    R, L = r[-1], box_length(N)
    f = a.copy()
    kappa = _tail_kappa(a, r)
    for _ in range(iters):
        A = np.zeros((N_SAMPLES, N_SAMPLES))
        for m in _AXIS_IMAGES:
            d = np.sqrt((r - m[0] * L) ** 2 + (m[1] * L) ** 2 + (m[2] * L) ** 2)
            A += _profile_matrix(d, R, kappa)
        f = np.linalg.solve(A, a)
        kappa = _tail_kappa(f, r)
    return f, kappa


def profile_start(samples: np.ndarray, N: float, n: int, seed: Optional[int] = None,
                  amp: float = 1e-3) -> np.ndarray:
    """Radial samples of a droplet in the periodic box, placed on the n^3 grid.

    The samples (|psi| along the axes, as radial_samples returns) are turned into the isolated
    profile f (free_profile), and the field is the image sum sum_m f(|x - m L|) over the 27
    nearest periodic images, clipped at zero, with phase noise as for the Gaussian and
    normalised to N; complex128 (n, n, n), Fortran order.  A purely radial placement would
    miss the cubic (image-induced) shape of a small droplet's tail, which imaginary time then
    removes only at the slow rate |mu|."""
    f, kappa = free_profile(samples, N)
    r = radii(N)
    R, L = r[-1], box_length(N)
    x = axis(n, L)
    h = n // 2
    xp = x[h:]  # the field is symmetric under each x_i -> -x_i: build one octant
    dmax = math.sqrt(3.0) * (xp[-1] + L)
    tab_d = np.linspace(0.0, dmax, 400001)
    tab_f = _profile_matrix(tab_d, R, kappa) @ f
    octant = np.zeros((n - h,) * 3)
    for m in _GRID_IMAGES:
        d = np.sqrt((xp[:, None, None] - m[0] * L) ** 2 + (xp[None, :, None] - m[1] * L) ** 2
                    + (xp[None, None, :] - m[2] * L) ** 2)
        octant += np.interp(d, tab_d, tab_f)
    if n % 2:
        raise ValueError("profile_start needs an even grid")
    line = np.concatenate([np.arange(h - 1, -1, -1), np.arange(h)])  # x_i -> |x_i| index
    psi = octant[np.ix_(line, line, line)]
    psi = np.maximum(psi, 0.0).astype(np.complex128)
    psi = _phase_noise(psi, seed, amp)
    return np.asfortranarray(_normalise(psi, N, L / n))


def lsq_samples(psi: np.ndarray, N: float) -> np.ndarray:
    """Axis samples whose profile_start placement best fits |psi| on its grid.

    The isolated profile f (spline inside R = 2 N^(1/3), screened-Coulomb tail outside, with the
    tail rate of the state's own axis samples) is fitted to |psi| by least squares over one
    octant of the grid with the 27 periodic images profile_start sums (normal equations, with
    a weak ridge toward the profile of the axis samples); the result is returned as the axis
    samples of that image sum, which free_profile turns back into f.  Samples of the state's own axes
    (radial_samples) miss what the images add off the axes; on 128^3 droplets these targets
    save 2.1x the imaginary-time steps where the axis samples save 1.6x."""
    a = np.abs(np.asarray(psi))
    if a.ndim == 4:
        a = a[..., 0]
    n = a.shape[0]
    f_axis, kappa = free_profile(radial_samples(a, N), N)
    r = radii(N)
    R, L = r[-1], box_length(N)
    h = n // 2
    xp = axis(n, L)[h:]
    AtA = np.zeros((N_SAMPLES, N_SAMPLES))
    Aty = np.zeros(N_SAMPLES)
    y = a[h:, h:, h:]
    for k0 in range(0, n - h, 8):  # slices of the octant bound the memory
        A = np.zeros(((n - h) ** 2 * min(8, n - h - k0), N_SAMPLES))
        for m in _GRID_IMAGES:
            d = np.sqrt((xp[:, None, None] - m[0] * L) ** 2 + (xp[None, :, None] - m[1] * L) ** 2
                        + (xp[None, None, k0:k0 + 8] - m[2] * L) ** 2).ravel()
            A += _profile_matrix(d, R, kappa)
        yk = y[:, :, k0:k0 + 8].ravel()
        AtA += A.T @ A
        Aty += A.T @ yk
    # a weak pull toward the axis samples' profile keeps the coefficients that few grid points
    # constrain (the innermost radii, on coarse grids) from drifting
    lam = 1e-6 * float(np.mean(np.diag(AtA)))
    f = np.linalg.solve(AtA + lam * np.eye(N_SAMPLES), Aty + lam * f_axis)
    s = np.zeros(N_SAMPLES)
    for m in _AXIS_IMAGES:
        d = np.sqrt((r - m[0] * L) ** 2 + (m[1] * L) ** 2 + (m[2] * L) ** 2)
        s += _profile_matrix(d, R, kappa) @ f
    return s


def _lsq_job(args):
    psi, N = args
    return lsq_samples(psi, N)


# ---- the network ------------------------------------------------------------------------------
def features(params: Iterable[dict]) -> np.ndarray:
    """Standardised inputs: ((log N - 5.3) / 1.33, (c3 + 3) / 0.2, omega / 0.05 - 1)."""
    rows = [((math.log(p["N"]) - 5.3) / 1.33, (p["c3"] + 3.0) / 0.2, p.get("omega", 0.0) / 0.05 - 1.0)
            for p in params]
    return np.asarray(rows, dtype=np.float32).reshape(-1, 3)


class WarmStart:
    """The trained network and the states it predicts."""

    def __init__(self, device: int = 0, seed: int = 0, params: Optional[np.ndarray] = None):
        self.net = _abi.Mlp(device=device, seed=seed)
        if params is not None:
            self.net.set_params(params)

    def train(self, params: Sequence[dict], samples: np.ndarray, epochs: int, batch: int = 256,
              lr: float = 1e-3, seed: int = 0, lr_decay_every: int = 0) -> np.ndarray:
        """Adam on the MSE of the radial samples; with lr_decay_every > 0 the learning rate
        halves every lr_decay_every epochs.  Returns the per-epoch loss."""
        x = features(params)
        t = np.asarray(samples, dtype=np.float32).reshape(-1, N_SAMPLES)
        if lr_decay_every <= 0:
            return self.net.train(x, t, epochs, batch, lr, seed)
        hist, done, k = [], 0, 0
        while done < epochs:
            e = min(lr_decay_every, epochs - done)
            hist.append(self.net.train(x, t, e, batch, lr * 0.5 ** k, seed + k))
            done += e
            k += 1
        return np.concatenate(hist)

    def predict(self, params: Sequence[dict]) -> np.ndarray:
        return self.net.forward(features(params)).astype(np.float64)

    def start(self, p: dict, n: int, seed: Optional[int] = None, amp: float = 1e-3) -> np.ndarray:
        return profile_start(self.predict([p])[0], p["N"], n, seed, amp)

    def get_params(self) -> np.ndarray:
        return self.net.get_params()

    def save(self, path: str) -> None:
        np.savez_compressed(path, params=self.get_params())

    @classmethod
    def load(cls, path: str = DEFAULT_WEIGHTS, device: int = 0) -> "WarmStart":
        with np.load(path) as z:
            return cls(device=device, params=z["params"])

    def close(self):
        self.net.close()


# ---- data from the batched solver -----------------------------------------------------------
def solve_ground_states(params: Sequence[dict], grid, tol: float, chunk: int = 512,
                        check_every: int = 100, max_steps: int = 400000, precision: int = _abi.GP5_C128,
                        starts=None, device: int = 0, seed: int = 0, keep=None, progress=None,
                        devices: Optional[Sequence[int]] = None, method: int = _abi.GP5_BATCH_RK4):
    """Solves every parameter set with the batched solver from a Gaussian (or
    starts(p, n, index)) on grid(p) (an int or a function of p); returns (states, results)
    lists in the order of params, each state passed through keep(p, psi) when keep is given.
    method: GP5_BATCH_RK4 (imaginary time; results count RK4 steps) or GP5_BATCH_PRECOND (the
    preconditioned iteration to the same ground states, with its step 0.5; results count
    iterations).

    The solves go to the batched solver `chunk` at a time (gp5cu_batch_*), which takes
    finished solves out of its launches at every convergence check, so slow solves cost only
    their own work.  devices: GPUs of this process to spread each chunk over (the solves are
    independent and exchange nothing); default [device].  progress(done, total) is called
    before each chunk."""
    count = len(params)
    gridof = (lambda p: grid(p)) if callable(grid) else (lambda p: int(grid))
    descs = [solve_desc(p, gridof(p)) for p in params]
    devs = list(devices) if devices is not None else [device]
    states, results = [None] * count, [None] * count
    for c0 in range(0, count, chunk):
        part = list(range(c0, min(count, c0 + chunk)))
        if progress is not None:
            progress(c0, count)
        b = _abi.Batch([descs[i] for i in part], precision=precision, devices=devs)
        try:
            if method != _abi.GP5_BATCH_RK4:
                b.set_method(method, 0.5)
            for k, i in enumerate(part):
                if starts is not None:
                    psi = starts(params[i], descs[i]["n"], i)
                else:
                    psi = gaussian_start(params[i]["N"], descs[i]["n"], seed + i)
                b.set_state(k, psi)
            res = b.solve(tol=tol, check_every=check_every, max_steps=max_steps)
            for k, i in enumerate(part):
                results[i] = dict(res[k])
                psi = b.get_state(k)[..., 0]
                states[i] = keep(params[i], psi) if keep is not None else psi
        finally:
            b.close()
    return states, results


# ---- training and evaluation ---------------------------------------------------------------
TRAIN_SEED, TEST_SEED = 1, 2


def training_grid(p: dict) -> int:
    """32^3 where it gives a spacing of at most 0.5 (N <= 64), else 64^3."""
    return smallest_grid(p["N"], (32, 64), 0.5)


def make_training_set(count: int = 4096, seed: int = TRAIN_SEED, grid=training_grid, tol: float = 1e-7,
                      chunk: int = 1024, device: int = 0, devices: Optional[Sequence[int]] = None,
                      targets: str = "axis", start_model: Optional["WarmStart"] = None, workers: int = 8,
                      precision: int = _abi.GP5_C128, method: int = _abi.GP5_BATCH_RK4):
    """Ground states of `count` seeded parameter sets (batched imaginary-time RK4 from the
    noise-free Gaussian, or from start_model's prediction, to residual tol, on grid(p)^3),
    spread over `devices` when given; returns (params, samples [count][64], solver results).

    targets "axis": the states' axis samples (radial_samples); "lsq": the least-squares
    samples (lsq_samples), fitted after each chunk of solves by `workers` spawned processes.
    method: the batched solver's method (GP5_BATCH_PRECOND reaches the same ground states in
    tens of iterations instead of thousands of RK4 steps)."""
    params = sample_params(count, seed)
    import sys
    import time

    t0 = time.time()
    report = lambda done, total: print(f"[{time.time() - t0:7.1f} s] {done} of {total} solves done",
                                       file=sys.stderr, flush=True)
    if start_model is not None:
        starts = lambda p, n, k: start_model.start(p, n)
    else:
        starts = lambda p, n, k: gaussian_start(p["N"], n, None)
    if targets == "axis":
        keep = lambda p, psi: radial_samples(psi, p["N"])
        samples, results = solve_ground_states(params, grid, tol=tol, chunk=chunk, device=device, keep=keep,
                                               progress=report, devices=devices, starts=starts,
                                               precision=precision, method=method,
                                               check_every=5 if method == _abi.GP5_BATCH_PRECOND else 100)
        return params, np.asarray(samples), results
    if targets != "lsq":
        raise ValueError("targets must be 'axis' or 'lsq'")
    import multiprocessing as mp

    for var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ.setdefault(var, "1")  # one BLAS thread per fitting process
    samples, results = [None] * count, [None] * count
    with mp.get_context("spawn").Pool(workers) as pool:
        for c0 in range(0, count, chunk):
            part = list(range(c0, min(count, c0 + chunk)))
            report(c0, count)
            keep = lambda p, psi: np.abs(psi).astype(np.float32)
            st, rs = solve_ground_states([params[i] for i in part], grid, tol=tol, chunk=len(part),
                                         device=device, keep=keep, devices=devices, precision=precision,
                                         starts=lambda p, n, k: starts(p, n, k), method=method,
                                         check_every=5 if method == _abi.GP5_BATCH_PRECOND else 100)
            fits = pool.map(_lsq_job, [(st[k], params[i]["N"]) for k, i in enumerate(part)])
            for k, i in enumerate(part):
                samples[i], results[i] = fits[k], rs[k]
            report(c0 + len(part), count)
    return params, np.asarray(samples), results


def evaluate(model: "WarmStart", count: int = 64, seed: int = TEST_SEED, n: int = 128, tol: float = 1e-8,
             check_every: int = 100, device: int = 0) -> dict:
    """Steps to `tol` from the Gaussian and from the network's start for `count` unseen seeded
    parameter sets on n^3 grids (complex128, both starts noise-free), with the converged
    energies and the network's profile error against the converged states."""
    import sys
    import time

    params = sample_params(count, seed)
    pred = model.predict(params)
    keep = lambda p, psi: radial_samples(psi, p["N"])
    t0 = time.time()
    report = lambda done, total: print(f"[{time.time() - t0:7.1f} s] {done} of {total} solves done",
                                       file=sys.stderr, flush=True)
    sg, rg = solve_ground_states(params, n, tol=tol, chunk=count, check_every=check_every, device=device,
                                 keep=keep, progress=report,
                                 starts=lambda p, m, k: gaussian_start(p["N"], m, None))
    sw, rw = solve_ground_states(params, n, tol=tol, chunk=count, check_every=check_every, device=device,
                                 keep=keep, progress=report,
                                 starts=lambda p, m, k: profile_start(pred[k], p["N"], m, None))
    sg = np.asarray(sg)
    steps_g = np.array([r["steps"] for r in rg])
    steps_w = np.array([r["steps"] for r in rw])
    Eg = np.array([r["energy"] for r in rg])
    Ew = np.array([r["energy"] for r in rw])
    peak = np.max(np.abs(sg), axis=1)
    return dict(
        count=count, seed=seed, grid=n, tol=tol, check_every=check_every,
        params=params,
        steps_gaussian=steps_g.tolist(), steps_warm=steps_w.tolist(),
        converged_gaussian=[bool(r["converged"]) for r in rg], converged_warm=[bool(r["converged"]) for r in rw],
        energy_gaussian=Eg.tolist(), energy_warm=Ew.tolist(),
        total_steps_gaussian=int(steps_g.sum()), total_steps_warm=int(steps_w.sum()),
        step_ratio_total=float(steps_g.sum() / max(steps_w.sum(), 1)),
        step_ratio_median=float(np.median(steps_g / np.maximum(steps_w, 1))),
        max_rel_energy_diff=float(np.max(np.abs(Ew - Eg) / np.abs(Eg))),
        profile_rms_error=float(np.sqrt(np.mean((pred - sg) ** 2))),
        profile_max_rel_error=float(np.max(np.abs(pred - sg) / peak[:, None])),
    )


def main(argv=None):
    import argparse
    import json
    import time

    ap = argparse.ArgumentParser(description="Train or evaluate the droplet warm-start network.")
    ap.add_argument("--train", metavar="OUT_NPZ", help="generate the training set, train, save weights")
    ap.add_argument("--evaluate", metavar="MODEL_NPZ", help="evaluate saved weights on unseen droplets")
    ap.add_argument("--report", metavar="JSON", help="where --evaluate writes its report")
    ap.add_argument("--count", type=int, default=4096)
    ap.add_argument("--epochs", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--decay-every", type=int, default=800)
    ap.add_argument("--data", metavar="NPZ", help="reuse (or save) the training set here")
    ap.add_argument("--test-count", type=int, default=64)
    ap.add_argument("--test-grid", type=int, default=128)
    ap.add_argument("--devices", type=int, nargs="+", default=None,
                    help="GPUs to spread the training-set solves over (independent solves)")
    ap.add_argument("--targets", choices=["axis", "lsq"], default="axis",
                    help="training targets: the states' axis samples, or least-squares samples")
    ap.add_argument("--train-grid", type=int, default=0,
                    help="grid of the training solves (0: 32^3 / 64^3 by the spacing rule)")
    ap.add_argument("--start-from", metavar="MODEL_NPZ",
                    help="start the training solves from this network's prediction")
    ap.add_argument("--chunk", type=int, default=1024, help="training solves per batch")
    ap.add_argument("--workers", type=int, default=8, help="processes fitting least-squares targets")
    ap.add_argument("--complex64", action="store_true",
                    help="training solves with the complex64 bulk and complex128 polish")
    ap.add_argument("--solver", choices=["rk4", "precond"], default="rk4",
                    help="training solves by imaginary-time RK4 or by the preconditioned iteration "
                         "(the same ground states, tens of iterations per solve)")
    a = ap.parse_args(argv)
    if a.train:
        t0 = time.time()
        if a.data and os.path.exists(a.data):
            z = np.load(a.data)
            params = [dict(N=float(r[0]), c3=float(r[1]), omega=float(r[2])) for r in z["params"]]
            samples, steps = z["samples"].astype(np.float64), z["steps"]
        else:
            grid = a.train_grid if a.train_grid > 0 else training_grid
            start_model = WarmStart.load(a.start_from) if a.start_from else None
            params, samples, results = make_training_set(
                a.count, grid=grid, devices=a.devices, targets=a.targets, start_model=start_model,
                chunk=a.chunk, workers=a.workers,
                precision=_abi.GP5_C64 if a.complex64 else _abi.GP5_C128,
                method=_abi.GP5_BATCH_PRECOND if a.solver == "precond" else _abi.GP5_BATCH_RK4)
            if start_model is not None:
                start_model.close()
            steps = np.array([r["steps"] for r in results])
            if a.data:
                table = np.array([[p["N"], p["c3"], p["omega"]] for p in params])
                np.savez_compressed(a.data, params=table, samples=samples.astype(np.float32),
                                    steps=steps.astype(np.int32))
        t1 = time.time()
        model = WarmStart(seed=0)
        hist = model.train(params, samples, a.epochs, a.batch, a.lr, seed=0, lr_decay_every=a.decay_every)
        t2 = time.time()
        model.save(a.train)
        pred = model.predict(params)
        print(json.dumps(dict(count=len(params), data_seconds=round(t1 - t0, 1), train_seconds=round(t2 - t1, 1),
                              solver_steps_mean=float(np.mean(steps)), loss_first=float(hist[0]),
                              loss_last=float(hist[-1]),
                              train_rms=float(np.sqrt(np.mean((pred - samples) ** 2))))))
    if a.evaluate:
        model = WarmStart.load(a.evaluate)
        t0 = time.time()
        rep = evaluate(model, a.test_count, n=a.test_grid)
        rep["seconds"] = round(time.time() - t0, 1)
        if a.report:
            with open(a.report, "w") as fh:
                json.dump(rep, fh, indent=1)
        print(json.dumps({k: v for k, v in rep.items() if not isinstance(v, list)}))


if __name__ == "__main__":
    main()
