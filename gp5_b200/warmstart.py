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
from typing import Iterable, List, Optional, Sequence

import numpy as np

from . import _abi

N_SAMPLES = 64
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


def profile_start(samples: np.ndarray, N: float, n: int, seed: Optional[int] = None,
                  amp: float = 1e-3) -> np.ndarray:
    """Radial samples interpolated onto the n^3 grid (cubic spline with zero slope at r = 0;
    beyond the last radius the last sample), clipped at zero, phase noise as for the Gaussian,
    normalised to N; complex128 (n, n, n), Fortran order."""
    from scipy.interpolate import CubicSpline

    s = np.maximum(np.asarray(samples, dtype=np.float64), 0.0)
    r = radii(N)
    spl = CubicSpline(r, s, bc_type=((1, 0.0), "not-a-knot"))
    L = box_length(N)
    x = axis(n, L)
    R = np.sqrt(x[:, None, None] ** 2 + x[None, :, None] ** 2 + x[None, None, :] ** 2)
    prof = np.where(R <= r[-1], spl(np.minimum(R, r[-1])), s[-1])
    psi = np.maximum(prof, 0.0).astype(np.complex128)
    psi = _phase_noise(psi, seed, amp)
    return np.asfortranarray(_normalise(psi, N, L / n))


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
    def load(cls, path: str, device: int = 0) -> "WarmStart":
        with np.load(path) as z:
            return cls(device=device, params=z["params"])

    def close(self):
        self.net.close()


# ---- data from the batched solver -----------------------------------------------------------
def solve_ground_states(params: Sequence[dict], grid, tol: float, chunk: int = 512,
                        check_every: int = 100, max_steps: int = 400000, precision: int = _abi.GP5_C128,
                        starts=None, device: int = 0, seed: int = 0, keep=None):
    """Solves every parameter set with the batched solver from a Gaussian (or
    starts(p, n, index)) on grid(p) (an int or a function of p); returns (states, results)
    lists, each state passed through keep(p, psi) when keep is given."""
    states, results = [], []
    for c0 in range(0, len(params), chunk):
        part = params[c0:c0 + chunk]
        descs = [solve_desc(p, grid(p) if callable(grid) else int(grid)) for p in part]
        b = _abi.Batch(descs, precision=precision, device=device)
        try:
            for k, (p, d) in enumerate(zip(part, descs)):
                psi = (starts(p, d["n"], c0 + k) if starts is not None
                       else gaussian_start(p["N"], d["n"], seed + c0 + k))
                b.set_state(k, psi)
            res = b.solve(tol=tol, check_every=check_every, max_steps=max_steps)
            for k, p in enumerate(part):
                psi = b.get_state(k)[..., 0]
                states.append(keep(p, psi) if keep is not None else psi)
            results.extend(res)
        finally:
            b.close()
    return states, results
