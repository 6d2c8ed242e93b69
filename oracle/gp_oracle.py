"""CPU oracle for the GP5 pseudo-spectral time stepper (test infrastructure only).

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference`` leg of
``bench.py`` may import it.  It restates, in plain numpy FP64, the arithmetic of
the reference (lucaparisi91/GP5) hot path, in the reference's own order of
operations, so that the CUDA path can be compared against it on the same inputs.

Layout contract (``src/traits.h:20``, ``src/pyTools.h:93-104``): a field is a
complex128 array of shape ``(nx, ny, nz, ncomp)`` in Fortran (ColMajor) order,
x fastest, component slowest.  Every function here accepts any numpy array of
that shape; memory order does not change the values.

Third-party arithmetic: the reference transforms with FFTW3 (unpinned version,
``init.cmake:8-9``; ``fftw_plan_many_dft`` in ``src/fourierTransform.cpp:146-174``).
FFTW is absent here; the DFT it computes (unnormalised, forward e^{-2 pi i jk/n},
backward e^{+2 pi i jk/n}) is restated with ``numpy.fft`` / ``scipy.fft``
(pocketfft) and pinned on small grids by the long-double direct DFT in
``oracle/dft_ld.c``.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field as dc_field
from typing import Optional, Sequence

import numpy as np

try:  # scipy.fft takes a worker count; numpy.fft is the fallback
    import scipy.fft as _sfft
except Exception:  # pragma: no cover
    _sfft = None

_WORKERS = int(os.environ.get("GP5_ORACLE_WORKERS", "0")) or (os.cpu_count() or 1)

# Element-wise work (the K^2 multiply, the functional's point-wise terms, the RK stage
# combinations) can run over z-slabs on a thread pool: numpy releases the GIL inside its
# loops, and every element goes through the same expression as in the serial form.
# Reductions (norms) stay serial.  Default: one thread (the tests' setting).
_EW_THREADS = 1
_EW_POOL = None


def set_elementwise_threads(n: int) -> None:
    global _EW_THREADS, _EW_POOL
    n = max(1, int(n))
    if n > 1 and (_EW_POOL is None or _EW_THREADS != n):
        from concurrent.futures import ThreadPoolExecutor
        _EW_POOL = ThreadPoolExecutor(max_workers=n)
    _EW_THREADS = n


def _slabs(fn, *arrays, min_size: int = 1 << 16):
    """fn(*arrays) for element-wise fn; with more than one thread, evaluated slab by slab
    along axis 2 (arrays of 3 or more dimensions are sliced, anything else is passed as is)."""
    first = next((a for a in arrays if isinstance(a, np.ndarray) and a.ndim >= 3), None)
    if _EW_THREADS <= 1 or first is None or first.size < min_size or first.shape[2] < 2:
        return fn(*arrays)
    nz = first.shape[2]
    nt = min(_EW_THREADS, nz)
    b = np.linspace(0, nz, nt + 1).astype(int)

    def cut(a, i):
        return a[:, :, b[i]:b[i + 1]] if isinstance(a, np.ndarray) and a.ndim >= 3 else a

    parts = list(_EW_POOL.map(lambda i: fn(*[cut(a, i) for a in arrays]), range(nt)))
    # the serial expression keeps its first operand's layout; so does this (a transform of the
    # result rounds differently on a differently laid out array)
    order = "F" if first.flags.f_contiguous and not first.flags.c_contiguous else "C"
    out = np.empty(parts[0].shape[:2] + (nz,) + parts[0].shape[3:], dtype=parts[0].dtype, order=order)

    def put(i):
        out[:, :, b[i]:b[i + 1]] = parts[i]

    list(_EW_POOL.map(put, range(nt)))
    return out



# --------------------------------------------------------------------------------------
# geometry (src/geometry.h, src/geometry.cpp)
# --------------------------------------------------------------------------------------
@dataclass
class Geometry:
    """Uniform periodic box: mesh shape + domain [left, right] per axis.

    Mirrors ``gp::mesh`` / ``gp::domain`` / ``gp::discretization``
    (``src/geometry.h:9-98``) for a single rank (global mesh == local mesh,
    offset 0).
    """

    shape: Sequence[int]
    left: Sequence[float] = (-1.0, -1.0, -1.0)
    right: Sequence[float] = (1.0, 1.0, 1.0)

    def __post_init__(self):
        self.shape = tuple(int(s) for s in self.shape)
        self.left = tuple(float(v) for v in self.left)
        self.right = tuple(float(v) for v in self.right)

    @property
    def lbox(self):
        # domain::updateLBox, geometry.cpp:31-37
        return tuple(self.right[d] - self.left[d] for d in range(3))

    def space_step(self, d: int) -> float:
        # discretization::getSpaceStep, geometry.h:88
        return self.lbox[d] / self.shape[d]

    def fourier_step(self, d: int) -> float:
        # discretization::getFourierStep, geometry.h:90
        return 2 * math.pi / self.lbox[d]

    @property
    def dV(self) -> float:
        # norm(), geometry.cpp:206-210: product of the space steps, in axis order
        dv = 1.0
        for d in range(3):
            dv *= self.space_step(d)
        return dv

    @property
    def n_sites(self) -> int:
        return self.shape[0] * self.shape[1] * self.shape[2]


def momentum_axis(geo: Geometry, d: int) -> np.ndarray:
    """k_d for every index along axis d (``gp::momentums``, geometry.cpp:108-152).

    Even n: m = i for i < n/2, else i - n (Nyquist maps to -n/2).
    Odd n:  m = i for i <= (n-1)/2, else i - n.   k = delta * m, delta = 2 pi / L.
    """
    n = geo.shape[d]
    delta = geo.fourier_step(d)
    out = np.empty(n, dtype=np.float64)
    for i in range(n):
        if n % 2 == 0:
            out[i] = delta * i if i < n // 2 else (-n + i) * delta
        else:
            out[i] = delta * i if i <= (n - 1) // 2 else (-n + i) * delta
    return out


def position_axis(geo: Geometry, d: int) -> np.ndarray:
    """Cell-centred coordinates x_i = left + delta*(i + 0.5) (geometry.cpp:165-188)."""
    n = geo.shape[d]
    delta = geo.space_step(d)
    return np.array([geo.left[d] + delta * (i + 0.5) for i in range(n)], dtype=np.float64)


def grid(geo: Geometry):
    """X, Y, Z as (nx, ny, nz) arrays, indexing 'ij' (``gp.field.grid``, gp.py:77-95)."""
    x, y, z = (position_axis(geo, d) for d in range(3))
    return np.meshgrid(x, y, z, indexing="ij")


def k2_tensor(geo: Geometry) -> np.ndarray:
    """K^2 = KX*KX + KY*KY + KZ*KZ, in that summation order (operators.cpp:17-20)."""
    kx, ky, kz = (momentum_axis(geo, d) for d in range(3))
    KX = kx[:, None, None]
    KY = ky[None, :, None]
    KZ = kz[None, None, :]
    return (KX * KX + KY * KY) + KZ * KZ


def new_field(geo: Geometry, ncomp: int = 1) -> np.ndarray:
    return np.zeros(tuple(geo.shape) + (ncomp,), dtype=np.complex128, order="F")


def init_gaussian(geo: Geometry, sigma, psi: np.ndarray, comp: int = 0) -> None:
    """psi = exp(-(ax x^2 + ay y^2 + az z^2)), a = 1/(2 sigma^2) (geometry.cpp:246-276)."""
    if np.isscalar(sigma):
        sigma = (float(sigma),) * 3
    alpha = [1.0 / (2 * s * s) for s in sigma]
    X, Y, Z = grid(geo)
    tmp = alpha[0] * X * X + alpha[1] * Y * Y + alpha[2] * Z * Z
    psi[..., comp] = np.exp(-tmp) + 0j


def norm(psi: np.ndarray, comp: int, geo: Geometry) -> float:
    """dV * sum(re^2 + im^2) over one component (geometry.cpp:190-214)."""
    f = psi[..., comp]
    s = float(np.sum(f.real * f.real + f.imag * f.imag))
    return s * geo.dV


def normalize(N: float, psi: np.ndarray, comp: int, geo: Geometry) -> None:
    """psi_c *= sqrt(N / norm_c) (geometry.cpp:217-229)."""
    fac = math.sqrt(N * 1.0 / norm(psi, comp, geo))
    psi[..., comp] *= fac


# --------------------------------------------------------------------------------------
# Fourier transform (src/fourierTransform.cpp:146-214) and Laplacian (src/operators.cpp)
# --------------------------------------------------------------------------------------
FORWARD = -1
BACKWARD = +1


def fft3(psi: np.ndarray, direction: int) -> np.ndarray:
    """Unnormalised 3D C2C DFT of every component (fftwFourierTransform::apply, :184-214).

    FORWARD uses e^{-2 pi i jk/n}; BACKWARD uses e^{+2 pi i jk/n} without 1/n.
    """
    a = np.asarray(psi, dtype=np.complex128)
    if _sfft is not None:
        if direction == FORWARD:
            return _sfft.fftn(a, axes=(0, 1, 2), workers=_WORKERS)
        return _sfft.ifftn(a, axes=(0, 1, 2), norm="forward", workers=_WORKERS)
    if direction == FORWARD:
        return np.fft.fftn(a, axes=(0, 1, 2))
    return np.fft.ifftn(a, axes=(0, 1, 2)) * (a.shape[0] * a.shape[1] * a.shape[2])


def laplacian(psi: np.ndarray, geo: Geometry) -> np.ndarray:
    """dst = IFFT(-K^2 * FFT(src)) * (1/N^3) (laplacian::apply, operators.cpp:28-36)."""
    K2 = k2_tensor(geo)[..., None]
    fk = fft3(psi, FORWARD)
    fk = _slabs(lambda f, k: -f * k, fk, K2)
    out = fft3(fk, BACKWARD)
    scale = 1.0 / complex(geo.n_sites, 0)
    return _slabs(lambda o: o * scale, out)


# --------------------------------------------------------------------------------------
# potentials (src/externalPotential.cpp)
# --------------------------------------------------------------------------------------
def harmonic_potential(geo: Geometry, omegas, ncomp: int = 1) -> np.ndarray:
    """V_c = (wx^2 X^2 + wy^2 Y^2 + wz^2 Z^2) * 0.5 (harmonicPotential::create, :11-32).

    ``omegas`` is one (wx, wy, wz) triple per component.  Returns a real array
    (nx, ny, nz, ncomp); the reference stores it as a complex tensor with zero
    imaginary part, which multiplies identically.
    """
    X, Y, Z = grid(geo)
    V = np.zeros(tuple(geo.shape) + (ncomp,), dtype=np.float64, order="F")
    for c in range(ncomp):
        w = omegas[c]
        V[..., c] = (w[0] * w[0] * X * X + w[1] * w[1] * Y * Y + w[2] * w[2] * Z * Z) * 0.5
    return V


# --------------------------------------------------------------------------------------
# functionals (src/functional.cpp)
# --------------------------------------------------------------------------------------
@dataclass
class Functional:
    """H applied by ``functional::apply`` (functional.h:15).

    kind:
      'gp'           gpFunctional (functional.cpp:13-43): -1/2 (1/m_c) lap + V + mean field
                     (1 comp: g|psi|^2 psi, :54-68; 2 comp: g11,g22,g12, :71-89).
      'lhy'          LHYDropletFunctional (functional.cpp:105-122):
                     -1/2 lap + (c3 n + c4 n^{3/2}) psi, n = |psi|^2, c3=-3, c4=5/2 by default;
                     (c3, c4) extended so that quench/batch configs can vary them; the
                     defaults reproduce the reference's hard-coded constants.
      'lhy_unlocked' LHYDropletUnlockedFunctional (functional.cpp:125-150), 2 components.
    """

    kind: str = "lhy"
    couplings: Optional[np.ndarray] = None  # (ncomp, ncomp) for 'gp'
    masses: Optional[Sequence[float]] = None
    c3: float = -3.0
    c4: float = 2.5
    alpha: float = 0.0
    beta: float = 0.0
    eta: float = 0.0
    V: Optional[np.ndarray] = None  # real (nx,ny,nz,ncomp)

    def kinetic(self, psi: np.ndarray, geo: Geometry) -> np.ndarray:
        """-1/2 (1/m) lap(psi) as the reference forms it (before potential/interaction)."""
        return self._kinetic_of(laplacian(psi, geo))

    def _kinetic_of(self, lap: np.ndarray) -> np.ndarray:
        if self.kind == "gp":
            ncomp = lap.shape[3]
            masses = list(self.masses) if self.masses is not None else [1.0] * ncomp
            out = np.empty_like(lap)
            for c in range(ncomp):
                inv_m = 1.0 / masses[c]
                out[..., c] = -0.5 * inv_m * lap[..., c]
            return out
        return -0.5 * lap

    def interaction_factor(self, psi: np.ndarray) -> np.ndarray:
        """f_c(n) so that the interaction part of H psi is f_c * psi_c."""
        ncomp = psi.shape[3]
        if self.kind == "gp":
            if self.couplings is None:
                return np.zeros(psi.shape, dtype=np.float64)
            G = np.asarray(self.couplings, dtype=np.float64)
            n = [psi[..., c].real * psi[..., c].real + psi[..., c].imag * psi[..., c].imag
                 for c in range(ncomp)]
            f = np.zeros(psi.shape, dtype=np.float64)
            if ncomp == 1:
                f[..., 0] = G[0, 0] * n[0]
            elif ncomp == 2:
                f[..., 0] = G[0, 0] * n[0] + G[0, 1] * n[1]
                f[..., 1] = G[1, 1] * n[1] + G[0, 1] * n[0]
            return f
        if self.kind == "lhy":
            n = psi.real * psi.real + psi.imag * psi.imag
            return self.c3 * n + self.c4 * np.power(n, 1.5)
        if self.kind == "lhy_unlocked":
            n1 = np.abs(psi[..., 0]) ** 2
            n2 = np.abs(psi[..., 1]) ** 2
            p = np.power(n1 + self.beta * n2, 1.5)
            f = np.zeros(psi.shape, dtype=np.float64)
            f[..., 0] = n1 + self.eta * n2 + self.alpha * p
            f[..., 1] = self.eta * self.beta * n1 + self.beta * n2 + self.alpha * self.beta * self.beta * p
            return f
        raise ValueError(self.kind)

    def apply(self, psi: np.ndarray, geo: Geometry) -> np.ndarray:
        """H psi in the reference's order: kinetic, (+ V psi), + f psi."""
        return _slabs(self._apply_tail, laplacian(psi, geo), psi, self.V)

    def _apply_tail(self, lap: np.ndarray, psi: np.ndarray, V) -> np.ndarray:
        out = self._kinetic_of(lap)
        if self.kind == "gp":
            # gpFunctional::apply: kinetic, addPotential, then mean field (functional.cpp:13-43)
            if V is not None:
                out = out + V * psi
            out = out + self.interaction_factor(psi) * psi
        else:
            # LHY: kinetic + f psi in one expression, then addPotential (functional.cpp:112-121)
            out = out + self.interaction_factor(psi) * psi
            if V is not None:
                out = out + V * psi
        return out

    # ---- energy density pieces (no reference counterpart; project definitions) -------
    def interaction_energy_density(self, psi: np.ndarray) -> np.ndarray:
        """e_int(n) with d e_int / d n = f(n): GP (g/2) n^2; LHY (c3/2) n^2 + (2 c4/5) n^{5/2}."""
        if self.kind == "gp":
            if self.couplings is None:
                return np.zeros(psi.shape[:3])
            G = np.asarray(self.couplings, dtype=np.float64)
            n = [np.abs(psi[..., c]) ** 2 for c in range(psi.shape[3])]
            if psi.shape[3] == 1:
                return 0.5 * G[0, 0] * n[0] ** 2
            return 0.5 * G[0, 0] * n[0] ** 2 + 0.5 * G[1, 1] * n[1] ** 2 + G[0, 1] * n[0] * n[1]
        if self.kind == "lhy":
            n = np.abs(psi[..., 0]) ** 2
            return 0.5 * self.c3 * n * n + 0.4 * self.c4 * n * n * np.sqrt(n)
        if self.kind == "lhy_unlocked":
            n1 = np.abs(psi[..., 0]) ** 2
            n2 = np.abs(psi[..., 1]) ** 2
            m = n1 + self.beta * n2
            return 0.5 * n1 * n1 + 0.5 * self.beta * n2 * n2 + self.eta * n1 * n2 + 0.4 * self.alpha * m * m * np.sqrt(m)
        raise ValueError(self.kind)


def observables(func: Functional, psi: np.ndarray, geo: Geometry) -> dict:
    """Energy, chemical potential and residual of psi (project definitions).

    E   = dV sum[ <psi|T psi> + V |psi|^2 + e_int(n) ]
    mu  = Re<psi|H psi> / <psi|psi>
    res = ||H psi - mu psi|| / ||psi||
    """
    dV = geo.dV
    T = func.kinetic(psi, geo)
    Hpsi = func.apply(psi, geo)
    nrm2 = float(np.sum(np.abs(psi) ** 2)) * dV
    ekin = float(np.sum((np.conj(psi) * T).real)) * dV
    epot = float(np.sum(func.V * np.abs(psi) ** 2)) * dV if func.V is not None else 0.0
    eint = float(np.sum(func.interaction_energy_density(psi))) * dV
    hexp = float(np.sum((np.conj(psi) * Hpsi).real)) * dV
    mu = hexp / nrm2
    res = math.sqrt(float(np.sum(np.abs(Hpsi - mu * psi) ** 2)) * dV / nrm2)
    return {"norm": nrm2, "E": ekin + epot + eint, "ekin": ekin, "epot": epot,
            "eint": eint, "mu": mu, "residual": res}


# --------------------------------------------------------------------------------------
# steppers (src/stepper.cpp) and the Python time stepper (src/gpCpp.cpp:202-287)
# --------------------------------------------------------------------------------------
@dataclass
class Stepper:
    """euleroStepper / RK4Stepper with complex time step (stepper.cpp:30-71).

    dt is real for imaginary time (tau = (dt, 0)), i*dt for real time
    (gpCpp.cpp:217-224).  ``normalizations`` enables stepper::normalize on every
    stage input and on the result (stepper.cpp:7-22, 51, 56, 61, 67).
    """

    func: Functional
    geo: Geometry
    dt: float
    name: str = "RK4"
    imaginary: bool = True
    normalizations: Optional[Sequence[float]] = None
    constraint_phase: Optional[np.ndarray] = None  # phaseConstraint (constraint.cpp:6-9)
    t: float = 0.0

    @property
    def tau(self) -> complex:
        return complex(self.dt, 0.0) if self.imaginary else complex(0.0, self.dt)

    def _normalize(self, f: np.ndarray) -> None:
        if self.normalizations is not None:
            for c, N in enumerate(self.normalizations):
                normalize(N, f, c, self.geo)

    def _constrain(self, f: np.ndarray) -> np.ndarray:
        if self.constraint_phase is None:
            return f
        return _slabs(lambda a, ph: np.sqrt(a * np.conj(a)) * np.exp(1j * ph), f, self.constraint_phase)

    def step(self, psi0: np.ndarray) -> np.ndarray:
        tau = self.tau
        H = lambda u: self.func.apply(u, self.geo)  # noqa: E731
        if self.name.lower() in ("eulero", "euler"):
            k1 = H(psi0)
            new = _slabs(lambda a, k: a - tau * k, psi0, k1)
            new = self._constrain(new)
            self._normalize(new)
            return new
        k1 = H(psi0)
        new = _slabs(lambda a, k: a - tau * 0.5 * k, psi0, k1)
        self._normalize(new)
        k2 = H(new)
        new = _slabs(lambda a, k: a - tau * 0.5 * k, psi0, k2)
        self._normalize(new)
        k3 = H(new)
        new = _slabs(lambda a, k: a - tau * k, psi0, k3)
        self._normalize(new)
        k4 = H(new)
        new = _slabs(lambda a, b, c, d, e: a - (1.0 / 6) * tau * (b + 2 * c + 2 * d + e), psi0, k1, k2, k3, k4)
        new = self._constrain(new)
        self._normalize(new)
        return new

    def advance(self, psi: np.ndarray, n_steps: int = 1) -> np.ndarray:
        """timeStepper::advance (gpCpp.cpp:255-269): n steps, t += dt each."""
        for _ in range(n_steps):
            psi = self.step(psi)
            self.t += self.dt
        return psi


# --------------------------------------------------------------------------------------
# the reference's imaginary-time mu protocol (python/test/regressionTests/LHY_imaginary.py)
# --------------------------------------------------------------------------------------
def mu_from_norm_decay(N: float, norm_after: float, dt: float) -> float:
    """mu = 0.5 ln(N / ||psi||^2) / dt after one unnormalised step (LHY_imaginary.py:48)."""
    return 0.5 * math.log(N / norm_after) / dt


def lhy_mu_protocol(shape=(30, 30, 30), box=10.0, sigma=5.0, N=370.0, dt_factor=0.01,
                    steps_per_block=1000, tol=1e-9, max_blocks=1000, callback=None):
    """Runs LHY_imaginary.py:8-49: normalise before every RK4 step, mu per 1000-step block,
    stop when |mu - old_mu| <= tol.  Returns (mu, blocks, psi)."""
    geo = Geometry(shape, (-box,) * 3, (box,) * 3)
    psi = new_field(geo)
    init_gaussian(geo, sigma, psi)
    normalize(N, psi, 0, geo)
    st = Stepper(Functional("lhy"), geo, dt_factor * geo.space_step(0) ** 2, "RK4", True)
    old_mu, mu, it = 0.0, 1.0e18, 0
    while abs(mu - old_mu) > tol and it < max_blocks:
        it += 1
        for _ in range(steps_per_block):
            normalize(N, psi, 0, geo)
            psi = st.advance(psi, 1)
        old_mu = mu
        mu = mu_from_norm_decay(N, norm(psi, 0, geo), st.dt)
        normalize(N, psi, 0, geo)
        if callback is not None:
            callback(it, mu)
    return mu, it, psi


# --------------------------------------------------------------------------------------
# preconditioned ground-state iteration (a project method: the reference reaches ground
# states only by imaginary-time stepping)
# --------------------------------------------------------------------------------------
def precond_ground_state(func: "Functional", geo: Geometry, psi: np.ndarray, N: float, theta: float = 0.5,
                         tol: float = 1e-8, check_every: int = 5, max_iter: int = 2000,
                         alpha_min: float = 0.05, v_share: float = 0.5):
    """psi <- normalise_N(psi - theta (alpha - 1/2 lap)^{-1} (H psi - mu psi)) until the residual
    ||H psi - mu psi|| / ||psi|| (observables) is at most tol, checked every check_every
    iterations; mu = Re<psi|H psi>/<psi|psi> of the current state and alpha = max(|mu|,
    alpha_min, v_share max V), the shifted inverse kinetic operator (unit mass, one component)
    applied in k-space.  The preconditioner does not see the external potential V: a shift well
    below its maximum lets the slowly varying modes where V is large overshoot (theta (V - mu) /
    alpha must stay below 2), so the shift takes a share of max V over the grid (0 without a
    potential).  The same arithmetic as the batched solver's GP5_BATCH_PRECOND.  Returns (psi,
    iterations, observables of the last check)."""
    vcap = v_share * float(np.max(func.V)) if func.V is not None else 0.0
    psi = np.array(psi, dtype=np.complex128, order="F")
    half_k2 = 0.5 * k2_tensor(geo)
    it = 0
    while True:
        if it % check_every == 0 or it >= max_iter:
            ob = observables(func, psi, geo)
            if ob["residual"] <= tol or it >= max_iter:
                return psi, it, ob
        h = func.apply(psi, geo)
        mu = float(np.sum((np.conj(psi) * h).real)) / float(np.sum(np.abs(psi) ** 2))
        r = (h - mu * psi)[..., 0]
        d = np.fft.ifftn(np.fft.fftn(r) / (max(abs(mu), alpha_min, vcap) + half_k2))
        psi[..., 0] = psi[..., 0] - theta * d
        normalize(N, psi, 0, geo)
        it += 1


# --------------------------------------------------------------------------------------
# seeded synthetic inputs for the benchmark configurations
# --------------------------------------------------------------------------------------
def gaussian_with_noise(geo: Geometry, sigma: float, amp: float, seed: int, N: float,
                        phase_noise: bool = False) -> np.ndarray:
    """Gaussian start plus seeded noise, normalised to N.

    phase_noise=False: psi = G + amp*(U(-1,1) + i U(-1,1)) (64^3 harmonic GP start).
    phase_noise=True:  psi = G * exp(i amp U(-1,1))          (droplet starts).
    """
    rng = np.random.default_rng(seed)
    psi = new_field(geo)
    init_gaussian(geo, sigma, psi)
    shp = tuple(geo.shape)
    if phase_noise:
        ph = rng.uniform(-1.0, 1.0, size=shp)
        psi[..., 0] = psi[..., 0] * np.exp(1j * amp * ph)
    else:
        re = rng.uniform(-1.0, 1.0, size=shp)
        im = rng.uniform(-1.0, 1.0, size=shp)
        psi[..., 0] = psi[..., 0] + amp * (re + 1j * im)
    normalize(N, psi, 0, geo)
    return psi
