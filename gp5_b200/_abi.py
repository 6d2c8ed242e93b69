"""ctypes binding of the C ABI in include/gp5cu.h, plus small owning wrappers.

The wrappers (``Plan``, ``DeviceField``, ``Functional``, ``Stepper``) hold device memory
allocated through the library itself, so no other GPU framework is needed.  Every call
checks the status code and raises ``Gp5Error`` with the library's message; there is no
fallback path: if ``libgp5cu.so`` is missing, importing this module fails.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import weakref
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgp5cu.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "gp5cu.h")

GP5_OK, GP5_ERR_ARG, GP5_ERR_CUDA, GP5_ERR_NONFINITE, GP5_ERR_TIMEOUT = 0, 1, 2, 3, 4
GP5_ERR_UNSUPPORTED, GP5_ERR_STATE, GP5_ERR_NOMEM, GP5_ERR_IO = 5, 6, 7, 8
GP5_C128, GP5_C64 = 0, 1
GP5_GEMM_WAIT_DEFAULT_NS = 2_000_000_000
GP5_RING_WAIT_DEFAULT_NS = 2_000_000_000
GP5_FORWARD, GP5_BACKWARD = -1, 1
GP5_FUNC_GP, GP5_FUNC_LHY, GP5_FUNC_LHY_UNLOCKED = 0, 1, 2
GP5_POT_NONE, GP5_POT_HARMONIC, GP5_POT_ARRAY = 0, 1, 2
GP5_STEP_EULER, GP5_STEP_RK4 = 0, 1
GP5_BATCH_RK4, GP5_BATCH_PRECOND = 0, 1


class Gp5Error(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"gp5cu status {status}: {msg}")
        self.status = status


class FunctionalDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_int),
        ("has_couplings", C.c_int),
        ("couplings", C.c_double * 4),
        ("masses", C.c_double * 2),
        ("c3", C.c_double),
        ("c4", C.c_double),
        ("alpha", C.c_double),
        ("beta", C.c_double),
        ("eta", C.c_double),
        ("potential", C.c_int),
        ("omegas", (C.c_double * 3) * 2),
        ("dpotential", C.c_void_p),
    ]


class Observables(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("norm", "energy", "ekin", "epot", "eint", "mu", "residual")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class SolveDesc(C.Structure):
    _fields_ = [("n", C.c_int), ("L", C.c_double), ("N", C.c_double), ("c3", C.c_double), ("c4", C.c_double),
                ("omega", C.c_double), ("dt", C.c_double)]


class SolveResult(C.Structure):
    _fields_ = [("steps", C.c_int), ("converged", C.c_int), ("residual", C.c_double), ("energy", C.c_double),
                ("mu", C.c_double), ("norm", C.c_double), ("steps_c64", C.c_int)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


def header_functions(path: str = HEADER):
    """Names of every function declared in include/gp5cu.h."""
    txt = open(path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(gp5cu_\w+)\s*\(", txt)))


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built (python -m gp5_b200.build)")
    L = C.CDLL(LIB_PATH)
    vp, i, d, pp = C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_void_p)
    proto = {
        "gp5cu_version": (i, []),
        "gp5cu_status_string": (C.c_char_p, [i]),
        "gp5cu_last_error": (C.c_char_p, []),
        "gp5cu_plan_create": (i, [pp, C.POINTER(C.c_int), C.POINTER(d), C.POINTER(d), i, i, i]),
        "gp5cu_plan_destroy": (i, [vp]),
        "gp5cu_plan_set_stream": (i, [vp, vp]),
        "gp5cu_plan_synchronize": (i, [vp]),
        "gp5cu_field_bytes": (C.c_size_t, [vp]),
        "gp5cu_field_alloc": (i, [vp, pp]),
        "gp5cu_field_free": (i, [vp, vp]),
        "gp5cu_upload": (i, [vp, vp, vp]),
        "gp5cu_download": (i, [vp, vp, vp]),
        "gp5cu_upload_c128": (i, [vp, vp, vp]),
        "gp5cu_download_c128": (i, [vp, vp, vp]),
        "gp5cu_fft": (i, [vp, vp, vp, i]),
        "gp5cu_laplacian": (i, [vp, vp, vp]),
        "gp5cu_norm": (i, [vp, vp, i, C.POINTER(d)]),
        "gp5cu_normalize": (i, [vp, vp, i, d]),
        "gp5cu_max_density": (i, [vp, vp, C.POINTER(d)]),
        "gp5cu_init_gaussian": (i, [vp, vp, i, C.POINTER(d)]),
        "gp5cu_functional_desc_init": (None, [C.POINTER(FunctionalDesc)]),
        "gp5cu_functional_create": (i, [vp, C.POINTER(FunctionalDesc), pp]),
        "gp5cu_functional_destroy": (i, [vp]),
        "gp5cu_apply_H": (i, [vp, vp, vp]),
        "gp5cu_observables": (i, [vp, vp, C.POINTER(Observables)]),
        "gp5cu_stepper_create": (i, [vp, i, d, i, pp]),
        "gp5cu_stepper_destroy": (i, [vp]),
        "gp5cu_stepper_set_renormalization": (i, [vp, i, C.POINTER(d)]),
        "gp5cu_stepper_set_phase_constraint": (i, [vp, vp]),
        "gp5cu_stepper_set_compensation": (i, [vp, i]),
        "gp5cu_stepper_set_stochastic_rounding": (i, [vp, C.c_int]),
        "gp5cu_stepper_advance": (i, [vp, vp, i]),
        "gp5cu_stepper_get_time": (i, [vp, C.POINTER(d)]),
        "gp5cu_stepper_set_time": (i, [vp, d]),
        "gp5cu_stepper_advance_host": (i, [vp, vp, vp, i]),
        "gp5cu_stepper_advance_host_many": (i, [vp, i, C.POINTER(vp), C.POINTER(vp), i]),
        "gp5cu_stepper_launches_per_step": (i, [vp]),
        "gp5cu_stepper_profile": (i, [vp, vp, i, C.POINTER(d), C.POINTER(i), i, C.POINTER(i)]),
        "gp5cu_norm_noalloc": (i, [vp, i, C.POINTER(C.c_int), i, i, d, vp, C.POINTER(d)]),
        "gp5cu_h5_save_field": (i, [C.c_char_p, vp, C.POINTER(C.c_int), i]),
        "gp5cu_h5_field_shape": (i, [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "gp5cu_h5_load_field": (i, [C.c_char_p, vp, C.POINTER(C.c_int), i]),
        "gp5cu_h5_dataset_info": (i, [C.c_char_p, C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_longlong),
                                      C.POINTER(C.c_int)]),
        "gp5cu_h5_read_dataset": (i, [C.c_char_p, C.c_char_p, vp, C.c_longlong]),
        "gp5cu_batch_create": (i, [pp, i, C.POINTER(SolveDesc), i, i]),
        "gp5cu_batch_create_devices": (i, [pp, i, C.POINTER(SolveDesc), i, i, C.POINTER(C.c_int)]),
        "gp5cu_batch_assign_devices": (i, [i, C.POINTER(SolveDesc), i, C.POINTER(C.c_int)]),
        "gp5cu_batch_device": (i, [vp, i]),
        "gp5cu_batch_destroy": (i, [vp]),
        "gp5cu_batch_set_state": (i, [vp, i, vp]),
        "gp5cu_batch_get_state": (i, [vp, i, vp]),
        "gp5cu_batch_solve": (i, [vp, d, i, i, C.POINTER(SolveResult)]),
        "gp5cu_batch_launches": (C.c_longlong, [vp]),
        "gp5cu_batch_set_method": (i, [vp, i, d]),
        "gp5cu_decompose": (i, [vp, vp, i, d, vp, C.POINTER(C.c_int)]),
        "gp5cu_decompose_host": (i, [vp, vp, i, d, vp, C.POINTER(C.c_int)]),
        "gp5cu_plan_autotune": (i, [vp]),
        "gp5cu_plan_get_tiles": (i, [vp, C.POINTER(C.c_int)]),
        "gp5cu_plan_set_tiles": (i, [vp, C.POINTER(C.c_int)]),
        "gp5cu_plan_get_radix": (i, [vp, C.POINTER(C.c_int)]),
        "gp5cu_plan_set_radix": (i, [vp, C.POINTER(C.c_int)]),
        "gp5cu_plan_set_wait_bound": (i, [vp, C.c_ulonglong]),
        "gp5cu_mlp_create": (i, [pp, i, C.c_ulonglong]),
        "gp5cu_mlp_destroy": (i, [vp]),
        "gp5cu_mlp_num_params": (C.c_longlong, [vp]),
        "gp5cu_mlp_get_params": (i, [vp, vp]),
        "gp5cu_mlp_set_params": (i, [vp, vp]),
        "gp5cu_mlp_forward": (i, [vp, vp, i, vp]),
        "gp5cu_mlp_gradients": (i, [vp, vp, vp, i, vp, C.POINTER(d)]),
        "gp5cu_mlp_train": (i, [vp, vp, vp, i, i, i, C.c_float, C.c_ulonglong, vp]),
        "gp5cu_mlp_set_wait_bound": (i, [vp, C.c_ulonglong]),
        "gp5cu_gemm_bf16": (i, [vp, C.c_longlong, C.c_longlong, vp, C.c_longlong, C.c_longlong, vp,
                                C.c_longlong, i, i, i, vp]),
    }
    for name, (res, args) in proto.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(status: int) -> None:
    if status != GP5_OK:
        msg = lib().gp5cu_last_error().decode(errors="replace")
        raise Gp5Error(status, msg)


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class Plan:
    """Discretisation + FFT plan on one device (fourierTransformCreator::create)."""

    def __init__(self, shape: Sequence[int], left: Sequence[float], right: Sequence[float],
                 ncomp: int = 1, precision: int = GP5_C128, device: int = 0):
        self.shape = tuple(int(s) for s in shape)
        self.left = tuple(float(v) for v in left)
        self.right = tuple(float(v) for v in right)
        self.ncomp = int(ncomp)
        self.precision = precision
        self._children = weakref.WeakSet()
        h = C.c_void_p()
        check(lib().gp5cu_plan_create(C.byref(h), (C.c_int * 3)(*self.shape), (C.c_double * 3)(*self.left),
                                      (C.c_double * 3)(*self.right), self.ncomp, precision, device))
        self.h = h

    @property
    def cdtype(self):
        return np.complex128 if self.precision == GP5_C128 else np.complex64

    @property
    def field_shape(self):
        return self.shape + (self.ncomp,)

    @property
    def field_bytes(self) -> int:
        return int(lib().gp5cu_field_bytes(self.h))

    def field(self, host: Optional[np.ndarray] = None) -> "DeviceField":
        f = DeviceField(self)
        if host is not None:
            f.upload(host)
        return f

    def fft(self, src: "DeviceField", dst: "DeviceField", direction: int) -> None:
        check(lib().gp5cu_fft(self.h, src.ptr, dst.ptr, direction))

    def laplacian(self, src: "DeviceField", dst: "DeviceField") -> None:
        check(lib().gp5cu_laplacian(self.h, src.ptr, dst.ptr))

    def norm(self, f: "DeviceField", comp: int = 0) -> float:
        out = C.c_double()
        check(lib().gp5cu_norm(self.h, f.ptr, comp, C.byref(out)))
        return out.value

    def normalize(self, f: "DeviceField", N: float, comp: int = 0) -> None:
        check(lib().gp5cu_normalize(self.h, f.ptr, comp, float(N)))

    def init_gaussian(self, f: "DeviceField", sigma, comp: int = 0) -> None:
        """f[..., comp] = exp(-sum_d x_d^2 / (2 sigma_d^2)) on the device (gp5cu_init_gaussian)."""
        sig = (float(sigma),) * 3 if np.isscalar(sigma) else tuple(float(v) for v in sigma)
        check(lib().gp5cu_init_gaussian(self.h, f.ptr, comp, (C.c_double * 3)(*sig)))

    def max_density(self, f: "DeviceField") -> float:
        out = C.c_double()
        check(lib().gp5cu_max_density(self.h, f.ptr, C.byref(out)))
        return out.value

    def decompose(self, f: "DeviceField", cutoff: float, comp: int = 0):
        """Droplet labels (gp5cu_decompose_host): int32 (nx, ny, nz, ncomp), Fortran order, and
        the number of clusters."""
        out = np.empty(self.field_shape, dtype=np.int32, order="F")
        k = C.c_int()
        check(lib().gp5cu_decompose_host(self.h, f.ptr, int(comp), float(cutoff), C.c_void_p(_ptr(out)),
                                         C.byref(k)))
        return out, k.value

    def tiles(self):
        """Threads per CTA of (y fwd, y inv, z fwd, z inv, z fwd*K^2*inv); 0 = default shape."""
        t = (C.c_int * 5)()
        check(lib().gp5cu_plan_get_tiles(self.h, t))
        return list(t)

    def set_tiles(self, threads) -> None:
        t = (C.c_int * 5)(*[int(v) for v in threads])
        check(lib().gp5cu_plan_set_tiles(self.h, t))

    def radix(self):
        """Radix schedules (0/1) of (y fwd, y inv, z fwd, z inv, z fwd*K^2*inv), then the x stage
        boundary's choice (bit 0 schedule, bit 1 bulk-copy ring)."""
        r = (C.c_int * 6)()
        check(lib().gp5cu_plan_get_radix(self.h, r))
        return list(r)

    def set_radix(self, radix) -> None:
        r = (C.c_int * 6)(*[int(v) for v in radix])
        check(lib().gp5cu_plan_set_radix(self.h, r))

    def set_wait_bound(self, ns: int) -> None:
        """Bound of the bulk-copy ring's stage waits (gp5cu_plan_set_wait_bound)."""
        check(lib().gp5cu_plan_set_wait_bound(self.h, int(ns)))

    def autotune(self) -> None:
        check(lib().gp5cu_plan_autotune(self.h))

    def synchronize(self) -> None:
        check(lib().gp5cu_plan_synchronize(self.h))

    def set_stream(self, stream_handle: int) -> None:
        check(lib().gp5cu_plan_set_stream(self.h, C.c_void_p(stream_handle or None)))

    def close(self):
        # children (fields, functionals, steppers) go first: their handles refer to the plan
        if getattr(self, "h", None):
            for c in sorted(list(self._children), key=lambda c: -c._order):
                c.close()
            lib().gp5cu_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceField:
    """One field (nx, ny, nz, ncomp) in device memory, allocated by the library."""

    _order = 0

    def __init__(self, plan: Plan):
        self.plan = plan
        p = C.c_void_p()
        check(lib().gp5cu_field_alloc(plan.h, C.byref(p)))
        self.ptr = p
        plan._children.add(self)

    def upload(self, host: np.ndarray) -> None:
        a = np.asarray(host)
        if a.ndim == 3:
            a = a[..., None]
        if a.shape != self.plan.field_shape:
            raise ValueError(f"shape {a.shape} != {self.plan.field_shape}")
        a = np.asfortranarray(a.astype(np.complex128, copy=False))
        if self.plan.precision == GP5_C128:
            check(lib().gp5cu_upload(self.plan.h, self.ptr, C.c_void_p(_ptr(a))))
        else:
            check(lib().gp5cu_upload_c128(self.plan.h, self.ptr, C.c_void_p(_ptr(a))))

    def download(self) -> np.ndarray:
        out = np.empty(self.plan.field_shape, dtype=np.complex128, order="F")
        if self.plan.precision == GP5_C128:
            check(lib().gp5cu_download(self.plan.h, self.ptr, C.c_void_p(_ptr(out))))
        else:
            check(lib().gp5cu_download_c128(self.plan.h, self.ptr, C.c_void_p(_ptr(out))))
        return out

    def close(self):
        if getattr(self, "ptr", None) and getattr(self.plan, "h", None):
            lib().gp5cu_field_free(self.plan.h, self.ptr)
        self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Functional:
    _order = 1

    def __init__(self, plan: Plan, kind: int = GP5_FUNC_LHY, couplings=None, masses=None, c3=-3.0, c4=2.5,
                 alpha=0.0, beta=0.0, eta=0.0, omegas=None, potential: Optional[DeviceField] = None,
                 potential_ptr: Optional[int] = None):
        self.plan = plan
        d = FunctionalDesc()
        lib().gp5cu_functional_desc_init(C.byref(d))
        d.kind = kind
        if couplings is not None:
            g = np.asarray(couplings, dtype=np.float64).reshape(-1)
            if g.size == 1:
                d.couplings[0] = g[0]
            else:
                for k in range(4):
                    d.couplings[k] = g[k]
            d.has_couplings = 1
        if masses is not None:
            for c, m in enumerate(masses):
                d.masses[c] = m
        d.c3, d.c4, d.alpha, d.beta, d.eta = c3, c4, alpha, beta, eta
        if omegas is not None:
            d.potential = GP5_POT_HARMONIC
            for c, w in enumerate(omegas):
                for k in range(3):
                    d.omegas[c][k] = w[k]
        if potential_ptr is not None:
            d.potential = GP5_POT_ARRAY
            d.dpotential = potential_ptr
        self.desc = d
        h = C.c_void_p()
        check(lib().gp5cu_functional_create(plan.h, C.byref(d), C.byref(h)))
        self.h = h
        plan._children.add(self)

    def apply(self, src: DeviceField, dst: DeviceField) -> None:
        check(lib().gp5cu_apply_H(self.h, src.ptr, dst.ptr))

    def observables(self, f: DeviceField) -> dict:
        o = Observables()
        check(lib().gp5cu_observables(self.h, f.ptr, C.byref(o)))
        return o.as_dict()

    def close(self):
        # a plan that is already gone took the functional's memory with it
        if getattr(self, "h", None) and getattr(self.plan, "h", None):
            lib().gp5cu_functional_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Stepper:
    _order = 2

    def __init__(self, func: Functional, dt: float, kind: int = GP5_STEP_RK4, imaginary: bool = True):
        self.func = func
        self.dt = float(dt)
        h = C.c_void_p()
        check(lib().gp5cu_stepper_create(func.h, kind, self.dt, 1 if imaginary else 0, C.byref(h)))
        self.h = h
        func.plan._children.add(self)

    def set_renormalization(self, N: Optional[Sequence[float]]) -> None:
        if N is None:
            check(lib().gp5cu_stepper_set_renormalization(self.h, 0, None))
        else:
            arr = (C.c_double * len(N))(*N)
            check(lib().gp5cu_stepper_set_renormalization(self.h, len(N), arr))

    def set_compensation(self, on: bool) -> None:
        """Compensated complex64 state update (gp5cu_stepper_set_compensation)."""
        check(lib().gp5cu_stepper_set_compensation(self.h, 1 if on else 0))

    def set_stochastic_rounding(self, on: bool) -> None:
        """Unbiased (stochastic) rounding of the complex64 state update."""
        check(lib().gp5cu_stepper_set_stochastic_rounding(self.h, 1 if on else 0))

    def set_phase_constraint(self, phase: Optional[DeviceField]) -> None:
        check(lib().gp5cu_stepper_set_phase_constraint(self.h, phase.ptr if phase is not None else None))

    def advance(self, f: DeviceField, nsteps: int = 1) -> None:
        check(lib().gp5cu_stepper_advance(self.h, f.ptr, int(nsteps)))

    def advance_host(self, host_in: np.ndarray, host_out: np.ndarray, nsteps: int) -> None:
        check(lib().gp5cu_stepper_advance_host(self.h, C.c_void_p(_ptr(host_in)), C.c_void_p(_ptr(host_out)),
                                               int(nsteps)))

    def advance_host_many(self, host_in, host_out, nsteps: int) -> None:
        """Independent host states, pipelined (gp5cu_stepper_advance_host_many); host_in and
        host_out are lists of arrays (or of raw addresses) of one field each."""
        n = len(host_in)
        addr = lambda a: a if isinstance(a, int) else _ptr(a)  # noqa: E731
        ins = (C.c_void_p * n)(*[addr(a) for a in host_in])
        outs = (C.c_void_p * n)(*[addr(a) for a in host_out])
        check(lib().gp5cu_stepper_advance_host_many(self.h, n, ins, outs, int(nsteps)))

    @property
    def time(self) -> float:
        t = C.c_double()
        check(lib().gp5cu_stepper_get_time(self.h, C.byref(t)))
        return t.value

    def profile(self, f: DeviceField, nrep: int = 3):
        """Mean duration (ms) and kind of every kernel launch of one step."""
        cap = 256
        ms = (C.c_double * cap)()
        kinds = (C.c_int * cap)()
        n = C.c_int()
        check(lib().gp5cu_stepper_profile(self.h, f.ptr, int(nrep), ms, kinds, cap, C.byref(n)))
        return [(int(kinds[k]), float(ms[k])) for k in range(min(n.value, cap))]

    @property
    def launches_per_step(self) -> int:
        return int(lib().gp5cu_stepper_launches_per_step(self.h))

    def close(self):
        if getattr(self, "h", None) and getattr(self.func.plan, "h", None):
            lib().gp5cu_stepper_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def h5_save_field(path: str, psi: np.ndarray) -> None:
    """Writes a (nx, ny, nz[, ncomp]) complex field to an HDF5 file in the reference's layout
    (gp5cu_h5_save_field)."""
    a = np.asarray(psi)
    if a.ndim == 3:
        a = a[..., None]
    a = np.asfortranarray(a.astype(np.complex128, copy=False))
    check(lib().gp5cu_h5_save_field(os.fsencode(path), C.c_void_p(_ptr(a)), (C.c_int * 3)(*a.shape[:3]),
                                    a.shape[3]))


def h5_field_shape(path: str):
    """((nx, ny, nz), ncomp) of the "field" dataset of an HDF5 file."""
    s, nc = (C.c_int * 3)(), C.c_int()
    check(lib().gp5cu_h5_field_shape(os.fsencode(path), s, C.byref(nc)))
    return tuple(s), nc.value


def h5_load_field(path: str) -> np.ndarray:
    """The "field" dataset of an HDF5 file as a (nx, ny, nz, ncomp) complex128 array."""
    shape, nc = h5_field_shape(path)
    out = np.empty(shape + (nc,), dtype=np.complex128, order="F")
    check(lib().gp5cu_h5_load_field(os.fsencode(path), C.c_void_p(_ptr(out)), (C.c_int * 3)(*shape), nc))
    return out


def h5_read_dataset(path: str, name: str) -> np.ndarray:
    """Any float64 dataset (real or complex) of the root group, with its HDF5 dims."""
    rank, dims, cplx = C.c_int(), (C.c_longlong * 8)(), C.c_int()
    check(lib().gp5cu_h5_dataset_info(os.fsencode(path), name.encode(), C.byref(rank), dims, C.byref(cplx)))
    shape = tuple(dims[k] for k in range(rank.value))
    n = int(np.prod(shape, dtype=np.int64)) * (2 if cplx.value else 1)
    out = np.empty(n, dtype=np.float64)
    check(lib().gp5cu_h5_read_dataset(os.fsencode(path), name.encode(), C.c_void_p(_ptr(out)), n))
    return out.view(np.complex128).reshape(shape) if cplx.value else out.reshape(shape)


def solve_descs(solves):
    arr = (SolveDesc * len(solves))()
    for k, sd in enumerate(solves):
        arr[k] = SolveDesc(int(sd["n"]), float(sd["L"]), float(sd["N"]), float(sd.get("c3", -3.0)),
                           float(sd.get("c4", 2.5)), float(sd.get("omega", 0.0)), float(sd["dt"]))
    return arr


def assign_devices(solves, ndevices: int):
    """Positions in [0, ndevices) of the device each solve runs on (gp5cu_batch_assign_devices);
    host-only, no GPU needed."""
    out = (C.c_int * len(solves))()
    check(lib().gp5cu_batch_assign_devices(len(solves), solve_descs(solves), int(ndevices), out))
    return list(out)


class Batch:
    """Independent LHY droplet ground-state solves advanced together (gp5cu_batch_*).

    solves: list of dicts with n, L, N, c3, c4, omega, dt.
    """

    def __init__(self, solves, precision: int = GP5_C128, device: int = 0, devices: Optional[Sequence[int]] = None):
        arr = solve_descs(solves)
        self.solves = [dict(sd) for sd in solves]
        h = C.c_void_p()
        if devices is None:
            check(lib().gp5cu_batch_create(C.byref(h), len(solves), arr, precision, device))
        else:
            devs = (C.c_int * len(devices))(*devices)
            check(lib().gp5cu_batch_create_devices(C.byref(h), len(solves), arr, precision, len(devices), devs))
        self.h = h

    def device(self, k: int) -> int:
        """Device ordinal that runs solve k."""
        return int(lib().gp5cu_batch_device(self.h, k))

    def set_state(self, k: int, psi: np.ndarray) -> None:
        a = np.asfortranarray(np.asarray(psi, dtype=np.complex128).reshape((self.solves[k]["n"],) * 3, order="F"))
        check(lib().gp5cu_batch_set_state(self.h, k, C.c_void_p(_ptr(a))))

    def get_state(self, k: int) -> np.ndarray:
        n = self.solves[k]["n"]
        out = np.empty((n, n, n, 1), dtype=np.complex128, order="F")
        check(lib().gp5cu_batch_get_state(self.h, k, C.c_void_p(_ptr(out))))
        return out

    def set_method(self, method: int, theta: float = 0.5) -> None:
        """GP5_BATCH_RK4 (imaginary-time RK4, the default) or GP5_BATCH_PRECOND (preconditioned
        gradient iteration with step theta) for the following solve calls."""
        check(lib().gp5cu_batch_set_method(self.h, int(method), float(theta)))

    def solve(self, tol: float, check_every: int = 100, max_steps: int = 100000):
        res = (SolveResult * len(self.solves))()
        check(lib().gp5cu_batch_solve(self.h, float(tol), int(check_every), int(max_steps), res))
        return [r.as_dict() for r in res]

    @property
    def launches(self) -> int:
        return int(lib().gp5cu_batch_launches(self.h))

    def close(self):
        if getattr(self, "h", None):
            lib().gp5cu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bf16_round(a: np.ndarray) -> np.ndarray:
    """float32 values rounded to the nearest BF16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


class Mlp:
    """The warm-start MLP (gp5cu_mlp_*): 3 -> 256 -> 256 -> 256 -> 64, GELU hidden layers."""

    IN, HIDDEN, OUT = 3, 256, 64
    SHAPES = [(256, 3), (256, 256), (256, 256), (64, 256)]

    def __init__(self, device: int = 0, seed: int = 0):
        h = C.c_void_p()
        check(lib().gp5cu_mlp_create(C.byref(h), device, int(seed)))
        self.h = h
        self.nparam = int(lib().gp5cu_mlp_num_params(self.h))

    def get_params(self) -> np.ndarray:
        out = np.empty(self.nparam, dtype=np.float32)
        check(lib().gp5cu_mlp_get_params(self.h, C.c_void_p(_ptr(out))))
        return out

    def set_params(self, p: np.ndarray) -> None:
        a = np.ascontiguousarray(p, dtype=np.float32)
        assert a.size == self.nparam
        check(lib().gp5cu_mlp_set_params(self.h, C.c_void_p(_ptr(a))))

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, self.IN)
        y = np.empty((x.shape[0], self.OUT), dtype=np.float32)
        check(lib().gp5cu_mlp_forward(self.h, C.c_void_p(_ptr(x)), x.shape[0], C.c_void_p(_ptr(y))))
        return y

    def gradients(self, x: np.ndarray, t: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, self.IN)
        t = np.ascontiguousarray(t, dtype=np.float32).reshape(-1, self.OUT)
        g = np.empty(self.nparam, dtype=np.float32)
        loss = C.c_double()
        check(lib().gp5cu_mlp_gradients(self.h, C.c_void_p(_ptr(x)), C.c_void_p(_ptr(t)), x.shape[0],
                                        C.c_void_p(_ptr(g)), C.byref(loss)))
        return g, loss.value

    def train(self, x: np.ndarray, t: np.ndarray, epochs: int, batch: int = 256, lr: float = 1e-3,
              seed: int = 0) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, self.IN)
        t = np.ascontiguousarray(t, dtype=np.float32).reshape(-1, self.OUT)
        hist = np.empty(epochs, dtype=np.float32)
        check(lib().gp5cu_mlp_train(self.h, C.c_void_p(_ptr(x)), C.c_void_p(_ptr(t)), x.shape[0], int(epochs),
                                    int(batch), float(lr), int(seed), C.c_void_p(_ptr(hist))))
        return hist

    def set_wait_bound(self, ns: int) -> None:
        """Bound of the GEMMs' per-chunk MMA wait (gp5cu_mlp_set_wait_bound)."""
        check(lib().gp5cu_mlp_set_wait_bound(self.h, int(ns)))

    def close(self):
        if getattr(self, "h", None):
            lib().gp5cu_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gemm_bf16(A_dev: int, sam: int, sak: int, B_dev: int, sbn: int, sbk: int, C_dev: int, ldc: int,
              M: int, N: int, K: int, stream: int = 0) -> None:
    """C = A B^T on device pointers (BF16 operands, FP32 result), see gp5cu_gemm_bf16."""
    check(lib().gp5cu_gemm_bf16(C.c_void_p(A_dev), sam, sak, C.c_void_p(B_dev), sbn, sbk, C.c_void_p(C_dev), ldc,
                                M, N, K, C.c_void_p(stream)))
