"""Generates the golden fixtures in this folder from the CPU oracle (seeded inputs).

The reference (lucaparisi91/GP5) cannot be built or imported here (Eigen Tensor, FFTW3,
MPI and yaml-cpp are absent), so its known answers are carried by the oracle, which
tests/test_oracle.py pins against the reference's own analytic tests.  Transforms are
taken from the long-double direct DFT (oracle/dft_ld.c).

Run:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import dft3_ld  # noqa: E402
from oracle import gp_oracle as o  # noqa: E402


def rand_field(shape, seed, ncomp=1):
    rng = np.random.default_rng(seed)
    s = tuple(shape) + (ncomp,)
    return np.asfortranarray(rng.uniform(-1, 1, s) + 1j * rng.uniform(-1, 1, s))


def main():
    # 1. mixed-radix transform (shared-memory engine on every axis)
    a = rand_field((6, 10, 12), 11)
    np.savez_compressed(os.path.join(HERE, "fft_6x10x12.npz"), a=a, fwd=dft3_ld(a, -1), bwd=dft3_ld(a, 1))
    # 2. power-of-two x (register engine) with short strided axes
    b = rand_field((32, 64, 8), 12)
    np.savez_compressed(os.path.join(HERE, "fft_32x64x8.npz"), a=b, fwd=dft3_ld(b, -1))
    # 3. LHY H applied to a seeded droplet-like state
    geo = o.Geometry((16, 12, 10), (-6, -5, -4), (6, 5, 4))
    psi = o.gaussian_with_noise(geo, 2.0, 1e-2, seed=13, N=30.0, phase_noise=True)
    np.savez_compressed(os.path.join(HERE, "lhy_H_16x12x10.npz"), psi=psi,
                        H=o.Functional("lhy").apply(psi, geo),
                        left=geo.left, right=geo.right)
    # 4. GP with harmonic trap: one imaginary-time RK4 step, one real-time Euler step
    geo = o.Geometry((12, 10, 8), (-5,) * 3, (5,) * 3)
    psi = o.gaussian_with_noise(geo, 1.0, 1e-3, seed=14, N=1.0)
    f = o.Functional("gp", couplings=[[1.0]], V=o.harmonic_potential(geo, [(1, 1, 1)]))
    rk = o.Stepper(f, geo, 1e-3, "RK4", True).advance(psi.copy(), 1)
    eu = o.Stepper(f, geo, 1e-3, "eulero", False).advance(psi.copy(), 1)
    np.savez_compressed(os.path.join(HERE, "gp_steps_12x10x8.npz"), psi=psi, rk4_imag=rk, euler_real=eu,
                        left=geo.left, right=geo.right)
    # 5. LHY, RK4 imaginary time with in-stepper renormalisation (N = 25), 3 steps
    geo = o.Geometry((10, 12, 14), (-5, -6, -7), (5, 6, 7))
    psi = o.gaussian_with_noise(geo, 1.5, 1e-3, seed=15, N=25.0, phase_noise=True)
    st = o.Stepper(o.Functional("lhy"), geo, 2e-3, "RK4", True, normalizations=[25.0])
    out = st.advance(psi.copy(), 3)
    np.savez_compressed(os.path.join(HERE, "lhy_rk4_renorm_10x12x14.npz"), psi=psi, out=out,
                        left=geo.left, right=geo.right)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
