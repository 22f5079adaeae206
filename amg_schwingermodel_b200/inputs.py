"""Seeded synthetic inputs for the Schwinger-model solve.

Gauge links are U_mu(n) = exp(i theta_mu(n)) with theta i.i.d. N(0, 1/beta); sources are
complex Gaussian (re, im ~ N(0, 1)) on both spin components.  Arrays use the reference's
site order n = x*Nt + t (src/variables.cpp:10-16) and its [N][2] layout: U[n][mu] with
mu = 0 the time direction and mu = 1 the space direction (include/boundary.h:29-31),
psi[n][spin].  The reference itself draws uniform angles with libc rand()
(src/gauge_conf.cpp:3-8); Gaussian angles at a given beta are the workload definition
used here instead, and the same arrays are what the CPU oracle receives.
"""
from __future__ import annotations

import numpy as np


def gauge_field(nx: int, nt: int, beta: float, seed: int) -> np.ndarray:
    """U[N][2] complex128, theta_mu(n) ~ N(0, 1/beta)."""
    rng = np.random.default_rng(seed)
    theta = rng.normal(0.0, 1.0 / np.sqrt(beta), size=(nx * nt, 2))
    return np.exp(1j * theta)


def gauge_angles(nx: int, nt: int, beta: float, seed: int) -> np.ndarray:
    """theta[N][2] float64 with the same draw as gauge_field (U = exp(i theta))."""
    rng = np.random.default_rng(seed)
    return rng.normal(0.0, 1.0 / np.sqrt(beta), size=(nx * nt, 2))


def gaussian_spinor(nsites: int, dof: int, seed: int, nrhs: int | None = None) -> np.ndarray:
    """Complex-Gaussian vector(s): [N][dof] or [nrhs][N][dof] complex128."""
    rng = np.random.default_rng(seed)
    shape = (nsites, dof) if nrhs is None else (nrhs, nsites, dof)
    return rng.normal(size=shape) + 1j * rng.normal(size=shape)
