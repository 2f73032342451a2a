"""Meshes of BASELINE's configurations (the role of the reference's
AbstractSingleBlockMesh::getMesh subclasses, e.g.
src/AlgebraicSingleBlockMesh.hpp:210-266 for its cylinder), as (x, y, z)
arrays shaped (Nz, Ny, Nx), x fastest, for CurvilinearCSolver.set_mesh."""
from __future__ import annotations

import math

import numpy as np


def cylinder_ogrid(Nx: int, Ny: int, Nz: int, r0: float = 0.5, r1: float = 30.0, span: float = 2.0):
    """O-grid around a circular cylinder of radius r0: Nx azimuthal points
    (periodic, running clockwise so that the (theta, r, z) frame is
    right-handed and J > 0), Ny radial points spaced geometrically from r0 to
    r1 (ratio (r1/r0)^(1/(Ny-1))), Nz spanwise points (periodic, length span).
    Returns (x, y, z, ratio)."""
    ratio = (r1 / r0) ** (1.0 / (Ny - 1))
    th = 2 * math.pi * np.arange(Nx) / Nx
    r = r0 * ratio ** np.arange(Ny)
    zz = span * np.arange(Nz) / Nz
    Z, Rr, TH = np.meshgrid(zz, r, th, indexing="ij")
    return Rr * np.cos(TH), -Rr * np.sin(TH), Z, ratio


def cylinder_flow_ic(shape, mach: float = 0.2, perturb: float = 0.01, seed: int = 3, gamma: float = 1.4):
    """Uniform flow along x at Mach `mach` (rho = 1, p = 1/gamma, c = 1) with a
    seeded relative velocity perturbation: (rho, U, V, W, p)."""
    rng = np.random.default_rng(seed)
    return [np.ones(shape), mach * (1 + perturb * rng.standard_normal(shape)),
            mach * perturb * rng.standard_normal(shape), mach * perturb * rng.standard_normal(shape),
            np.full(shape, 1 / gamma)]
