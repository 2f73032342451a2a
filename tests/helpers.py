"""Shared test helpers: golden fixtures and oracle configurations."""
import os

import numpy as np

from oracle import mc3d_oracle as O
from tests.golden import gen_golden as G

HERE = os.path.dirname(os.path.abspath(__file__))


def golden_ops():
    return np.load(os.path.join(HERE, "golden", "ops.npz"))


def golden_steps():
    return np.load(os.path.join(HERE, "golden", "steps.npz"))


def golden_relax():
    return np.load(os.path.join(HERE, "golden", "sponge_relax.npz"))


def golden_metrics():
    return np.load(os.path.join(HERE, "golden", "metrics.npz"))


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def rel_max(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def oracle_config(name):
    grid, kw, n, seed = G.STEP_CASES[name]
    return O.Config(N=grid, mu_ref=G.MU_REF, **kw), G.step_ic(grid, seed), n
