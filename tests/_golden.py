"""Helpers to load the committed golden vectors (produced by tests/golden/make_golden.py)."""
import os

import numpy as np

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
THEORIES = ["nuclear", "omega", "coulomb", "rho", "berger", "lightly_bound"]


def available():
    return [t for t in THEORIES if os.path.exists(os.path.join(GOLDEN_DIR, f"{t}.npz"))]


def load(theory):
    return dict(np.load(os.path.join(GOLDEN_DIR, f"{theory}.npz")))


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(float(np.max(np.abs(b))), 1e-300)
    return float(np.max(np.abs(a - b))) / scale
