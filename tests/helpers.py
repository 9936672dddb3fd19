"""Shared test helpers: seeded problems built with the oracle and the product."""
import numpy as np

from fhs_b200 import synth


def coverage(M, seed, edge_fraction=0.1):
    """Gaussian (v, u) coverage plus a share of uniform points near +-pi
    (exercises the grid wrap-around)."""
    om_y, om_x = synth.base_coverage(M, seed)
    rng = np.random.default_rng(seed + 5)
    k = int(edge_fraction * M)
    if k:
        om_y[:k] = rng.uniform(-np.pi, np.pi, k)
        om_x[:k] = rng.uniform(-np.pi, np.pi, k)
    return om_y, om_x


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
