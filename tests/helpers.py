"""Shared helpers of the test suite."""
import numpy as np

# (group, (Lx, Ly, Lz, Lt), ndims): SU(2) in d = 2, 3, 4 and U(1) in d = 2, 4
GEOMS = [
    (0, (4, 4, 4, 4), 4),
    (0, (4, 2, 2, 6), 4),
    (0, (6, 1, 1, 4), 2),
    (0, (4, 6, 1, 4), 3),
    (1, (4, 4, 4, 4), 4),
    (1, (8, 1, 1, 6), 2),
]
GEOM_IDS = [f"{'su2' if g == 0 else 'u1'}-{'x'.join(map(str, d))}-d{nd}" for g, d, nd in GEOMS]


def rel(a, b):
    """Norm-wise relative difference |a - b| / |b|."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def group_name(g):
    return "su2" if g == 0 else "u1"
