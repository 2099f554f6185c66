"""Test helpers: fixture loading and comparisons (test infrastructure)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ALL = ["x", "y", "z", "p", "q", "r", "dxdt", "dydt", "dzdt", "dpdt", "dqdt", "drdt", "h", "b", "vol",
       "stretch", "tag", "xo", "yo", "zo", "xf", "yf", "zf", "po", "qo", "ro", "pf", "qf", "rf"]


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def geom(d):
    g = d["geom"]
    return int(g[0]), int(g[1]), int(g[2]), float(g[3]), float(g[4]), float(g[5])


def rel(a, b):
    s = np.abs(b).max()
    return np.abs(a - b).max() / (s if s > 0 else 1.0)


def rel_l2(a, b):
    s = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (s if s > 0 else 1.0)


def lattice_parcels(nx, ny, nz, lx, ly, lz, n_per_dir=2):
    """basic_parcelsetup.F90:90-118 (per-cell sub-lattice centres, vol = 1.0),
    in its order: cell x outer, then y, then z; sub-points x outer, z inner."""
    dx, dy, dz = lx / nx, ly / ny, lz / nz
    ii, jj, kk, a, b, c = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), np.arange(n_per_dir),
                                      np.arange(n_per_dir), np.arange(n_per_dir), indexing="ij")
    ddx, ddy, ddz = dx / n_per_dir, dy / n_per_dir, dz / n_per_dir
    x = ii * dx + ddx / 2 + a * ddx
    y = jj * dy + ddy / 2 + b * ddy
    z = kk * dz + ddz / 2 + c * ddz
    n = x.size
    return {"x": x.ravel(), "y": y.ravel(), "z": z.ravel(), "vol": np.ones(n)}
