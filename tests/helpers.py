"""Field builders shared by the tests (numpy, float64, ghost-shaped)."""

import numpy as np

GOLDEN = __import__("os").path.join(__import__("os").path.dirname(__file__), "golden")


def load_golden(name):
    import os

    return np.load(os.path.join(GOLDEN, name))


def positions(comp, nx, ny, dx, dy, z_f, z_c):
    """Physical (X, Y, Z) of every entry of the ghost-shaped array of `comp`
    (u at x-faces, v at y-faces, w at z-faces, one ghost layer per side)."""
    if comp == "u":
        X = (np.arange(0, nx + 1) * dx)[:, None, None]
        Y = ((np.arange(0, ny + 2) - 0.5) * dy)[None, :, None]
        Z = np.asarray(z_c)[None, None, :]
    elif comp == "v":
        X = ((np.arange(0, nx + 2) - 0.5) * dx)[:, None, None]
        Y = (np.arange(0, ny + 1) * dy)[None, :, None]
        Z = np.asarray(z_c)[None, None, :]
    elif comp == "w":
        X = ((np.arange(0, nx + 2) - 0.5) * dx)[:, None, None]
        Y = ((np.arange(0, ny + 2) - 0.5) * dy)[None, :, None]
        Z = np.asarray(z_f)[None, None, :]
    else:
        raise ValueError(comp)
    return X, Y, Z


def shape_of(comp, nx, ny, nz):
    return {"u": (nx + 1, ny + 2, nz + 2), "v": (nx + 2, ny + 1, nz + 2),
            "w": (nx + 2, ny + 2, nz + 1)}[comp]


def make_field(comp, fn, nx, ny, nz, dx, dy, z_f, z_c):
    """Ghost-shaped array of `comp` filled with fn(X, Y, Z) everywhere."""
    X, Y, Z = positions(comp, nx, ny, dx, dy, z_f, z_c)
    return np.ascontiguousarray(fn(X, Y, Z) * np.ones(shape_of(comp, nx, ny, nz)))


def interior(comp, a, nx, ny, nz):
    if comp == "w":
        return a[1 : nx + 1, 1 : ny + 1, 1:nz]
    return a[1 : nx + 1, 1 : ny + 1, 1 : nz + 1]


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.abs(b).max()
    scale = scale if scale > 0 else 1.0
    return float(np.abs(a - b).max() / scale)
