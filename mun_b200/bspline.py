"""Clamped uniform cubic tensor-product B-spline node grid (the velocity
parametrisation of the batched/serving workloads: v = v_base + B theta).

This grid has no counterpart in MUN (whose "B-spline nodes" are the control points of
a closed interface curve); it is the linear parametrisation the batched workloads
use, with dL/dtheta = B^T dL/dv."""
import numpy as np


def clamped_knots(n_ctrl, degree=3):
    inner = np.linspace(0.0, 1.0, n_ctrl - degree + 1)
    return np.concatenate([np.zeros(degree), inner, np.ones(degree)])


def basis_1d(u, n_ctrl, degree=3):
    """(len(u), n_ctrl) basis values by Cox-de Boor; u in [0,1], right end inclusive."""
    u = np.clip(np.asarray(u, dtype=np.float64), 0.0, 1.0)
    t = clamped_knots(n_ctrl, degree)
    m = len(t) - 1
    B = np.zeros((len(u), m))
    for i in range(m):
        B[:, i] = (t[i] <= u) & (u < t[i + 1])
    last = np.nonzero(t < 1.0)[0][-1]
    B[u >= 1.0, :] = 0.0
    B[u >= 1.0, last] = 1.0
    for k in range(1, degree + 1):
        Bn = np.zeros((len(u), m - k))
        for i in range(m - k):
            a = t[i + k] - t[i]
            b = t[i + k + 1] - t[i + 1]
            if a > 0:
                Bn[:, i] += (u - t[i]) / a * B[:, i]
            if b > 0:
                Bn[:, i] += (t[i + k + 1] - u) / b * B[:, i + 1]
        B = Bn
    return B[:, :n_ctrl]


def grid_basis(coords, xlim, zlim, nx, nz):
    """Dense (P, nx*nz) tensor basis at node coordinates, theta index = iz*nx + ix."""
    ux = (coords[:, 0] - xlim[0]) / (xlim[1] - xlim[0])
    uz = (coords[:, 1] - zlim[0]) / (zlim[1] - zlim[0])
    Bx = basis_1d(ux, nx)
    Bz = basis_1d(uz, nz)
    return (Bz[:, :, None] * Bx[:, None, :]).reshape(len(coords), nz * nx)


def layered_velocity(z, interfaces, velocities):
    """Horizontally layered background (layered velocity.py:187-219: searchsorted right)."""
    idx = np.searchsorted(np.asarray(interfaces, dtype=np.float64), z, side="right")
    return np.asarray(velocities, dtype=np.float64)[idx]
