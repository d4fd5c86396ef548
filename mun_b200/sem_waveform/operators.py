"""Element operators (API of MUN ``sem_waveform/operators.py:6-84``).  The solver does
not assemble them — the kernels apply the equivalent 1-D line operators — but they are
kept for callers that inspect them."""
import numpy as np

from ..gll import diff_matrix, gll_points, gll_weights, lagrange_basis


def precompute_sem_operators(dx_elem, dz_elem, npol):
    nodes = gll_points(npol)
    w = gll_weights(nodes)
    D = diff_matrix(nodes)
    ng = npol + 1
    L = np.array([[float(lagrange_basis(nodes[j], n, nodes)) for n in range(ng)] for j in range(ng)])
    J = (dx_elem * dz_elem) * 0.25
    Gx = (2.0 / dx_elem) * np.kron(L, D)
    Gz = (2.0 / dz_elem) * np.kron(D, L)
    S = np.kron(L, L)
    w2D = ((w[:, None] * w[None, :]) * J).reshape(-1)
    return Gx, Gz, S, w2D


def assemble_mass_matrix_lumped_torch(global_connectivity, dx_elem, dz_elem, npol, npoints):
    import torch
    w = gll_weights(gll_points(npol))
    J = (dx_elem / 2.0) * (dz_elem / 2.0)
    conn = np.asarray(global_connectivity, dtype=np.int64)
    wl = (w[None, :] * w[:, None]).reshape(-1) * J
    M = np.zeros(npoints)
    np.add.at(M, conn.reshape(-1), np.tile(wl, conn.shape[0]))
    return torch.from_numpy(M)
