"""Structured GLL mesh and its map to the reference's node numbering.

Nodes live on the structured grid (gx, gz), gx in [0, nelx*N], gz in [0, nelz*N].
MUN numbers nodes in first-seen order while sweeping elements ez-major, ex-minor and
local nodes j-major, i-minor (``Bspline_Coupling/SEM/sem_waveform/mesh.py:4-43``);
``node_grid[id] = gz*nxg + gx`` is that permutation, built here without float keys.
"""
import numpy as np

from .gll import gll_points


def create_global_mesh(xmin, xmax, zmin, zmax, nelem_x, nelem_z, npol):
    """Returns (coords (P,2), connectivity (E,(N+1)^2) int64, node_grid (P,) int64)."""
    N = int(npol)
    ng = N + 1
    xi = gll_points(N)
    cx = np.linspace(xmin, xmax, nelem_x + 1)
    cz = np.linspace(zmin, zmax, nelem_z + 1)
    nxg = nelem_x * N + 1
    ez, ex, j, i = np.meshgrid(np.arange(nelem_z), np.arange(nelem_x), np.arange(ng),
                               np.arange(ng), indexing="ij")
    lin = ((ez * N + j) * nxg + (ex * N + i)).reshape(-1)
    uniq, first = np.unique(lin, return_index=True)
    order = np.argsort(first, kind="stable")
    node_grid = uniq[order].astype(np.int64)
    ids = np.empty(nxg * (nelem_z * N + 1), dtype=np.int64)
    ids[node_grid] = np.arange(len(node_grid))
    conn = ids[lin].reshape(nelem_z * nelem_x, ng * ng)
    f = first[order]
    exf, ezf = ex.reshape(-1)[f], ez.reshape(-1)[f]
    a, b = xi[i.reshape(-1)[f]], xi[j.reshape(-1)[f]]
    x = 0.5 * ((1 - a) * cx[exf] + (1 + a) * cx[exf + 1])
    z = 0.5 * ((1 - b) * cz[ezf] + (1 + b) * cz[ezf + 1])
    return np.stack([x, z], axis=1), conn, node_grid


def grid_coords_1d(vmin, vmax, nel, npol):
    """Coordinate of every grid line (same arithmetic as the element sweep)."""
    xi = gll_points(npol)
    c = np.linspace(vmin, vmax, nel + 1)
    out = np.empty(nel * npol + 1)
    for e in range(nel):
        out[e * npol:(e + 1) * npol + 1] = 0.5 * ((1 - xi) * c[e] + (1 + xi) * c[e + 1])
    return out


def find_closest_node(x, z, coords):
    d = np.sqrt((coords[:, 0] - x) ** 2 + (coords[:, 1] - z) ** 2)
    return int(np.argmin(d))
