"""Mesh API of MUN ``sem_waveform/mesh.py:4-54`` on top of the structured grid."""
from collections.abc import Mapping

import numpy as np

from ..mesh import create_global_mesh as _structured
from ..mesh import find_closest_node as _closest


class NodeMap(Mapping):
    """{(round(x,6), round(z,6)): node id}, built on first use (the reference returns
    this dict; for large meshes it is rarely needed, so it is lazy)."""

    def __init__(self, coords, node_grid):
        self._coords = coords
        self.node_grid = node_grid
        self._d = None

    def _dict(self):
        if self._d is None:
            self._d = {(round(float(x), 6), round(float(z), 6)): i
                       for i, (x, z) in enumerate(self._coords)}
        return self._d

    def __getitem__(self, k):
        return self._dict()[k]

    def __iter__(self):
        return iter(self._dict())

    def __len__(self):
        return len(self._coords)


def create_global_mesh(xmin, xmax, zmin, zmax, nelem_x, nelem_z, npol):
    """(global_coords (P,2), global_connectivity (E,(N+1)^2), node_map)."""
    coords, conn, node_grid = _structured(xmin, xmax, zmin, zmax, nelem_x, nelem_z, npol)
    return coords, conn, NodeMap(coords, node_grid)


def find_closest_node(x, z, global_coords, tol=1e-6):
    return _closest(x, z, np.asarray(global_coords))
