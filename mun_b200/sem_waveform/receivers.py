"""Receiver interpolation (API of MUN ``sem_waveform/receivers.py:6-108`` and the
layered package's ``_setup_receivers_from_positions``, ``core.py:90-172``)."""
import numpy as np
import scipy.sparse as sp
import torch

from ..gll import gll_points, lagrange_basis


def circle_positions(src_x, src_z, radius, n):
    ang = np.linspace(0, 2 * np.pi, int(n), endpoint=False)
    return np.stack([src_x + radius * np.cos(ang), src_z + radius * np.sin(ang)], axis=1)


def receiver_matrix(positions, xmin, zmin, dx, dz, nelx, nelz, conn, npol, npoints):
    """(R scipy CSR (nrec, P), R torch sparse COO) with weights l_i(xi) l_j(eta)."""
    nodes = gll_points(npol)
    ng = npol + 1
    rows, cols, vals = [], [], []
    for r, (rx, rz) in enumerate(np.asarray(positions, dtype=np.float64).reshape(-1, 2)):
        ex = min(max(int((rx - xmin) / dx), 0), nelx - 1)
        ez = min(max(int((rz - zmin) / dz), 0), nelz - 1)
        xi = 2.0 * (rx - (xmin + ex * dx)) / dx - 1.0
        eta = 2.0 * (rz - (zmin + ez * dz)) / dz - 1.0
        e = ez * nelx + ex
        for j in range(ng):
            lz = float(lagrange_basis(eta, j, nodes))
            for i in range(ng):
                rows.append(r)
                cols.append(int(conn[e][j * ng + i]))
                vals.append(float(lagrange_basis(xi, i, nodes)) * lz)
    R = sp.csr_matrix((vals, (rows, cols)), shape=(len(np.atleast_2d(positions)), npoints))
    coo = R.tocoo()
    Rt = torch.sparse_coo_tensor(torch.from_numpy(np.vstack([coo.row, coo.col]).astype(np.int64)),
                                 torch.from_numpy(coo.data), coo.shape, dtype=torch.float64).coalesce()
    return R, Rt


def setup_receivers(src_x, src_z, receiver_radius, num_receivers, xmin, zmin, dx_elem, dz_elem,
                    nelem_x, nelem_z, global_connectivity, global_coords, npol):
    pos = circle_positions(src_x, src_z, receiver_radius, num_receivers)
    R, Rt = receiver_matrix(pos, xmin, zmin, dx_elem, dz_elem, nelem_x, nelem_z,
                            global_connectivity, npol, len(global_coords))
    info = []
    for r, p in enumerate(pos):
        row = R.getrow(r)
        info.append({"node_indices": row.indices, "weights": row.data, "global_coords": tuple(p)})
    return [tuple(p) for p in pos], info, R, Rt
