"""Sponge set-up (API of MUN ``sem_waveform/boundary.py:5-58``): cubic ramp on all four
sides, d0 = -(m+1) c_max ln R / (2 delta), decay = exp(-sigma dt)."""
import numpy as np
import torch


def setup_pml(xmin, xmax, zmin, zmax, pml_thickness_m, global_coords, dt, R=1e-8, c_max=None):
    if c_max is None:
        raise ValueError("c_max must be provided from config")
    m = 3
    d = float(pml_thickness_m)
    d0 = -(m + 1) * float(c_max) * np.log(R) / (2.0 * d)
    x, z = global_coords[:, 0], global_coords[:, 1]
    sx = np.zeros(len(global_coords))
    sz = np.zeros(len(global_coords))
    lo, hi = x < xmin + d, x > xmax - d
    sx[lo] = d0 * ((xmin + d - x[lo]) / d) ** m
    sx[hi] = d0 * ((x[hi] - (xmax - d)) / d) ** m
    lo, hi = z < zmin + d, z > zmax - d
    sz[lo] = d0 * ((zmin + d - z[lo]) / d) ** m
    sz[hi] = d0 * ((z[hi] - (zmax - d)) / d) ** m
    sig = sx + sz
    mask = sig > 0.0
    return torch.where(torch.from_numpy(mask))[0], mask, torch.from_numpy(np.exp(-sig * dt))
