"""GLL helpers and the CFL rule (API of MUN ``sem_waveform/utils.py:5-111``)."""
import numpy as np

from ..gll import diff_matrix, gll_points, gll_weights, lagrange_basis  # noqa: F401


def compute_gll_weights(nodes):
    return gll_weights(np.asarray(nodes, dtype=np.float64))


def barycentric_weights(x):
    n = len(x)
    w = np.ones(n)
    for j in range(n):
        for k in range(n):
            if k != j:
                w[j] /= (x[j] - x[k])
    return w


def differentiation_matrix_gll(x):
    return diff_matrix(np.asarray(x, dtype=np.float64))


def check_cfl_condition(velocity_model, dt, npol, dx_elem, dz_elem, vmax):
    """dt_max = 0.35 * (min(dx,dz)/(p+1)) / (max(c) (p+1) sqrt(2)); ValueError on NaN/Inf."""
    v = np.asarray(velocity_model)
    if not np.all(np.isfinite(v)):
        raise ValueError(f"[CFL] velocity_model contains non-finite values (NaN/Inf). "
                         f"Min: {np.nanmin(v):.6f}, Max: {np.nanmax(v):.6f}, "
                         f"NaN count: {np.sum(np.isnan(v))}")
    cmax = float(np.max(v))
    p = npol
    dt_max = 0.35 * (min(dx_elem, dz_elem) / (p + 1)) / (cmax * (p + 1) * np.sqrt(2.0))
    return dt <= dt_max, dt_max


def adjust_time_step_for_stability(velocity_model, current_dt, total_time, npol, dx_elem, dz_elem,
                                   vmax):
    """Lower dt to the CFL limit only if it exceeds it; nt = ceil(T/dt)."""
    stable, dt_limit = check_cfl_condition(velocity_model, current_dt, npol, dx_elem, dz_elem, vmax)
    if not stable:
        new_dt = float(dt_limit)
        return new_dt, int(np.ceil(total_time / new_dt))
    return current_dt, int(np.ceil(total_time / current_dt))
