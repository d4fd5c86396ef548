"""Observation handling on the host (float64): resampling onto the simulation time
grid (``Bspline_Coupling/SEM/sem_waveform/core.py:109-128``: linear interpolation,
zero outside the observed span) and the CO2 misfit window/decimation
(``CO2_plume/one_stage/single_cubic/sem_waveform/core.py:1441-1467``)."""
import numpy as np


def align_observation(y, src_dt, src_nt, dst_dt, dst_nt):
    y = np.asarray(y, dtype=np.float64)
    if y.ndim == 1:
        y = y[:, None]
    src_t = np.arange(int(src_nt), dtype=np.float64) * float(src_dt)
    dst_t = np.arange(int(dst_nt), dtype=np.float64) * float(dst_dt)
    if y.shape[0] > src_nt:
        y = y[:int(src_nt)]
    if y.shape[0] == dst_nt and np.allclose(src_t[:int(dst_nt)], dst_t, atol=1e-12, rtol=0.0):
        return y
    out = np.zeros((int(dst_nt), y.shape[1]))
    inside = (dst_t >= src_t[0]) & (dst_t <= src_t[-1])
    for r in range(y.shape[1]):
        out[inside, r] = np.interp(dst_t[inside], src_t, y[:, r])
    return out


def misfit_window(mw, dt, nt):
    """(it0, it1, decim) from a ``method.misfit_window`` dict (None/disabled = all)."""
    if not (mw and mw.get("enabled", False)):
        return 0, int(nt), 1
    tmin = mw.get("tmin", 0.0)
    tmin = float(tmin) if tmin is not None else 0.0
    tmax = mw.get("tmax", None)
    if tmax is None and mw.get("window_len", None) is not None:
        tmax = tmin + float(mw["window_len"])
    tmax = float(tmax) if tmax is not None else float(dt * (nt - 1))
    if tmax <= tmin:
        raise ValueError(f"misfit_window invalid: tmax({tmax}) <= tmin({tmin})")
    decim = max(1, int(mw.get("decim", 1)))
    it0 = max(0, min(int(round(tmin / dt)), nt - 1))
    it1 = max(it0 + 1, min(int(round(tmax / dt)) + 1, nt))
    return it0, it1, decim
