"""Source wavelet (API of MUN ``sem_waveform/sources.py:3-21``)."""
import numpy as np

from ..plan import ricker_source


def ricker_wavelet(t, f0=20.0, t0=0.1):
    return (1.0 - 2.0 * (np.pi * f0 * (t - t0)) ** 2) * np.exp(-(np.pi * f0 * (t - t0)) ** 2)


def create_source_wavelet(nt, dt, f0=20.0, t0=0.1, gate_time=0.3, amp=1.0):
    return ricker_source(nt, dt, f0, amp, t0=t0, gate=gate_time)
