"""Drop-in replacement for MUN's ``sem_waveform`` package, running on a B200.

    from mun_b200.sem_waveform import SEMSimulation          # instead of
    from sem_waveform import SEMSimulation                   # MUN's CPU package
"""
from .core import SEMSimulation, run_forward_and_adjoint_sources

__version__ = "1.0.0"
__all__ = ["SEMSimulation", "run_forward_and_adjoint_sources"]
