"""B200-native (sm_100a) spectral-element acoustic solver with adjoint gradient.

Drop-in for MUN's ``sem_waveform`` package: ``mun_b200.sem_waveform.SEMSimulation``
keeps the reference call surface; underneath, PyTorch host code drives hand-written
CUDA kernels through the C ABI declared in ``include/mun_sem.h``.
"""
from .plan import SEMPlan, build_plan_arrays  # noqa: F401
from .solver import Batch, SolveSpec, forward, forward_adjoint  # noqa: F401

__all__ = ["SEMPlan", "build_plan_arrays", "Batch", "SolveSpec", "forward", "forward_adjoint"]
