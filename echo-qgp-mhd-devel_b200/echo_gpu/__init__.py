"""B200 (sm_100a) implementation of ECHO-QGP's per-time-step right-hand side
and update, behind the reference's evolve.f90 / work.f90 interfaces.

The compute lives in ``lib/libechogpu.so`` (CUDA, C-ABI declared in
``include/echo_gpu.h``); this package is the host-side mirror of the
reference interface (``lib.Evolve``), the run-time parameters
(``params``) and the synthetic initial conditions (``initial``).
"""
from . import params  # noqa: F401
from .lib import CrashError, Evolve, load  # noqa: F401
