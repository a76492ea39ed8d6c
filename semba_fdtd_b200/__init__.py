"""semba_fdtd_b200 -- B200 (sm_100a) implementation of semba-fdtd's Yee
leapfrog core (E/H curl updates, CPML, electric pole-residue ADE, plane-wave
TF/SF, nodal sources, point probes) behind a C ABI (include/semba_gpu.h).

The compute path is libsemba_gpu.so (CUDA); the Python package reads cases,
drives the library and hosts the batched and served forms.
"""
from .case import Problem, read_case  # noqa: F401
from .solver import Solver  # noqa: F401

__all__ = ["Problem", "read_case", "Solver"]
