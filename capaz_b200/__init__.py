"""capaz_b200 — Blackwell-native (sm_100a) CAPAZ multiphase-filtration time step.

The compute path is libcapaz_b200.so (C ABI in include/capaz_b200.h, CUDA
kernels for sm_100a).  This package holds its Python bindings, the
defines.ini helpers and the benchmark workload generators.
"""
from .native import FIELDS, CapazError, Params, load  # noqa: F401
from .simulation import Adjoint, Ensemble, Simulation, default_params, params_from_ini, write_ini  # noqa: F401
