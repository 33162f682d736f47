"""B200 (sm_100a) implementation of the GENESIS per-tick particle hot path.

The compute path is ``libgenesis_gpu.so`` (CUDA C++ for sm_100a behind the C
ABI in include/genesis_gpu.h).  This package holds its ctypes binding
(:mod:`genesis_b200._lib`), the host-side mirror of the reference's systems
(:mod:`genesis_b200.systems`), the TOML config reader and the synthetic
workload generator.
"""
from . import elements  # noqa: F401
from .config import Config, ConfigError, default_config, from_file, from_toml  # noqa: F401

__all__ = ["Config", "ConfigError", "default_config", "from_file", "from_toml"]
