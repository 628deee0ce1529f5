"""B200-native Metropolis sweep / parallel-tempering engine.

A drop-in for the CPU sweep of EldosZhupanov/ising_engine (src/solver/engine.rs
``step`` driven by src/solver/ultimate.rs ``UltimateSolver``): hand-written CUDA
for sm_100a behind a C ABI (include/ising_b200.h), with thin Python bindings.
"""
from .core import CsrMatrix, QuboModel
from .engine import BatchEngine, Engine, geometric_temps, suggested_temp_range

__all__ = ["CsrMatrix", "QuboModel", "Engine", "BatchEngine", "geometric_temps",
           "suggested_temp_range"]
