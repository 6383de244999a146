"""B200-native DEM contact step (Hertz-Mindlin, walls, bonded DEM) behind a C ABI.

The compute path is libb200dem.so (CUDA C++ for sm_100a, built from csrc/); this
package holds its ctypes binding (_lib), a Python mirror of the reference's
Particles / Wall / Force / Integrator / SolverDEM interface (api), the reference's
array-layout state containers (state), its JSON input reader (inputs) and seeded
scenario builders (scenarios).
"""
from . import inputs, scenarios, state  # noqa: F401

__all__ = ["api", "inputs", "scenarios", "state"]

