"""B200 continuum-dislocation-dynamics time step: torch-facing API over libcdd.so.

``Plan`` / ``Instance`` wrap the C ABI in include/cdd.h; ``gaussian_random_field`` builds the
seeded initial conditions the workloads are defined on.
"""
from ._lib import CDDError, load as load_library
from .engine import Instance, Plan, stress_to_tensor9
from .initial import gaussian_random_field
from .pipeline import HostPipeline

__all__ = ["CDDError", "HostPipeline", "Instance", "Plan", "gaussian_random_field", "load_library",
           "stress_to_tensor9"]
