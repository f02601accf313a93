"""shearwave_b200: the shear_fdtd hot path of pinton-lab/shearwave on NVIDIA B200.

Drop-in replacements for the reference's solver and strain functions
(src/shearwave/__init__.py:21-32) backed by hand-written sm_100a CUDA kernels
behind the C ABI in include/shearwave_b200.h.  Importing the package does not
touch the GPU; the first call loads ``_lib/libshearwave_b200.so`` and fails
loudly if it is missing or no CUDA device is present.
"""

from .solver import (
    divergence_center,
    elastic_solve_static,
    gradient_center,
    hann1d,
    laplacian_center,
    project_body_force_to_shear,
    project_vector_field,
    shear_fdtd,
    shear_fdtd_batch,
    shear_fdtd_jax,
)
from .radiation import compute_radiation_force, compute_radiation_force_velocity
from .strain import compute_strain_fields, compute_strain_invariants, compute_strain_tensor

__version__ = "0.1.0"

__all__ = [
    "__version__",
    "compute_radiation_force",
    "compute_radiation_force_velocity",
    "compute_strain_fields",
    "compute_strain_invariants",
    "compute_strain_tensor",
    "divergence_center",
    "elastic_solve_static",
    "gradient_center",
    "hann1d",
    "laplacian_center",
    "project_body_force_to_shear",
    "project_vector_field",
    "shear_fdtd",
    "shear_fdtd_batch",
    "shear_fdtd_jax",
]
