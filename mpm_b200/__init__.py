"""mpm_b200 -- B200-native MPM snow step behind the reference's solver API.

The compute path is the sm_100a shared library ``libmpm_b200.so`` (C ABI in
``include/mpm_b200.h``); this package is its Python binding.
"""
from ._abi import (BOUNDARY_REFERENCE, BOUNDARY_STICKY, FIELD_B, FIELD_DET_FE, FIELD_DET_FP, FIELD_FE, FIELD_FP,
                   FIELD_MASS, FIELD_POSITION, FIELD_POSITION4, FIELD_VELOCITY, FIELD_VOLUME0, GRID_FORCE,
                   GRID_MASS, GRID_VELOCITY, GRID_VELOCITY_STAR, INTERP_CUBIC, INTERP_LINEAR, INTERP_QUADRATIC,
                   MODEL_FIXED_COROTATED, MODEL_NEO_HOOKEAN, TRANSFER_APIC, TRANSFER_PIC_FLIP,
                   VOLUME_GRID_ESTIMATE, VOLUME_PRESCRIBED, MPMError)
from .solver import (APICMPMSolver3D, ConstitutiveModel, InterpolationType, Material, MPMSolver3D, Particles,
                     scene_desc)

__all__ = ["MPMSolver3D", "APICMPMSolver3D", "Particles", "Material", "InterpolationType", "ConstitutiveModel",
           "scene_desc", "MPMError"]
