"""spd_K on B200: spectral-difference hydro step (ADER / SSP-RK, LLF/HLLC,
NAD + MUSCL-Hancock fallback) as hand-written sm_100a CUDA behind a C ABI.

The compute path is libspdk_cuda.so; this package is its host-side mirror
of the reference driver objects. There is no CPU fallback.
"""
from .api import (HydroSolver, SpdkError, config_from_params, parse_athinput, apply_overrides,
                  load_library, FIELD_U_SP, FIELD_W_CV, FIELD_TROUBLES, FIELD_THETA, EXPORTS)

__all__ = ["HydroSolver", "SpdkError", "config_from_params", "parse_athinput", "apply_overrides",
           "load_library", "FIELD_U_SP", "FIELD_W_CV", "FIELD_TROUBLES", "FIELD_THETA", "EXPORTS"]
