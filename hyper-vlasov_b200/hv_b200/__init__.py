"""hv_b200: B200-native (sm_100a) hyper-vlasov step behind a C ABI.

The compute lives in lib/libhv_b200.so (hand-written CUDA kernels); this
package is the Python side of its C ABI (include/hv_b200.h).
"""
from . import _lib
from ._lib import (HV_DEPOSIT_ATOMIC, HV_DEPOSIT_SORTED, HV_F32, HV_F64, HV_FIELD_COULOMB, HV_FIELD_DENSITY,
                   HV_FIELD_DENSITY_RAW, HV_FIELD_FORCE_X, HV_FIELD_FORCE_Y, HV_FIELD_FORCE_Z,
                   HV_FIELD_POTENTIAL, HV_PATH_FUSED, HV_PATH_PLAIN, HV_RNG_LIBC, HV_RNG_PHILOX, HV_SOR_EXCHANGE_AUTO, HV_SOR_EXCHANGE_FLAGS,
                   HV_SOR_MAX_UPDATE, HV_SOR_REL_RESIDUAL, HV_WARM_EXTRAPOLATE, HV_WARM_PREVIOUS, HV_WARM_QUADRATIC, OBS_DTYPE,
                   HVError, load)
from .api import Session, generate_nucleus, simulate, simulate_release, workload_particles
from .workloads import CA40_SMALL, PB208_2M, PB208_20K_128, PB208_104K, WORKLOADS, Workload

__all__ = [
    "HV_DEPOSIT_ATOMIC", "HV_DEPOSIT_SORTED", "HV_F32", "HV_F64", "HV_FIELD_COULOMB", "HV_FIELD_DENSITY",
    "HV_FIELD_DENSITY_RAW", "HV_FIELD_FORCE_X", "HV_FIELD_FORCE_Y", "HV_FIELD_FORCE_Z",
    "HV_FIELD_POTENTIAL", "HV_PATH_FUSED", "HV_PATH_PLAIN", "HV_RNG_LIBC", "HV_RNG_PHILOX", "HV_SOR_EXCHANGE_AUTO", "HV_SOR_EXCHANGE_FLAGS",
    "HV_SOR_MAX_UPDATE", "HV_SOR_REL_RESIDUAL", "HV_WARM_EXTRAPOLATE", "HV_WARM_PREVIOUS", "HV_WARM_QUADRATIC", "OBS_DTYPE", "HVError", "load", "Session",
    "generate_nucleus", "simulate", "simulate_release", "workload_particles", "CA40_SMALL", "PB208_2M", "PB208_20K_128", "PB208_104K",
    "WORKLOADS", "Workload", "_lib",
]
