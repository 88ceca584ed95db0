"""conan_b200 -- B200-native particle-mesh step and initial conditions of conan.

The compute path is libconan_pm.so (CUDA sm_100a, C ABI in include/conan_pm.h);
this package is its Python mirror. Importing it loads the library and fails
loudly if the library has not been built (``python conan_b200/build.py``).
"""
from . import _lib
from ._lib import ConanError

_lib.lib()  # fail at import time if the native library is missing

from .pm import (  # noqa: E402
    Cosmology,
    FoF,
    Gravity,
    LeapFrog,
    cic,
    compute_displacement,
    fof,
    compute_potential,
    generate_random_field,
    ic_params,
    white_noise,
)
from .conanfile import ConanFile  # noqa: E402

__all__ = [
    "ConanError", "ConanFile", "Cosmology", "FoF", "Gravity", "LeapFrog", "cic", "compute_displacement",
    "compute_potential", "fof", "generate_random_field", "ic_params", "white_noise",
]
