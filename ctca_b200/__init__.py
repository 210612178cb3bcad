"""ctca_b200: the EMSES (MPIEMSES3D) particle hot path on B200 (sm_100a).

The compute lives in libemsesg.so (CUDA kernels + C ABI, include/emses_gpu.h);
this package holds its host-side mirror of the reference's subroutines
(emses.py), seeded synthetic inputs (inputs.py) and the build (build.py).
"""
from .emses import (PARTICLE_DTYPE, Config, Counter, Emses, EmsesError, Plasma, field_shape,  # noqa: F401
                    load_library)

__all__ = ["Emses", "EmsesError", "Config", "Counter", "Plasma", "PARTICLE_DTYPE", "field_shape", "load_library"]
