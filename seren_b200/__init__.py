"""B200-native force hot path of the SEREN grad-h SPH code.

The product is the CUDA library ``seren_b200/_build/libseren_gpu.so`` with the C
ABI declared in ``include/seren_gpu.h``; ``seren_b200.gpu`` is its ctypes
binding and ``seren_b200.ics`` generates the seeded synthetic workloads.
"""
from .ics import (batched_clouds, h_fac_for, plummer, pp_gather_for,  # noqa: F401
                  protostellar_disc, turbulent_core, uniform_sphere)
