"""B200-native force hot path of the SEREN grad-h SPH code.

The product is the CUDA library ``seren_b200/_build/libseren_gpu.so`` with the C
ABI declared in ``include/seren_gpu.h``; ``seren_b200.gpu`` is its ctypes
binding, ``seren_b200.ics`` generates the seeded synthetic workloads and
``seren_b200.snapshot`` reads and writes SEREN binary and DRAGON snapshots.
"""
from .ics import (batched_clouds, h_fac_for, plummer, pp_gather_for,  # noqa: F401
                  protostellar_disc, turbulent_core, uniform_sphere)
from .snapshot import (read_dragon_form, read_dragon_unform, read_seren_unform,  # noqa: F401
                       to_hot_path, write_dragon_form, write_dragon_unform, write_seren_unform)
