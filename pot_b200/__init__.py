"""pot_b200 -- pot's per-timestep particle loop on one B200 (sm_100a).

``pot_b200.gpu`` binds the C ABI of ``libpotgpu.so`` (include/pot_gpu.h);
``pot_b200.configs`` holds the synthetic plasma configurations;
``pot_b200.build`` compiles the CUDA sources in-tree.
"""
from .gpu import (DUST, ELECTRON, ION, PARTICLE_DTYPE, PotError, Run, RunConfig, header_symbols,  # noqa: F401
                  load_library)
