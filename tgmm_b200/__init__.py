"""B200-native (sm_100a) TGMM supervoxel variational-inference EM.

The CUDA engine (``libtgmm_gmem.so``) implements the per-time-point EM behind the
reference's ``GMEMupdateCUDA`` entry points and a C ABI (``include/tgmm_gmem.h``).
This package holds the Python bindings (``_lib``), the synthetic workload generator
(``synth``), the engine wrapper over device buffers (``engine``) and the batched /
served forms (``serve``).
"""
__all__ = ["_lib", "synth", "engine"]
