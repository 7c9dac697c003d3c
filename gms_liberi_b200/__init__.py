"""B200-native RHF Fock-build engine with libERI's handle API.

The compute path is the CUDA library ``_build/libliberi_b200.so`` (sm_100a),
reached through ``gms_liberi_b200.liberi`` (ctypes over include/liberi_b200.h).
"""
from . import molecules  # noqa: F401
