"""B200-native (sm_100a) backend of the Tetsuhiro-WOS propagation hot path.

The compute lives in libwosgpu.so (hand-written CUDA behind the C ABI in
include/wos_gpu.h); this package is its Python host binding, named after the
reference's Go `optics` API.  Import it with
    importlib.import_module("tetsuhiro-wos_b200")
"""
from .wosgpu import (EXPORTS, FP32, FP64, GPU, METHODS, WARN_CODES, CContext, CDiag, CField,  # noqa: F401
                     Context, Field, IndexDesc, WosError, backend_info, comm_unique_id, device_count, lib, LIB_PATH,
                     shard_range)
from .build import build  # noqa: F401
