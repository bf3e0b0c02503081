"""Python access to the B200 virtual-PE symmetric-memory library.

`Shmem` starts the library (virtual PEs on one GPU) and exposes the host API,
heap access and the host-callable operations; `Batch` drives the batched
request engine; `traffic` holds the seeded workload generators.  Everything
that runs on the GPU goes through libnvshmem_b200.so: the first use of a name
that needs it (Shmem, Batch, BatchConfig, ...) loads the library and fails
with ImportError if it is not built.  The ABI constants and `traffic` do not
load it.
"""
from . import _abi, traffic  # noqa: F401
from ._abi import (CMP_EQ, CMP_GE, CMP_GT, CMP_LE, CMP_LT, CMP_NE, DT_DOUBLE,  # noqa: F401
                   DT_FLOAT, DT_INT, DT_WIDTH, ERR_BOUNDS, ERR_COOP, ERR_CUDA,
                   ERR_INVALID, ERR_NOMEM, ERR_STATE, ERR_TIMEOUT, ERR_UNSUPPORTED, ERRORS_EXIT,
                   ERRORS_RETURN, MODE_BLOCK, MODE_BULK, MODE_THREAD, MODE_WARP, REQ_G, REQ_GET,
                   REQ_P, REQ_PUT, REQ_SIGNAL, REQUEST_COMPACT_DTYPE, REQUEST_DTYPE, SUCCESS,
                   TRACE_DTYPE, PICKED_GROUP_DTYPE, PATTERN_PAIRS, PATTERN_ALLTOALL, PATTERN_NEIGHBOR,
                   PATTERN_RANDOM)

# names backed by the shared library, resolved on first use
_NATIVE = {"LIB_PATH": "_lib", "BatchConfig": "_lib", "ShmemError": "_lib",
           "Batch": "api", "Shmem": "api", "default_batch_config": "api", "requests_bytes": "api",
           "to_compact": "api"}


def __getattr__(name):
    mod = _NATIVE.get(name)
    if mod is None:
        raise AttributeError(f"module 'nvshmem_b200' has no attribute {name!r}")
    import importlib
    value = getattr(importlib.import_module(f".{mod}", __name__), name)
    globals()[name] = value
    return value


__all__ = sorted([n for n in dir() if not n.startswith("_")] + list(_NATIVE))
