"""Python access to the B200 virtual-PE symmetric-memory library.

`Shmem` starts the library (virtual PEs on one GPU) and exposes the host API,
heap access and the host-callable operations; `Batch` drives the batched
request engine; `traffic` holds the seeded workload generators.  Everything
runs through libnvshmem_b200.so: importing this package fails if it is not
built.
"""
from . import _lib, traffic
from ._lib import (CMP_EQ, CMP_GE, CMP_GT, CMP_LE, CMP_LT, CMP_NE, DT_DOUBLE,
                   DT_FLOAT, DT_INT, DT_WIDTH, ERR_BOUNDS, ERR_COOP, ERR_CUDA,
                   ERR_INVALID, ERR_NOMEM, ERR_STATE, ERR_TIMEOUT, ERRORS_EXIT,
                   ERRORS_RETURN, LIB_PATH, MODE_BLOCK, MODE_BULK, MODE_THREAD,
                   MODE_WARP, REQ_G, REQ_GET, REQ_P, REQ_PUT, REQ_SIGNAL,
                   REQUEST_COMPACT_DTYPE, REQUEST_DTYPE, SUCCESS, TRACE_DTYPE, BatchConfig,
                   ShmemError)
from .api import Batch, Shmem, default_batch_config, requests_bytes, to_compact

__all__ = [n for n in dir() if not n.startswith("__")]
