"""oskar_b200: B200 (sm_100a) kernels for OSKAR's interferometer visibility
hot path, behind the C ABI declared in include/oskar_b200.h.

The compute path is liboskar_b200.so (hand-written CUDA). This package only
binds it (``_lib``), builds it (``build``), wraps the OSKAR-named C layer
(``oskar_api``), shards dumps over ranks (``sharding``), drives the learned
station-beam surrogate (``surrogate``) and generates the synthetic workloads
used by the benchmark (``workloads``).
"""
from ._lib import call, load, stream_ptr, OskbError  # noqa: F401

__all__ = ["call", "load", "stream_ptr", "OskbError"]
