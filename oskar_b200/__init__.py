"""oskar_b200: B200 (sm_100a) kernels for OSKAR's interferometer visibility
hot path, behind the C ABI declared in include/oskar_b200.h.

The compute path is liboskar_b200.so (hand-written CUDA). This package only
binds it (``_lib``), builds it (``build``), provides the host-side mirror of
the reference's per-block driver (``interferometer``) and the synthetic
workloads used by the benchmark (``workloads``).
"""
from ._lib import call, load, stream_ptr, OskbError  # noqa: F401

__all__ = ["call", "load", "stream_ptr", "OskbError"]
