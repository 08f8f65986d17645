"""pava_b200 -- B200-native (sm_100a) SpMV engine behind pava's format/benchmark surface.

The CVR and CSR5 conversions and SpMV kernels run as hand-written CUDA (pava_b200/csrc),
reached through the C ABI in include/pava_gpu.h; host-side generators, Matrix Market I/O and
COO->CSR live in include/pava_host.h.  Build with ``python -m pava_b200.build``.
"""
from . import _abi  # noqa: F401
from .matrices import CSR  # noqa: F401

__all__ = ["CSR", "SpMatrix", "AnonymousLibHandle", "conduct_cvr", "conduct_csr5"]


def __getattr__(name):
    if name in ("SpMatrix", "AnonymousLibHandle", "conduct_cvr", "conduct_csr5"):
        from . import api
        return getattr(api, name)
    raise AttributeError(name)
